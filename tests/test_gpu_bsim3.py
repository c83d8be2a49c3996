"""The BSIM3v3 DC core (models/bsim3.va) on the GPU against the oracle and
against the reference's ngspice fixtures.

- Independent cold lanes of a BSIM3 inverter chain (every branch of the DC
  core: given and derived k1/k2 and vth0, RSH internal nodes, impact
  ionisation, poly depletion, MOBMOD 1-3), each lane with its own input
  voltage and DELVTO per device: the oracle's converged flag and exactly
  its Newton iteration count on every lane, values within 1e-9 relative or
  1e-12 absolute, and bitwise (the kernels and the oracle share one exp,
  log and pow, esl_math.h).
- Sequential sweep lanes of the same chain (each lane's transfer curve).
- The reference's operating-point fixtures, BSIM3 among them, as one cold
  GPU lane each, at the fixtures' tolerances.
The DC sweep fixtures of BSIM3 run through the generic golden tests of
test_gpu_dc.py (independent points) and test_gpu_sweep.py (sweep lanes).
"""

import numpy as np
import pytest

import golden_util as gu
import parity
from espice_b200 import decks, lanes
from netlist import Deck
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-9, 1e-12


def _close(a, b):
    return np.abs(a - b) <= ATOL + RTOL * np.maximum(np.abs(a), np.abs(b))


@pytest.mark.parametrize("seed", [1, 2])
def test_bsim3_lanes_match_oracle_cold(seed):
    fr, slots, values = decks.bsim3_inverters(seed=seed, lanes=256)
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=None)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    xg, itg, stg, stats = ctx.solve(x0=None)
    ctx.close()
    conv = stg == lanes.LANE_CONVERGED
    assert conv.all()
    bitwise = parity.assert_dc_parity(fr, slots, values, None, oracle.newton_opts(), xg, itg, conv, xo, ito, cvo,
                                      f"seed {seed}")
    assert bitwise == 1.0, f"{bitwise:.3f} of the lanes bitwise the oracle's"


def test_bsim3_lanes_match_oracle_tight():
    """reltol 1e-6: lanes converge to the same point whatever their path."""
    fr, slots, values = decks.bsim3_inverters(seed=3, lanes=128)
    opts = dict(reltol=1e-6, vntol=1e-9, abstol=1e-15)
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=None, opts=oracle.newton_opts(**opts))
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    xg, itg, stg, _ = ctx.solve(x0=None, opts=lanes.newton_opts(**opts))
    ctx.close()
    assert (stg == lanes.LANE_CONVERGED).all() and cvo.all()
    parity.assert_dc_parity(fr, slots, values, None, oracle.newton_opts(**opts), xg, itg,
                            stg == lanes.LANE_CONVERGED, xo, ito, cvo, "reltol 1e-6")


def test_bsim3_sweep_lanes_match_oracle():
    """32 lanes (DELVTO per device), each sweeping the chain's input 0..1.8 V
    over 37 points as the reference's sequential .dc does."""
    fr, slots, values = decks.bsim3_inverters(seed=4, lanes=32)
    src, dv, lane_vals = slots[0], slots[1:], values[:, 1:]
    pts = np.linspace(0.0, 1.8, 37)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(dv, lane_vals)
    x, it, cv, st, _ = ctx.sweep(src, pts)
    ctx.close()
    xo, ito, cvo = oracle.dc_sweep_lanes(fr, dv, lane_vals, src, pts)
    assert (st == lanes.SWEEP_DONE).all(), st
    assert np.array_equal(cv, cvo.astype(bool))
    assert cv.all()
    flips = np.argwhere(it != ito)
    assert len(flips) == 0, f"iteration counts differ at (lane, point) {flips[:10].tolist()}"
    assert _close(x, xo).all(), float(np.max(np.abs(x - xo)))


OP_FIXTURES = [n for n in gu.names() if n.split("__")[0] in ("op", "convergence", "stress")
               and Deck(gu.load(n)["deck"]).analysis[0] == "op"]


@pytest.mark.parametrize("name", OP_FIXTURES)
def test_op_fixtures_as_gpu_lane(name):
    """A reference operating-point fixture as one cold GPU lane at reltol
    1e-6: converged, and the fixture's values at its tolerances. Circuits
    whose working set exceeds a warp lane (the 32 x 32 resistor grid: 1,027
    unknowns, 22,568 tape values; the 257-section resistor chain) run on the
    block lanes."""
    g = gu.load(name)
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    opts = dict(deck.newton_opts(), reltol=1e-6)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes([], np.zeros((1, 1)))
    x, it, st, _ = ctx.solve(x0=None, opts=lanes.newton_opts(max_iter=100, **opts))
    ctx.close()
    assert st[0] == lanes.LANE_CONVERGED, (name, int(st[0]), int(it[0]))
    for col, worst, count in gu.score(g, fr, x[:1]):
        assert worst <= 1.0, f"{name} {col}: {worst:.3g}x the fixture tolerance"

"""GPU sequential .dc sweeps, one per lane (esl_dc_sweep_device), against
the oracle's restatement of the reference's sweep (dc.zig Sweep: the
MODEINITPRED predictor limited against the last point, a warm Newton, the
cold plain rung on failure) and against the reference's golden fixtures,
which ngspice produced by the same sequential sweep."""

import numpy as np
import pytest

import golden_util as gu
from espice_b200 import decks, lanes
from espice_b200.circuit import R, V
from netlist import Deck
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-9, 1e-12


def _close(a, b):
    return np.abs(a - b) <= ATOL + RTOL * np.maximum(np.abs(a), np.abs(b))


def test_sweep_lanes_match_oracle():
    """32 lanes, each with four grid resistors scaled by its own factors,
    each sweeping the source 0..5 V over 41 points."""
    fr, _, _ = decks.grid_diodes(seed=1, points=4)
    rs = fr.slots_of(R, "r")[:4]
    nominal = np.array([fr.param(s) for s in rs])
    rng = np.random.default_rng(5)
    lane_vals = nominal * np.exp(rng.uniform(-0.5, 0.5, size=(32, len(rs))))
    src = fr.slots_of(V, "dc")[0]
    pts = np.linspace(0.0, 5.0, 41)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(rs, lane_vals)
    x, it, cv, st, ms = ctx.sweep(src, pts)
    ctx.close()
    xo, ito, cvo = oracle.dc_sweep_lanes(fr, rs, lane_vals, src, pts)
    assert (st == lanes.SWEEP_DONE).all(), st
    assert np.array_equal(cv, cvo.astype(bool))
    assert cv.all()
    assert np.array_equal(it, ito)
    assert _close(x, xo).all(), float(np.max(np.abs(x - xo)))


def _gpu_sweep(fr, slot, values, opts):
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes([], np.zeros((1, 1)))
    x, it, cv, st, _ = ctx.sweep(slot, values, lanes.newton_opts(**opts))
    ctx.close()
    _gpu_sweep.status.append(int(st[0]))
    return x[0], it[0], cv[0]


def _oracle_sweep(fr, slot, values, opts):
    return oracle.dc_sweep(fr, slot, values, oracle.newton_opts(**opts))


def _op(fr, opts):
    return oracle.op(fr, oracle.newton_opts(max_iter=100, **opts))


# every DC sweep fixture, and the reference's ladder deck (a MOS1 latch whose
# sweep restarts cold three times)
DC_FIXTURES = [n for n in gu.names("dc__")] + ["convergence__bench_mos_latch_ladder"]

# Sweeps that cross into reverse breakdown need other pivots than the lead
# tape built at their first point: their lanes pause there and take the
# host's factor on their own direct solver (lane_solver.zig peels), then
# continue on the device where they stopped.
LEAVES_TAPE = {"dc__bench_ensemble_sweep_lanes", "dc__bench_power_zener_reg", "dc__device_diode_breakdown"}


@pytest.mark.parametrize("name", DC_FIXTURES)
def test_golden_fixtures_as_sweep_lanes(name):
    """Every reference DC sweep fixture as sweep lanes (one lane per outer
    value): the oracle's points, iterations and convergence, and the
    reference's golden values at its tolerances. The sweeps that leave the
    lead tape finish through host peels with the same results."""
    g = gu.load(name)
    _gpu_sweep.status = []
    fr, rows, conv = gu.solve_deck(g, _gpu_sweep, _op)
    fro, rows_o, conv_o = gu.solve_deck(g, _oracle_sweep, _op)
    assert all(s == lanes.SWEEP_DONE for s in _gpu_sweep.status)
    assert np.array_equal(conv.astype(bool), conv_o.astype(bool))
    assert conv.all()
    assert _close(rows, rows_o).all(), float(np.max(np.abs(rows - rows_o)))
    for col, worst, count in gu.score(g, fr, rows):
        assert worst <= 1.0, f"{name} {col}: {worst:.3g}x the fixture tolerance"


@pytest.mark.parametrize("name", sorted(LEAVES_TAPE))
def test_sweep_lanes_peel_and_match_oracle_exactly(name):
    """The sweeps that leave the lead tape: every point's iteration count and
    convergence equal to the oracle's per-lane sweep, the solutions bitwise."""
    g = gu.load(name)
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    an = deck.analysis
    from netlist import sweep_values
    pts = np.array(sweep_values(an[2], an[3], an[4]))
    slot = fr.slot(an[1], "dc")
    opts = deck.newton_opts()
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes([], np.zeros((2, 1)))
    x, it, cv, st, _ = ctx.sweep(slot, pts, lanes.newton_opts(**opts))
    ctx.close()
    assert (st == lanes.SWEEP_DONE).all()
    xo, ito, cvo = oracle.dc_sweep(fr, slot, pts, oracle.newton_opts(**opts))
    for lane in range(2):
        assert np.array_equal(cv[lane], cvo.astype(bool)), lane
        assert np.array_equal(it[lane], ito), (lane, np.flatnonzero(it[lane] != ito))
        assert np.array_equal(x[lane].view(np.uint64), xo.view(np.uint64)), lane


def test_sweep_lanes_cold_ladder():
    """The reference's ladder deck swept at 0.5 V steps, 16 lanes over the
    second bit line's bias: a warm point fails and its cold restart leaves
    plain Newton on four lanes, which finish the point through gmin stepping
    on the device (dc.zig's cold ladder); every lane's points, iteration
    counts and convergence exactly the oracle's."""
    g = gu.load("convergence__bench_mos_latch_ladder")
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    an = deck.analysis
    from netlist import sweep_values
    pts = np.array(sweep_values(an[2], an[3], 0.5))
    slot = fr.slot(an[1], "dc")
    opts = deck.newton_opts()
    lane_values = np.linspace(1.6, 2.4, 16).reshape(-1, 1)
    slots = [fr.slot("vdb", "dc")]
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, lane_values)
    x, it, cv, st, _ = ctx.sweep(slot, pts, lanes.newton_opts(**opts))
    ctx.close()
    assert (st == lanes.SWEEP_DONE).all()
    xo, ito, cvo = oracle.dc_sweep_lanes(fr, slots, lane_values, slot, pts, oracle.newton_opts(**opts))
    assert np.array_equal(cv, cvo.astype(bool))
    assert np.array_equal(it, ito), np.argwhere(it != ito)
    assert np.array_equal(x.view(np.uint64), xo.view(np.uint64))
    assert (it > 100).sum() >= 4, it.max()
    print(f"cold ladder points: {int((it > 100).sum())} of {it.size}, iterations up to {int(it.max())}")

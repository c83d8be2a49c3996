"""Operating-point lanes (esl_op_solve) against the oracle's restatement of
op.zig's ladder on the B200.

Every lane solves its operating point from the cold start: plain Newton
with MODEINITFIX, then (on the device, between Newton runs) dynamic gmin
stepping with ngspice's diagonal placement and the BSIM3 junction gmin
following the rung, the clean solve at the target, source stepping and the
full-source Newton. The contract is the plain form's: every lane's
convergence, rung, iteration count (summed over every run of the ladder)
and solution exactly the oracle's, converged or not.

- the analog block (498 unknowns, 120 BSIM3) from the cold start on the
  block lanes: about 4% of its points leave plain Newton and converge on
  gmin stepping;
- the reference's ladder deck (a MOS1 latch) on the warp lanes;
- with every Newton run capped at a few iterations (iter_cap, applied the
  same way on both sides), the rungs behind gmin stepping: source stepping,
  its back-offs to the last good lambda, the full-source Newton and lanes
  that end unconverged; on the warp and the block lanes, with lanes that
  pause for the host's factor in the middle of the ladder.
"""

import numpy as np
import pytest

import golden_util as gu
from espice_b200 import decks, lanes
from netlist import Deck, sweep_values
from oracle import oracle

pytestmark = pytest.mark.gpu


def _deck_points(name):
    g = gu.load(name)
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    an = deck.analysis
    values = np.array(sweep_values(an[2], an[3], an[4])).reshape(-1, 1)
    return fr, [fr.slot(an[1], "dc")], values, deck.newton_opts()


def _op(fr, slots, values, path=lanes.PATH_AUTO, iter_cap=0, opts=None):
    ctx = lanes.DcLanes(fr)
    ctx.set_mode(path=path)
    ctx.set_lanes(slots, values)
    x, it, st, rung, stats = ctx.op(lanes.newton_opts(max_iter=100, iter_cap=iter_cap, **(opts or {})))
    ctx.close()
    return x, it, st, rung, stats


def _check(fr, slots, values, path=lanes.PATH_AUTO, iter_cap=0, opts=None, label=""):
    x, it, st, rung, stats = _op(fr, slots, values, path, iter_cap, opts)
    xo, ito, cvo, rungo = oracle.op_points(fr, slots, values, oracle.newton_opts(max_iter=100, **(opts or {})),
                                           iter_cap=iter_cap)
    conv = st == lanes.LANE_CONVERGED
    assert np.array_equal(conv, cvo.astype(bool)), f"{label}: convergence differs on lanes {np.flatnonzero(conv != cvo)}"
    assert np.array_equal(rung, rungo), f"{label}: rungs differ on lanes {np.flatnonzero(rung != rungo)}"
    assert np.array_equal(it, ito), f"{label}: iterations differ on lanes {np.flatnonzero(it != ito)}"
    same = (x.view(np.uint64) == xo.view(np.uint64)).all(axis=1)
    assert same.all(), f"{label}: solutions differ on lanes {np.flatnonzero(~same)}"
    hist = np.bincount(rung, minlength=4)
    print(f"{label}: rungs plain/gmin/source/none {hist.tolist()}, iterations mean {it.mean():.1f} "
          f"max {it.max()}, path {stats['path']}, peeled {stats['peeled']}, {stats['kernel_ms']:.1f} ms")
    return hist, stats


def test_op_lanes_analog_block_gmin_stepping():
    """64 analog-block points from the cold start on the block lanes: the
    ones plain Newton leaves go through gmin stepping on the device."""
    fr, expand = decks.analog_block()
    params, _ = decks.analog_block_params(seed=11, points=64)
    values = expand(params)
    hist, stats = _check(fr, expand.slots, values, label="analog block")
    assert stats["path"] == lanes.PATH_BLOCK
    assert hist[lanes.RUNG_GMIN] > 0 and hist[lanes.RUNG_NONE] == 0


def test_op_lanes_mos1_latch():
    """The reference's ladder deck: every sweep value as a cold operating
    point on the warp lanes; three leave plain Newton."""
    fr, slots, values, opts = _deck_points("convergence__bench_mos_latch_ladder")
    hist, stats = _check(fr, slots, values, opts=opts, label="latch")
    assert stats["path"] == lanes.PATH_WARP
    assert hist[lanes.RUNG_GMIN] > 0


CAPPED = [
    ("dc__bench_power_zener_reg", 3, lanes.PATH_AUTO),
    ("dc__bench_power_zener_reg", 3, lanes.PATH_BLOCK),
    ("dc__bench_mosfet_cmos_inverter", 3, lanes.PATH_AUTO),
    ("dc__bench_mosfet_cmos_inverter", 4, lanes.PATH_BLOCK),
    ("dc__device_bsim3_transfer", 3, lanes.PATH_AUTO),
]


@pytest.mark.parametrize("name,cap,path", CAPPED)
def test_op_lanes_capped_runs_reach_every_rung(name, cap, path):
    """Every Newton run capped at a few iterations: lanes reach source
    stepping, its back-offs and the full-source Newton, or end unconverged;
    all of it the oracle's."""
    fr, slots, values, opts = _deck_points(name)
    hist, stats = _check(fr, slots, values, path=path, iter_cap=cap, opts=opts, label=f"{name} cap {cap}")
    assert hist[lanes.RUNG_SOURCE] + hist[lanes.RUNG_NONE] > 0


def test_op_lanes_analog_block_capped():
    """The analog block with every run capped at 5 iterations (every lane
    walks the whole gmin descent with its back-offs) and at 3 (every lane
    ends unconverged after all rungs) on the block lanes."""
    fr, expand = decks.analog_block()
    params, _ = decks.analog_block_params(seed=11, points=32)
    values = expand(params)
    hist, _ = _check(fr, expand.slots, values, iter_cap=5, label="analog block cap 5")
    assert hist[lanes.RUNG_GMIN] == len(values)
    hist, _ = _check(fr, expand.slots, values, iter_cap=3, label="analog block cap 3")
    assert hist[lanes.RUNG_NONE] == len(values)

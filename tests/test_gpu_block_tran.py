"""Transient lanes on the block lanes (a CTA per lane, block.cu
tran_block_kernel) on the B200.

The block form runs the warp lanes' transient step for step: the same
operating point (op.zig's ladder), predictor, companion, LTE control, order
promotion and breakpoints, the Newton solves on the block programs. So:
- on decks the warp lanes also hold, every lane's step statistics and
  final solution equal the warp lanes' bit for bit, and the recorded
  waveforms too;
- the reference's transient fixtures as block lanes keep the oracle's step
  decisions and waveforms and the ngspice waveform at the fixture's
  tolerances;
- a circuit beyond the warp lanes (the 257-section RC ladder) runs with the
  oracle's step decisions.
"""

import numpy as np
import pytest

import golden_util as gu
from espice_b200 import decks, lanes
from espice_b200.circuit import Circuit
from netlist import Deck
from oracle import oracle

pytestmark = pytest.mark.gpu

DECISIONS = ["status", "accepted", "attempts", "rej_newton", "rej_lte", "bp_landings", "op_iters", "nr_iters"]


def _close(a, b, rtol=1e-9, atol=1e-12):
    return np.abs(a - b) <= atol + rtol * np.maximum(np.abs(a), np.abs(b))


def _tran(fr, slots, values, go, probes, max_pts, path):
    ctx = lanes.DcLanes(fr)
    ctx.set_mode(path=path)
    ctx.set_lanes(slots, values)
    res = ctx.tran(go, probes, max_pts)
    ctx.close()
    return res


def _check_oracle(g, o):
    tg, vg, ng, sg, xg, _ = g
    to, vo, no, so, xo = o
    for k, name in enumerate(lanes.TS_FIELDS):
        if name in DECISIONS:
            assert np.array_equal(sg[:, k], so[:, k]), f"{name}: gpu {sg[:, k]} oracle {so[:, k]}"
    assert np.array_equal(ng, no)
    for lane in range(len(ng)):
        n = int(ng[lane])
        assert _close(tg[lane, :n], to[lane, :n], atol=0.0).all()
        assert _close(vg[lane, :n], vo[lane, :n]).all()
    assert _close(xg, xo).all()


def test_ring_block_equals_warp_bitwise():
    """Four ring-oscillator lanes over 0.3 ns on both lane shapes."""
    fr, slots, values = decks.ring_oscillator(lanes=4)
    go = lanes.tran_opts(3e-10, decks.RING_T_STEP, decks.RING_T_MAX, max_steps=100_000)
    probes = [fr.unknown("v(s0)"), fr.unknown("v(s15)")]
    w = _tran(fr, slots, values, go, probes, 2000, lanes.PATH_WARP)
    b = _tran(fr, slots, values, go, probes, 2000, lanes.PATH_BLOCK)
    assert np.array_equal(b[3], w[3]), (b[3], w[3])
    assert np.array_equal(b[2], w[2])
    assert np.array_equal(b[4].view(np.uint64), w[4].view(np.uint64))
    for lane in range(4):
        n = int(b[2][lane])
        assert np.array_equal(b[0][lane, :n], w[0][lane, :n])
        assert np.array_equal(b[1][lane, :n].view(np.uint64), w[1][lane, :n].view(np.uint64))
    assert (b[3][:, 0] == lanes.TRAN_DONE).all()


TRAN_FIXTURES = [n for n in gu.names("tran__") if gu.load(n)["plots"]]


@pytest.mark.parametrize("name", TRAN_FIXTURES)
def test_golden_transients_as_block_lanes(name):
    g = gu.load(name)
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    cols = list(g["plots"][0]["columns"])
    probes = [fr.unknown(c) for c in cols]
    _, tstep, tstop, tstart, tmax = deck.analysis
    opts = deck.newton_opts()
    go = lanes.tran_opts(tstop, tstep, tmax, max_steps=200_000, **opts)
    oo = oracle.tran_opts(tstop, tstep, tmax, max_steps=200_000, **opts)
    values = np.zeros((2, 1))
    res_b = _tran(fr, [], values, go, probes, 60_000, lanes.PATH_BLOCK)
    res_o = oracle.tran(fr, [], values, oo, probes, 60_000)
    _check_oracle(res_b, res_o)
    tg, vg, ng, sg, _, _ = res_b
    assert (sg[:, 0] == lanes.TRAN_DONE).all()
    n = int(ng[0])
    for col, worst in gu.score_tran(g, tg[0, :n], vg[0, :n], cols):
        assert worst <= 1.0, f"{name} {col}: {worst:.3g}x the fixture tolerance"


def test_rc_ladder_beyond_the_warp_lanes():
    """A 257-section RC ladder driven by a PULSE (259 unknowns: beyond a
    warp lane), eight lanes over its section resistance, on the block
    lanes: the oracle's step decisions, waveforms and final solutions."""
    c = Circuit()
    c.V("vin", "n0", "0", pulse=(0.0, 1.0, 1e-10, 5e-11, 5e-11, 1e-9, 4e-9))
    for k in range(257):
        c.R(f"r{k}", f"n{k}", f"n{k + 1}", 100.0)
        c.C(f"c{k}", f"n{k + 1}", "0", 1e-15)
    fr = c.freeze()
    assert fr.n > 256
    slots = [fr.slot("r0", "r")]
    values = np.linspace(50.0, 400.0, 8).reshape(-1, 1)
    probes = [fr.unknown("v(n1)"), fr.unknown("v(n128)"), fr.unknown("v(n257)")]
    go = lanes.tran_opts(2e-9, 2e-11, 0.0, max_steps=100_000)
    oo = oracle.tran_opts(2e-9, 2e-11, 0.0, max_steps=100_000)
    res_b = _tran(fr, slots, values, go, probes, 20_000, lanes.PATH_AUTO)
    res_o = oracle.tran(fr, slots, values, oo, probes, 20_000)
    _check_oracle(res_b, res_o)
    assert (res_b[3][:, 0] == lanes.TRAN_DONE).all()
    print(f"rc ladder: {int(res_b[3][0, 1])} accepted steps a lane, {res_b[5]:.1f} ms")


def test_digital_block_20k_unknowns():
    """The large transient configuration's circuit (20,001 unknowns, 2,000
    BSIM3 MOSFETs in NAND2 cells on an RC mesh, PWL inputs with 50 ps edges)
    as two block lanes with per-device threshold shifts over its first
    100 ps: the oracle's step decisions and final solutions."""
    fr, slots = decks.digital_block()
    values = decks.digital_block_vto(len(slots), 2)
    probes = [fr.unknown("v(m0)")]
    go = lanes.tran_opts(1e-10, 1e-11, 0.0, max_steps=100_000)
    oo = oracle.tran_opts(1e-10, 1e-11, 0.0, max_steps=100_000)
    res_b = _tran(fr, slots, values, go, probes, 1000, lanes.PATH_AUTO)
    res_o = oracle.tran(fr, slots, values, oo, probes, 1000)
    _check_oracle(res_b, res_o)
    assert (res_b[3][:, 0] == lanes.TRAN_DONE).all()
    print(f"digital block: {int(res_b[3][0, 1])} steps, {int(res_b[3][0, 3])} Newton iterations a lane, "
          f"{res_b[5]:.0f} ms for 2 lanes")


def _tran_mixed(fr, slots, values, go, probes, max_pts, refine_skip):
    ctx = lanes.DcLanes(fr)
    ctx.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK, refine_skip=refine_skip)
    ctx.set_lanes(slots, values)
    res = ctx.tran(go, probes, max_pts)
    corrections = ctx.tran_refinements()
    ctx.close()
    return res, corrections


def _mixed_decks():
    """(name, circuit, slots, values, t_stop, t_step, probes): a linear RC
    ladder beyond the warp lanes and a nonlinear BSIM3 inverter chain."""
    c = Circuit()
    c.V("vin", "n0", "0", pulse=(0.0, 1.0, 1e-10, 5e-11, 5e-11, 1e-9, 4e-9))
    for k in range(257):
        c.R(f"r{k}", f"n{k}", f"n{k + 1}", 100.0)
        c.C(f"c{k}", f"n{k + 1}", "0", 1e-15)
    ladder = c.freeze()
    yield ("rc_ladder", ladder, [ladder.slot("r0", "r")], np.linspace(50.0, 400.0, 8).reshape(-1, 1), 2e-9, 2e-11,
           [ladder.unknown("v(n1)"), ladder.unknown("v(n257)")])
    fr, slots, values = decks.bsim3_inverters(seed=5, stages=4, lanes=8, c_load=20e-15,
                                              pulse=[0.0, 1.8, 0.1e-9, 50e-12, 50e-12, 0.4e-9, 1e-9])
    yield ("bsim3_chain", fr, slots[1:], values[:, 1:], 2e-9, 10e-12, [fr.unknown("v(s0)"), fr.unknown("v(s3)")])


@pytest.mark.parametrize("case", list(range(2)))
def test_mixed_block_transient_against_oracle(case):
    """Mixed-precision block transient lanes (FP32 refactor and solves, every
    Newton step refined in FP64 on the FP64 residual to 1e-12 of it;
    evaluation, the companion, the gates and the LTE control in FP64): the
    oracle's (FP64) step decisions on every lane, and waveforms and final
    solutions within 1e-9 relative or 1e-12 absolute."""
    name, fr, slots, values, t_stop, t_step, probes = list(_mixed_decks())[case]
    go = lanes.tran_opts(t_stop, t_step, 0.0, max_steps=100_000)
    oo = oracle.tran_opts(t_stop, t_step, 0.0, max_steps=100_000)
    res_m, corrections = _tran_mixed(fr, slots, values, go, probes, 20_000, 0.0)
    res_o = oracle.tran(fr, slots, values, oo, probes, 20_000)
    assert (res_m[3][:, 0] == lanes.TRAN_DONE).all()
    _check_oracle(res_m, res_o)
    nr = int(res_m[3][:, lanes.TS_FIELDS.index("nr_iters")].sum())
    assert corrections > 0
    print(f"{name}: {fr.n} unknowns, {int(res_m[3][0, 1])} steps a lane, "
          f"{corrections / nr:.2f} FP64 corrections a Newton iteration")


def test_mixed_block_transient_refining_near_convergence():
    """The mixed block transient with refine_skip (steps farther than 1e3
    tolerances from convergence taken unrefined): every lane finishes, the
    accepted step counts stay the oracle's and the final solutions are
    within 1e-9 relative or 1e-12 absolute of it (an unrefined step only
    moves an iterate the next iteration corrects)."""
    name, fr, slots, values, t_stop, t_step, probes = list(_mixed_decks())[1]
    go = lanes.tran_opts(t_stop, t_step, 0.0, max_steps=100_000)
    oo = oracle.tran_opts(t_stop, t_step, 0.0, max_steps=100_000)
    (tg, vg, ng, sg, xg, _), corrections = _tran_mixed(fr, slots, values, go, probes, 20_000, 1e3)
    to, vo, no, so, xo = oracle.tran(fr, slots, values, oo, probes, 20_000)
    assert (sg[:, 0] == lanes.TRAN_DONE).all()
    acc = lanes.TS_FIELDS.index("accepted")
    assert np.array_equal(sg[:, acc], so[:, acc])
    assert _close(xg, xo).all(), float(np.max(np.abs(xg - xo)))
    nr = int(sg[:, lanes.TS_FIELDS.index("nr_iters")].sum())
    print(f"{name}: {corrections / nr:.2f} FP64 corrections a Newton iteration with refine_skip 1e3")

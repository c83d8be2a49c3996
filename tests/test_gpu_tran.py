"""GPU transient lanes against the CPU oracle (B200).

Each lane runs its operating point and its whole trapezoidal transient in one
launch. Parity with the oracle's restatement of the reference's step control
(src/analysis/tran/tran.zig Sim): the same step decisions (accepted steps,
attempts, Newton and LTE rejections, breakpoint landings, Newton iterations),
the accepted time grid and the recorded waveforms within 1e-9 relative or
1e-12 absolute, and the reference's ngspice golden waveform at its own
tolerances.
"""

import numpy as np
import pytest

import golden_util as gu
from espice_b200 import decks, lanes
from espice_b200.circuit import M
from netlist import Deck
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-9, 1e-12
DECISIONS = ["status", "accepted", "attempts", "rej_newton", "rej_lte", "bp_landings", "op_iters", "nr_iters"]


def _close(a, b, rtol=RTOL, atol=ATOL):
    return np.abs(a - b) <= atol + rtol * np.maximum(np.abs(a), np.abs(b))


def _run_both(fr, slots, values, tstop, tstep, tmax=0.0, probes=(), max_pts=0):
    go = lanes.tran_opts(tstop, tstep, tmax, max_steps=200_000)
    oo = oracle.tran_opts(tstop, tstep, tmax, max_steps=200_000)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    g = ctx.tran(go, probes, max_pts)
    ctx.close()
    o = oracle.tran(fr, slots, values, oo, probes, max_pts)
    return g, o


def _check_parity(g, o):
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


def test_mos1_inverter_transient_one_lane():
    g = gu.load("tran__device_mos1_large_signal")
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    cols = list(g["plots"][0]["columns"])
    probes = [fr.unknown(c) for c in cols]
    _, tstep, tstop = deck.analysis[:3]
    res_g, res_o = _run_both(fr, [], np.zeros((1, 1)), tstop, tstep, probes=probes, max_pts=4000)
    _check_parity(res_g, res_o)
    tg, vg, ng, sg, _, _ = res_g
    assert sg[0, 0] == lanes.TRAN_DONE
    n = int(ng[0])
    for col, worst in gu.score_tran(g, tg[0, :n], vg[0, :n], cols):
        assert worst <= 1.0, f"{col}: {worst:.3g}x the fixture tolerance"


def test_mos1_inverter_transient_lanes_vary_threshold():
    """Eight lanes, each with its own NMOS and PMOS VTO."""
    g = gu.load("tran__device_mos1_large_signal")
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    slots = fr.slots_of(M, "vto")
    nominal = np.array([fr.param(s) for s in slots])
    rng = np.random.default_rng(7)
    values = nominal + rng.normal(0.0, 0.05, size=(8, len(slots)))
    probes = [fr.unknown("v(out)")]
    _, tstep, tstop = deck.analysis[:3]
    res_g, res_o = _run_both(fr, slots, values, tstop, tstep, probes=probes, max_pts=4000)
    _check_parity(res_g, res_o)
    assert (res_g[3][:, 0] == lanes.TRAN_DONE).all()


def test_ring_oscillator_short_window():
    """Sixteen ring-oscillator samples over the first 2 ns (about 2,000
    steps each, the supply ramp and the escape from the metastable point)."""
    fr, slots, values = decks.ring_oscillator(lanes=16)
    probes = [fr.unknown("v(s0)"), fr.unknown("v(s15)")]
    res_g, res_o = _run_both(fr, slots, values, 2e-9, decks.RING_T_STEP, decks.RING_T_MAX, probes=probes,
                             max_pts=2500)
    _check_parity(res_g, res_o)
    assert (res_g[3][:, 0] == lanes.TRAN_DONE).all()


def test_ring_oscillator_headline_window():
    """The bench's headline workload at its own window: 64 of its 1,024
    Monte-Carlo ring samples (seed 1, every 16th lane), each over the full
    20 ns with the 1 ps maximum step (about 20,000 accepted steps and 40,000
    Newton iterations a lane). Every step decision equal to the oracle's
    (accepted steps, attempts, Newton and LTE rejections, breakpoint
    landings, operating-point and transient Newton iterations) and the final
    solution within 1e-9 relative or 1e-12 absolute. The oracle's lanes run on
    all host threads."""
    import concurrent.futures as cf
    import os

    fr, slots, values = decks.ring_oscillator(seed=1, lanes=1024)
    values = values[::16]
    go = lanes.tran_opts(decks.RING_T_STOP, decks.RING_T_STEP, decks.RING_T_MAX, max_steps=200_000)
    oo = oracle.tran_opts(decks.RING_T_STOP, decks.RING_T_STEP, decks.RING_T_MAX, max_steps=200_000)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    _, _, _, sg, xg, _ = ctx.tran(go)
    ctx.close()

    def one(i):
        _, _, _, so, xo = oracle.tran(fr, slots, values[i:i + 1], oo)
        return so[0], xo[0]

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        res = list(ex.map(one, range(len(values))))
    so = np.stack([r[0] for r in res])
    xo = np.stack([r[1] for r in res])
    for k, name in enumerate(lanes.TS_FIELDS):
        if name in DECISIONS:
            bad = np.flatnonzero(sg[:, k] != so[:, k])
            assert len(bad) == 0, f"{name} differs on lanes {bad}: gpu {sg[bad, k]} oracle {so[bad, k]}"
    assert (sg[:, 0] == lanes.TRAN_DONE).all()
    assert (sg[:, 1] > 15_000).all(), sg[:, 1]
    assert _close(xg, xo).all(), float(np.max(np.abs(xg - xo)))


def test_source_waves_vary_per_lane():
    """An RC network driven by a SIN, an EXP and a PWL voltage source and a
    PWL current source, twelve lanes each with its own wave parameters (SIN
    amplitude and frequency, EXP time constant, PWL corner values and a
    shifted PWL delay): the oracle's step decisions, breakpoint landings
    included (each lane's own PWL corners), and its waveforms."""
    from espice_b200.circuit import Circuit, I, V
    c = Circuit()
    c.V("vs", "a", "0", dc=0.0, sin=[0.2, 1.0, 5e8, 0.0, 1e7, 30.0])
    c.V("ve", "b", "0", dc=0.0, exp=[0.0, 1.5, 1e-10, 4e-10, 1.2e-9, 3e-10])
    c.V("vp", "c", "0", dc=0.0, pwl=([0.0, 3e-10, 7e-10, 1.1e-9, 1.6e-9], [0.0, 1.0, 1.0, -0.5, 0.2], -1.0, 0.0))
    c.I("ip", "0", "d", dc=0.0, pwl=([0.0, 2e-10, 9e-10], [0.0, 1e-3, -5e-4], -1.0, 1e-10))
    c.R("r1", "a", "x", 1e3)
    c.R("r2", "b", "x", 2e3)
    c.R("r3", "c", "x", 1.5e3)
    c.R("r4", "d", "x", 500.0)
    c.C("c1", "x", "0", 1e-13)
    c.R("r5", "d", "0", 3e3)
    c.C("c2", "d", "0", 5e-14)
    fr = c.freeze()
    slots = [fr.slot("vs", "v2"), fr.slot("vs", "td"), fr.slot("ve", "tr"), fr.slot("vp", "pwl_v1"),
             fr.slot("vp", "pwl_v3"), fr.slot("ip", "td")]
    rng = np.random.default_rng(11)
    lanes_n = 12
    values = np.stack([rng.uniform(0.5, 1.5, lanes_n), rng.uniform(3e8, 9e8, lanes_n),
                       rng.uniform(2e-10, 6e-10, lanes_n), rng.uniform(0.5, 1.5, lanes_n),
                       rng.uniform(-1.0, 0.0, lanes_n), rng.uniform(0.0, 3e-10, lanes_n)], axis=1)
    probes = [fr.unknown("v(x)"), fr.unknown("v(d)")]
    res_g, res_o = _run_both(fr, slots, values, 2e-9, 1e-11, 2e-11, probes=probes, max_pts=4000)
    _check_parity(res_g, res_o)
    assert (res_g[3][:, 0] == lanes.TRAN_DONE).all()
    assert (res_g[3][:, 6] >= 4).all()  # every lane landed on its PWL corners


TRAN_FIXTURES = [n for n in gu.names("tran__") if gu.load(n)["plots"]]


@pytest.mark.parametrize("name", TRAN_FIXTURES)
def test_golden_transients_as_gpu_lanes(name):
    """Every reference transient fixture as GPU lanes at the deck's own
    options and .tran card (TMAX included): the oracle's step decisions and
    waveforms, and the reference's ngspice waveform at its tolerances."""
    g = gu.load(name)
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    cols = list(g["plots"][0]["columns"])
    probes = [fr.unknown(c) for c in cols]
    _, tstep, tstop, tstart, tmax = deck.analysis
    assert tstart == 0.0
    opts = deck.newton_opts()
    go = lanes.tran_opts(tstop, tstep, tmax, max_steps=200_000, **opts)
    oo = oracle.tran_opts(tstop, tstep, tmax, max_steps=200_000, **opts)
    values = np.zeros((2, 1))
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes([], values)
    res_g = ctx.tran(go, probes, 60_000)
    ctx.close()
    res_o = oracle.tran(fr, [], values, oo, probes, 60_000)
    _check_parity(res_g, res_o)
    tg, vg, ng, sg, _, _ = res_g
    assert (sg[:, 0] == lanes.TRAN_DONE).all()
    n = int(ng[0])
    for col, worst in gu.score_tran(g, tg[0, :n], vg[0, :n], cols):
        assert worst <= 1.0, f"{name} {col}: {worst:.3g}x the fixture tolerance"


def test_mos1_tox_runs_dc_and_refuses_transient():
    """MOS1 with TOX: the DC lanes solve (KP from U0 and TOX) and match the
    oracle; a transient is refused with ESL_NOT_ELIGIBLE, as the oracle
    refuses it (the bias-dependent Meyer halves are not built)."""
    from espice_b200.circuit import Circuit
    c = Circuit()
    c.V("vdd", "d", "0", dc=1.8)
    c.V("vg", "g", "0", dc=1.2)
    c.M("m1", "d", "g", "0", "0", type=1.0, vto=0.5, tox=20e-9, u0=400.0, w=2e-6, l=1e-6)
    fr = c.freeze()
    slot = fr.slot("vg", "dc")
    values = np.linspace(0.0, 1.8, 64).reshape(-1, 1)
    xo, ito, cvo = oracle.dc_points(fr, [slot], values, warm=None)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes([slot], values)
    x, it, st, _ = ctx.solve(x0=None)
    assert np.array_equal(st == lanes.LANE_CONVERGED, cvo.astype(bool)) and cvo.all()
    assert _close(x, xo).all()
    with pytest.raises(lanes.LaneError) as e:
        ctx.tran(lanes.tran_opts(1e-9, 1e-11))
    assert e.value.code == lanes.ESL_NOT_ELIGIBLE
    ctx.close()


def test_bsim3_inverter_chain_transient_lanes():
    """Eight lanes of a 4-stage BSIM3 inverter chain (20 fF per output, a
    PULSE input, each lane with its own DELVTO per device) through the BSIM3
    instantiation of the transient kernel: the oracle's step decisions,
    waveform and end state."""
    fr, slots, values = decks.bsim3_inverters(seed=5, stages=4, lanes=8, c_load=20e-15,
                                              pulse=[0.0, 1.8, 0.1e-9, 50e-12, 50e-12, 0.4e-9, 1e-9])
    probes = [fr.unknown("v(s0)"), fr.unknown("v(s3)")]
    res_g, res_o = _run_both(fr, slots[1:], values[:, 1:], 2e-9, 10e-12, probes=probes, max_pts=4000)
    _check_parity(res_g, res_o)
    assert (res_g[3][:, 0] == lanes.TRAN_DONE).all()


ZENER_TRAN = """* the reference's shunt regulator (power/zener_reg) driven by a supply ramp
Vsupply sup 0 PULSE(6 18 10n 200n 200n 200n 1u)
Rseries sup out 220
Dz out ref DZ
Vref ref 0 DC 5.1
Rload out 0 1k
Cout out 0 100p
.model DZ D(IS=1e-12 N=1)
.tran 1n 600n
.end
"""


def test_lanes_that_leave_the_tape_are_peeled():
    """The reference's shunt regulator with its supply ramped from 6 to 18 V
    and back (the ramp its DC sweep takes, whose breakdown points leave the
    lead pivot tape): the transient lanes that leave the tape pause, take the
    host's factor and resume, and every lane keeps the oracle's step
    decisions and waveforms."""
    deck = Deck(ZENER_TRAN)
    fr = deck.circuit().freeze()
    slots = [fr.slot("rseries", "r")]
    values = np.linspace(150.0, 330.0, 6).reshape(-1, 1)
    probes = [fr.unknown("v(out)")]
    go = lanes.tran_opts(600e-9, 1e-9, 0.0, max_steps=200_000)
    oo = oracle.tran_opts(600e-9, 1e-9, 0.0, max_steps=200_000)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    g = ctx.tran(go, probes, 5_000)
    peeled, solves, launches = ctx.peel_counts()
    ctx.close()
    o = oracle.tran(fr, slots, values, oo, probes, 5_000)
    print(f"peeled lanes {peeled}, host solves {solves}, launches {launches}")
    _check_parity(g, o)
    assert (g[3][:, 0] == lanes.TRAN_DONE).all()
    assert peeled > 0 and launches > 1


def test_operating_point_takes_the_ladder():
    """The reference's ladder deck (a MOS1 latch) as transient lanes over its
    swept drain bias: the operating points that plain Newton leaves
    (op.solve with tran_op) converge through gmin stepping inside the
    transient lane, with the oracle's iteration sums, step decisions and
    waveforms."""
    g = gu.load("convergence__bench_mos_latch_ladder")
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    from netlist import sweep_values
    an = deck.analysis
    slots = [fr.slot("vd", "dc")]
    values = np.array(sweep_values(an[2], an[3], an[4])).reshape(-1, 1)
    probes = [fr.unknown("v(q)"), fr.unknown("v(qb)")]
    go = lanes.tran_opts(1e-9, 1e-10, 1e-10)
    oo = oracle.tran_opts(1e-9, 1e-10, 1e-10)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    res_g = ctx.tran(go, probes, 200)
    ctx.close()
    res_o = oracle.tran(fr, slots, values, oo, probes, 200)
    _check_parity(res_g, res_o)
    sg = res_g[3]
    op_iters = sg[:, lanes.TS_FIELDS.index("op_iters")]
    assert np.array_equal(op_iters, res_o[3][:, lanes.TS_FIELDS.index("op_iters")])
    assert (sg[:, 0] == lanes.TRAN_DONE).all()
    assert (op_iters > 100).sum() >= 3, op_iters

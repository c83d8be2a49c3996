"""GPU streamed transient measures (esl_tran_meas_device) against the
oracle's restatement of the reference's .meas evaluation (measure.zig Cross
and At, after ngspice com_measure2.c) and its early stop (tran.zig
:1057-1064): the same step statistics (so the same early stops) and card
values within 1e-9 relative (the waveforms agree to that, their device-model
arithmetic differing from the CPU's in the last bits)."""

import numpy as np
import pytest

import golden_util as gu
from espice_b200 import decks, lanes
from netlist import Deck
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-9, 1e-15


def _same(a, b):
    both_nan = np.isnan(a) & np.isnan(b)
    close = np.abs(a - b) <= ATOL + RTOL * np.maximum(np.abs(a), np.abs(b))
    return both_nan | close


def _cards(fr, mod):
    s0, s5 = fr.unknown("v(s0)"), fr.unknown("v(s5)")
    return [
        mod.Measure(mod.MEAS_TRIG_TARG, 0, mod.meas_clause(s0, val=0.9, rise=2),
                    mod.meas_clause(s0, val=0.9, rise=3)),
        mod.Measure(mod.MEAS_TRIG_TARG, 0, mod.meas_clause(s0, val=0.9, cross=3),
                    mod.meas_clause(s5, val=0.9, cross=3)),
        mod.Measure(mod.MEAS_WHEN, 0, mod.meas_clause(s0, val=0.9, fall=1, td=0.2e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_WHEN, 0, mod.meas_clause(s5, val=0.5, cross=mod.MEAS_LAST), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_FIND_AT, 0, mod.meas_clause(s5, at=0.37e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_WHEN, 0, mod.meas_clause(s0, val=0.9, rise=1, from_=0.5e-9, to=1.5e-9),
                    mod.meas_clause(0)),
        mod.Measure(mod.MEAS_MAX, 0, mod.meas_clause(s0, from_=1e-9, to=2e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_MIN, 0, mod.meas_clause(s5, from_=0.5e-9, to=2.5e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_AVG, 0, mod.meas_clause(s0, from_=1e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_PP, 0, mod.meas_clause(s5, from_=1e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_INTEG, 0, mod.meas_clause(s0, from_=0.3e-9, to=2.2e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_RMS, 0, mod.meas_clause(s5, from_=0.5e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_DERIV, 0, mod.meas_clause(s0, at=1.1e-9), mod.meas_clause(0)),
    ]


@pytest.mark.parametrize("early", [False, True])
def test_ring_measures_match_oracle(early):
    """24 ring-oscillator samples over 3 ns: a period, a stage delay, a
    delayed fall, a LAST crossing, a FIND, a windowed rise, MAX, MIN, AVG
    and PP over windows, a windowed INTEGRAL, an RMS and a DERIVATIVE."""
    fr, slots, values = decks.ring_oscillator(lanes=24)
    go = lanes.tran_opts(3e-9, decks.RING_T_STEP, decks.RING_T_MAX, max_steps=200_000)
    oo = oracle.tran_opts(3e-9, decks.RING_T_STEP, decks.RING_T_MAX, max_steps=200_000)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    vg, sg, xg, _ = ctx.tran_meas(go, _cards(fr, lanes), early_stop=early)
    ctx.close()
    vo, so, xo = oracle.tran_meas(fr, slots, values, oo, _cards(fr, oracle), early_stop=early)
    assert np.array_equal(sg, so), (sg[:, :3], so[:, :3])
    same = _same(vg, vo)
    assert same.all(), (vg[~same], vo[~same])
    assert np.isfinite(vg[:, 0]).any()
    if early:
        # the LAST card resolves only at the end, so no lane stops early
        assert not (sg[:, 0] == lanes.TRAN_RESOLVED).any()


def test_early_stop_ends_lanes():
    """The period card alone: lanes that oscillate stop once it resolves,
    with the same step counts and value as the oracle."""
    fr, slots, values = decks.ring_oscillator(lanes=16)
    s0 = fr.unknown("v(s0)")
    go = lanes.tran_opts(5e-9, decks.RING_T_STEP, decks.RING_T_MAX, max_steps=200_000)
    oo = oracle.tran_opts(5e-9, decks.RING_T_STEP, decks.RING_T_MAX, max_steps=200_000)
    card_g = [lanes.trig_targ(lanes.meas_clause(s0, val=0.9, rise=2), lanes.meas_clause(s0, val=0.9, rise=3))]
    card_o = [oracle.Measure(oracle.MEAS_TRIG_TARG, 0, oracle.meas_clause(s0, val=0.9, rise=2),
                             oracle.meas_clause(s0, val=0.9, rise=3))]
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    vg, sg, _, _ = ctx.tran_meas(go, card_g, early_stop=True)
    ctx.close()
    vo, so, _ = oracle.tran_meas(fr, slots, values, oo, card_o, early_stop=True)
    assert np.array_equal(sg, so)
    assert _same(vg, vo).all()
    resolved = sg[:, 0] == lanes.TRAN_RESOLVED
    assert resolved.any()
    assert (np.isfinite(vg[resolved, 0])).all()


MEAS_FIXTURES = [n for n in gu.names("tran__") if gu.load(n).get("checks")]


@pytest.mark.parametrize("name", MEAS_FIXTURES)
def test_golden_measures_as_gpu_lanes(name):
    """A transient fixture's .meas cards on the device: the oracle's values
    and ngspice's printed ones at the fixture's tolerance."""
    g = gu.load(name)
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    tstop, tstep, tmax, kw = gu.tran_options(deck)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes([], np.zeros((2, 1)))
    vg, sg, _, _ = ctx.tran_meas(lanes.tran_opts(tstop, tstep, tmax, max_steps=2_000_000, **kw),
                                 gu.measure_cards(deck, fr, lanes))
    ctx.close()
    values_o, so = gu.solve_meas(g)
    vo = np.array([values_o[m["name"]] for m in deck.measures])
    assert (sg[:, 0] == lanes.TRAN_DONE).all()
    assert np.array_equal(sg[0], so)
    assert _same(vg[0], vo).all() and _same(vg[1], vo).all()
    values = {m["name"]: float(vg[0, k]) for k, m in enumerate(deck.measures)}
    for nm, worst in gu.score_meas(g, values):
        assert worst <= 1.0, f"{name} {nm}: {worst:.3g}x the fixture tolerance"


def test_integral_rms_derivative_on_rc_lanes():
    """16 RC charging lanes (R from 0.5 to 2 kohm, 1 nF, a 1 V step; the
    reference's hspice/meas_forms deck without its E source): INTEGRAL over
    0..5 us and over the whole run, DERIVATIVE at 1 us, RMS over 1..2 us,
    against the oracle."""
    from espice_b200.circuit import Circuit
    c = Circuit()
    c.V("v1", "in", "0", pulse=[0.0, 1.0, 0.0, 1e-12, 1e-12, 1.0, 2.0])
    c.R("r1", "in", "out", 1e3)
    c.C("c1", "out", "0", 1e-9)
    fr = c.freeze()
    out = fr.unknown("v(out)")
    slots = [fr.slot("r1", "r")]
    values = np.linspace(500.0, 2000.0, 16).reshape(-1, 1)

    def cards(mod):
        cl = mod.meas_clause
        return [mod.Measure(mod.MEAS_INTEG, 0, cl(out, from_=0.0, to=5e-6), cl(0)),
                mod.Measure(mod.MEAS_INTEG, 0, cl(out), cl(0)),
                mod.Measure(mod.MEAS_DERIV, 0, cl(out, at=1e-6), cl(0)),
                mod.Measure(mod.MEAS_RMS, 0, cl(out, from_=1e-6, to=2e-6), cl(0))]

    go = lanes.tran_opts(5e-6, 10e-9, 0.0, max_steps=200_000)
    oo = oracle.tran_opts(5e-6, 10e-9, 0.0, max_steps=200_000)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    vg, sg, _, _ = ctx.tran_meas(go, cards(lanes))
    ctx.close()
    vo, so, _ = oracle.tran_meas(fr, slots, values, oo, cards(oracle))
    assert np.array_equal(sg, so)
    same = _same(vg, vo)
    assert same.all(), (vg[~same], vo[~same])
    assert np.isfinite(vg).all()

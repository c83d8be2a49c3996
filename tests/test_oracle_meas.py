"""The oracle's streamed window measures (MIN, MAX, AVG, PP over FROM..TO,
measure.zig Extremum) against the same rules applied with numpy to the
oracle's own recorded waveform: the samples inside the window, the last
sample reaching the extreme, AVG the trapezoidal sum over the samples'
span."""

import numpy as np

from espice_b200 import decks
from oracle import oracle


def test_window_measures_follow_the_recorded_waveform():
    fr, slots, values = decks.ring_oscillator(lanes=2)
    s0 = fr.unknown("v(s0)")
    o = oracle.tran_opts(1e-9, decks.RING_T_STEP, decks.RING_T_MAX)
    t, v, npts, st, _ = oracle.tran(fr, slots, values, o, [s0], 100_000)
    lo, hi = 0.2e-9, 0.7e-9
    cards = [oracle.Measure(k, 0, oracle.meas_clause(s0, from_=lo, to=hi), oracle.meas_clause(0))
             for k in (oracle.MEAS_MIN, oracle.MEAS_MAX, oracle.MEAS_AVG, oracle.MEAS_PP)]
    got, _, _ = oracle.tran_meas(fr, slots, values, o, cards)
    for lane in range(2):
        n = int(npts[lane])
        tt, vv = t[lane, :n], v[lane, :n, 0]
        inside = (tt >= lo) & (tt <= hi)
        w, wt = vv[inside], tt[inside]
        avg = 0.0
        for k in range(1, len(w)):
            avg += 0.5 * (w[k] + w[k - 1]) * (wt[k] - wt[k - 1])
        span = 0.0
        for k in range(1, len(w)):
            span += wt[k] - wt[k - 1]
        assert got[lane, 0] == w.min()
        assert got[lane, 1] == w.max()
        assert got[lane, 2] == avg / span
        assert got[lane, 3] == w.max() - w.min()


def _rc(r=1e3):
    from espice_b200.circuit import Circuit
    c = Circuit()
    c.V("v1", "in", "0", pulse=[0.0, 1.0, 0.0, 1e-12, 1e-12, 1.0, 2.0])
    c.R("r1", "in", "out", r)
    c.C("c1", "out", "0", 1e-9)
    return c.freeze()


def test_integral_rms_and_derivative_on_the_rc_charge():
    """INTEGRAL, DERIVATIVE .. AT= and RMS on the RC charging curve of the
    reference's hspice/meas_forms fixture (1 kohm, 1 nF, a 1 V step; .tran
    10n 5u), against the fixture's analytic values at its tolerances: v(out)
    = 1 - exp(-t / 1 us), its integral over 0..5 us = 5 us - (1 - e^-5) us
    (rtol 2e-3), its slope at 1 us = e^-1 / 1 us (rtol 1e-2); and the RMS
    over 1..2 us from the same curve's closed form."""
    import math
    fr = _rc()
    out = fr.unknown("v(out)")
    o = oracle.tran_opts(5e-6, 10e-9, 0.0)
    m = oracle.Measure
    c = oracle.meas_clause
    cards = [m(oracle.MEAS_INTEG, 0, c(out, from_=0.0, to=5e-6), c(0)),
             m(oracle.MEAS_DERIV, 0, c(out, at=1e-6), c(0)),
             m(oracle.MEAS_RMS, 0, c(out, from_=1e-6, to=2e-6), c(0)),
             m(oracle.MEAS_INTEG, 0, c(out), c(0))]
    got, st, _ = oracle.tran_meas(fr, [], np.zeros((1, 1)), o, cards)
    assert st[0, 0] == 0
    tau = 1e-6
    area = 5e-6 - (1 - math.exp(-5.0)) * tau
    slope = math.exp(-1.0) / tau

    def sq(t):  # integral of (1 - exp(-t/tau))^2
        return t + 2 * tau * math.exp(-t / tau) - 0.5 * tau * math.exp(-2 * t / tau)

    rms = math.sqrt((sq(2e-6) - sq(1e-6)) / 1e-6)
    assert abs(got[0, 0] - area) <= 2e-3 * area
    assert abs(got[0, 1] - slope) <= 1e-2 * slope
    assert abs(got[0, 2] - rms) <= 2e-3 * rms
    assert abs(got[0, 3] - area) <= 2e-3 * area


def test_integral_panels_follow_the_recorded_waveform():
    """The streamed INTEGRAL over a window with interpolated ends against the
    same panel rules applied to the recorded waveform (numpy): Simpson's 3/8
    rule over four equally spaced points, else Simpson's rule over three,
    else the trapezoid."""
    fr, slots, values = decks.ring_oscillator(lanes=1)
    s0 = fr.unknown("v(s0)")
    o = oracle.tran_opts(1e-9, decks.RING_T_STEP, decks.RING_T_MAX)
    t, v, npts, st, _ = oracle.tran(fr, slots, values, o, [s0], 100_000)
    n = int(npts[0])
    tt, vv = t[0, :n], v[0, :n, 0]
    lo, hi = 0.2e-9 + 3e-13, 0.7e-9 + 3e-13
    card = oracle.Measure(oracle.MEAS_INTEG, 0, oracle.meas_clause(s0, from_=lo, to=hi), oracle.meas_clause(0))
    got, _, _ = oracle.tran_meas(fr, slots, values, o, [card])

    def line(x0, y0, x1, y1, at):
        slope = (y1 - y0) / (x1 - x0)
        return slope * at + (y0 - slope * x0)

    k0 = int(np.searchsorted(tt, lo))
    k1 = int(np.searchsorted(tt, hi, side="right"))
    # the first sample at or past FROM is read as the value at FROM, the
    # first past TO as the value at TO
    pts = [(lo, line(tt[k0 - 1], vv[k0 - 1], tt[k0], vv[k0], lo))] + [(tt[k], vv[k]) for k in range(k0 + 1, k1)]
    pts.append((hi, line(tt[k1 - 1], vv[k1 - 1], tt[k1], vv[k1], hi)))

    def close(a, b):
        return a == b or abs(a - b) <= 100 * np.spacing(max(abs(a), abs(b)))

    total, i = 0.0, 0
    while len(pts) - i > 1:
        w = [pts[i + j + 1][0] - pts[i + j][0] if i + j + 1 < len(pts) else 0.0 for j in range(3)]
        if close(w[0], w[1]) and close(w[0], w[2]):
            total += 3 * w[0] * (pts[i][1] + 3 * (pts[i + 1][1] + pts[i + 2][1]) + pts[i + 3][1]) / 8
            i += 3
        elif close(w[0], w[1]):
            total += w[0] * (pts[i][1] + 4 * pts[i + 1][1] + pts[i + 2][1]) / 3
            i += 2
        else:
            total += w[0] * (pts[i][1] + pts[i + 1][1]) / 2
            i += 1
    assert abs(got[0, 0] - total) <= 1e-12 * abs(total), (got[0, 0], total)

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

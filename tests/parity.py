"""Lane parity checks shared by the GPU tests: the plain FP64 form must take
exactly the oracle's Newton iteration count on every lane, and every lane's
solution must lie within 1e-9 relative or 1e-12 absolute of the oracle's.

A lane whose iteration count differs is a flip. Flips are never dropped from
the comparison: the check fails and its message lists each flipped lane with
the oracle's gate inputs at its last iterates (the delta score, the largest
residual over its gate, the limited flag: a flip from a rounding difference
shows a score within a few ulp of 1.0 there).
"""

from __future__ import annotations

import numpy as np

from oracle import oracle

RTOL, ATOL = 1e-9, 1e-12


def close(a, b, rtol=RTOL, atol=ATOL):
    return np.abs(a - b) <= atol + rtol * np.maximum(np.abs(a), np.abs(b))


def flip_report(fr, slots, values, warm, opts, lanes_, itg, ito, k=3):
    """The oracle's gate inputs of each flipped lane at its last k iterates."""
    values = np.asarray(values, np.float64).reshape(-1, max(1, len(slots)))
    sel = values[lanes_]
    w = None
    if warm is not None:
        w = np.asarray(warm, np.float64)
        if w.ndim == 2:
            w = w[lanes_]
            # per-lane warm starts: one trace call per lane
    lines = []
    for j, lane in enumerate(lanes_):
        wl = None if w is None else (w[j] if w.ndim == 2 else w)
        _, it, _, tr = oracle.dc_points_trace(fr, slots, sel[j:j + 1], warm=wl, opts=opts,
                                              cap=max(int(ito[lane]), int(itg[lane])) + 1)
        last = int(it[0])
        rows = []
        for i in range(max(0, last - k), min(tr.shape[1], max(last, int(itg[lane])) + 1)):
            s, r, lim = tr[0, i]
            if np.isnan(s):
                continue
            rows.append(f"it {i}: delta {s!r} resid/gate {r!r} limited {int(lim)}")
        lines.append(f"lane {lane}: gpu {int(itg[lane])} its, oracle {int(ito[lane])} its; " + "; ".join(rows))
    return "\n".join(lines)


def assert_dc_parity(fr, slots, values, warm, opts, xg, itg, stg_conv, xo, ito, cvo, what=""):
    """Exact iteration counts and convergence flags on every lane, x within
    the parity tolerance on every lane. Returns the fraction of lanes whose
    x is bitwise the oracle's."""
    assert np.array_equal(stg_conv, cvo.astype(bool)), f"{what}: convergence differs on {np.flatnonzero(stg_conv != cvo.astype(bool))}"
    flips = np.flatnonzero(itg != ito)
    if len(flips):
        raise AssertionError(f"{what}: {len(flips)} of {len(itg)} lanes flipped\n"
                             + flip_report(fr, slots, values, warm, opts, flips[:8], itg, ito))
    ok = close(xg, xo)
    assert ok.all(), f"{what}: x off on lanes {np.flatnonzero(~ok.all(axis=1))[:10]}, max |dx| {np.max(np.abs(xg - xo))}"
    return float((xg.view(np.uint64) == xo.view(np.uint64)).all(axis=1).mean())

"""Test helper: runs the library's compiled warp programs (as
esl_compile_tape returns them: rows of 32 ops of one kind over
v = [tape values | y | 0.0 | 1.0 | sink], padding ops writing the sink) on
the CPU, row by row, with numpy float64 (IEEE, no fused multiply-add).
Every op of a row reads the values as they stood before the row (the
parallel semantics), so a schedule that let two ops of one row touch the
same value in conflicting ways would show up as a mismatch. Bitwise
equality with the oracle's column replay shows the schedule keeps every
value's operation order."""

import numpy as np

FLOP, DIVG, DIVS, SUBNZ, DIVY, NOP = 0, 1, 2, 3, 4, 7


def _run(words, v):
    w = words.astype(np.int64)
    bad = False
    rows = len(w) // 64
    for r in range(rows):
        snap = v.copy()
        row = w[r * 64:(r + 1) * 64]
        for t in range(32):
            w0, w1 = row[2 * t], row[2 * t + 1]
            kind, dst, a, b = w0 >> 28, w0 & 0x0FFFFFFF, w1 & 0xFFFF, w1 >> 16
            if kind == FLOP:
                v[dst] = snap[dst] - snap[a] * snap[b]
            elif kind == DIVG:
                x, d = snap[b], snap[a]
                if not (abs(d) >= 1e-12 * abs(x)):
                    bad = True
                v[dst] = x / d
            elif kind == DIVS:
                l = snap[b] / snap[a]
                if not np.isfinite(l):
                    bad = True
                v[dst] = l
            elif kind == SUBNZ:
                if snap[b] != 0:
                    v[dst] = snap[dst] - snap[a] * snap[b]
            elif kind == DIVY:
                v[dst] = snap[b] / snap[a]
    return bad


def refactor_solve(tape, vals, rhs, n):
    """(tv, dx, bad) for one lane: program A, the peel tests, program B."""
    info = tape["info"]
    nu, nl, ntv = info["nu"], info["nl"], info["ntv"]
    v = np.zeros(ntv + n + 3)  # tape values | y | 0.0 | 1.0 | sink
    v[ntv + n + 1] = 1.0
    v[tape["amap"]] = vals
    v[ntv + tape["pinv"]] = -rhs
    bad = _run(tape["a_ops"], v)
    if not np.all(np.isfinite(v[:nu])):
        bad = True
    d = v[nu:nu + n]
    if np.any((d == 0) | ~np.isfinite(d)):
        bad = True
    L = v[nu + n:nu + n + nl]
    if np.any(~(np.abs(L[tape["l_scaled"][:nl] == 0]) <= 1e3)):
        bad = True
    _run(tape["b_ops"], v)
    dx = np.zeros(n)
    dx[tape["q"]] = v[ntv:ntv + n]
    return v[:ntv], dx, bad

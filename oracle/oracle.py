"""TEST INFRASTRUCTURE: ctypes binding of the CPU oracle (liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
this module, as the checker of the CUDA library; the library never does.
The oracle restates the reference's FP64 CPU path (see espice_oracle.h for
the file map) and is pinned against the reference's ngspice-44.2 fixtures.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
# The same restatement with the host C library's exp, log and pow in the
# model code (liboracle.so uses the kernels' shared esl_math.h functions).
LIB_LIBM = os.path.join(HERE, "liboracle_libm.so")

_lib = None
_lib_libm = None

u32p = ctypes.POINTER(ctypes.c_uint32)
f64p = ctypes.POINTER(ctypes.c_double)
u8p = ctypes.POINTER(ctypes.c_uint8)


class NewtonOpts(ctypes.Structure):
    _fields_ = [("reltol", ctypes.c_double), ("abstol", ctypes.c_double),
                ("vntol", ctypes.c_double), ("residual_tol", ctypes.c_double),
                ("gmin", ctypes.c_double), ("max_iter", ctypes.c_uint32)]


def newton_opts(reltol=1e-3, abstol=1e-12, vntol=1e-6, residual_tol=1e-9, gmin=0.0, max_iter=50):
    return NewtonOpts(reltol, abstol, vntol, residual_tol, gmin, max_iter)


def build():
    """Compiles liboracle.so from oracle/*.c (make)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(libm=False):
    """The oracle library; libm=True: the variant with the C library's
    transcendentals in the model code."""
    global _lib, _lib_libm
    if libm:
        if _lib_libm is None:
            if not os.path.exists(LIB_LIBM):
                build()
            _lib_libm = ctypes.CDLL(LIB_LIBM)
        return _lib_libm
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def pattern(frozen):
    cap = frozen.n + 64 + sum(nd.shape[0] * 80 for _, nd, _ in frozen.batches)
    cp = np.zeros(frozen.n + 1, np.uint32)
    ri = np.zeros(cap, np.uint32)
    f = lib().orc_pattern
    f.restype = ctypes.c_int64
    nnz = f(ctypes.byref(frozen.struct()), _p(cp, u32p), _p(ri, u32p), ctypes.c_size_t(cap))
    assert nnz >= 0
    return cp, ri[:nnz].copy()


def order(n, cp, ri):
    q = np.zeros(n, np.uint32)
    lib().orc_order(ctypes.c_uint32(n), _p(cp, u32p), _p(ri, u32p), _p(q, u32p))
    return q


def factor_tape(n, cp, ri, vals):
    """Fresh direct.Solver full factor: q, pinv, lp, li, lx, up, ui, ux, udiag, flags."""
    cap = 64 * (int(cp[n]) + n) + 64
    out = dict(q=np.zeros(n, np.uint32), pinv=np.zeros(n, np.uint32),
               lp=np.zeros(n + 1, np.uint32), li=np.zeros(cap, np.uint32),
               lx=np.zeros(cap), up=np.zeros(n + 1, np.uint32), ui=np.zeros(cap, np.uint32),
               ux=np.zeros(cap), udiag=np.zeros(n), flags=np.zeros(n, np.uint8))
    counts = np.zeros(3, np.uint32)
    vals = np.ascontiguousarray(vals, np.float64)
    rc = lib().orc_factor_tape(
        ctypes.c_uint32(n), _p(cp, u32p), _p(ri, u32p), _p(vals, f64p),
        _p(out["q"], u32p), _p(out["pinv"], u32p), _p(out["lp"], u32p), _p(out["li"], u32p),
        _p(out["lx"], f64p), _p(out["up"], u32p), _p(out["ui"], u32p), _p(out["ux"], f64p),
        _p(out["udiag"], f64p), _p(out["flags"], u8p), _p(counts, u32p), ctypes.c_size_t(cap))
    nl, nu = int(counts[0]), int(counts[1])
    for k in ("li", "lx"):
        out[k] = out[k][:nl].copy()
    for k in ("ui", "ux"):
        out[k] = out[k][:nu].copy()
    out["n_void_slots"] = int(counts[2])
    return rc, out


def lane_refactor_solve(n, cp, ri, lead, vals, rhs):
    """Bitwise host replay of the device refactor + solveNeg on lead's tape."""
    rc, tape = factor_tape(n, cp, ri, lead)
    assert rc == 0
    lanes = vals.shape[0]
    nl, nu = len(tape["li"]), len(tape["ui"])
    dx = np.zeros((lanes, n))
    lx = np.zeros((lanes, nl))
    ux = np.zeros((lanes, nu))
    ud = np.zeros((lanes, n))
    bad = np.zeros(lanes, np.uint8)
    vals = np.ascontiguousarray(vals, np.float64)
    rhs = np.ascontiguousarray(rhs, np.float64)
    lead = np.ascontiguousarray(lead, np.float64)
    lib().orc_lane_refactor_solve(
        ctypes.c_uint32(n), _p(cp, u32p), _p(ri, u32p), _p(lead, f64p), ctypes.c_uint32(lanes),
        _p(vals, f64p), _p(rhs, f64p), _p(dx, f64p), _p(lx, f64p), _p(ux, f64p), _p(ud, f64p),
        _p(bad, u8p))
    return dict(dx=dx, lx=lx, ux=ux, udiag=ud, bad=bad, tape=tape)


def solver_rounds(n, cp, ri, vals, rhs):
    """vals [rounds][lanes][nnz], rhs [rounds][lanes][n]: per-lane direct.Solver."""
    rounds, lanes = vals.shape[:2]
    dx = np.zeros((rounds, lanes, n))
    st = np.zeros((rounds, lanes), np.uint8)
    vals = np.ascontiguousarray(vals, np.float64)
    rhs = np.ascontiguousarray(rhs, np.float64)
    lib().orc_solver_rounds(ctypes.c_uint32(n), _p(cp, u32p), _p(ri, u32p),
                            ctypes.c_uint32(rounds), ctypes.c_uint32(lanes), _p(vals, f64p),
                            _p(rhs, f64p), _p(dx, f64p), _p(st, u8p))
    return dx, st


def dc_points(frozen, slots, values, warm=None, opts=None):
    """Independent sweep points (sweep/lanes.zig): x [lanes][n], iters, conv."""
    opts = opts or newton_opts()
    values = np.ascontiguousarray(values, np.float64).reshape(-1, max(1, len(slots)))
    lanes = values.shape[0]
    x = np.zeros((lanes, frozen.n))
    it = np.zeros(lanes, np.uint32)
    cv = np.zeros(lanes, np.uint8)
    sa = frozen.slots_array(slots)
    wp = None
    if warm is not None:
        warm = np.ascontiguousarray(warm, np.float64)
        wp = _p(warm, f64p)
    rc = lib().orc_dc_points(ctypes.byref(frozen.struct()), sa, ctypes.c_uint32(len(slots)),
                             _p(values, f64p), ctypes.c_uint32(lanes), wp, ctypes.byref(opts),
                             _p(x, f64p), _p(it, u32p), _p(cv, u8p))
    assert rc == 0
    return x, it, cv


def op_points(frozen, slots, values, opts=None, iter_cap=0):
    """Operating points of independent lanes through op.zig's ladder from the
    cold start: x [lanes][n], iters, conv, rung (0 plain, 1 gmin stepping,
    2 source stepping, 3 not converged). iter_cap > 0 caps every Newton run."""
    opts = opts or newton_opts(max_iter=100)
    values = np.ascontiguousarray(values, np.float64).reshape(-1, max(1, len(slots)))
    lanes = values.shape[0]
    x = np.zeros((lanes, frozen.n))
    it = np.zeros(lanes, np.uint32)
    cv = np.zeros(lanes, np.uint8)
    rung = np.zeros(lanes, np.uint8)
    sa = frozen.slots_array(slots)
    rc = lib().orc_op_points(ctypes.byref(frozen.struct()), sa, ctypes.c_uint32(len(slots)),
                             _p(values, f64p), ctypes.c_uint32(lanes), ctypes.byref(opts),
                             ctypes.c_uint32(iter_cap), _p(x, f64p), _p(it, u32p), _p(cv, u8p),
                             _p(rung, u8p))
    assert rc == 0
    return x, it, cv, rung


def math(which, x, y=None, libm=False):
    """The model code's exp ("exp"), log ("log") or pow ("pow") over arrays."""
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(np.zeros_like(x) if y is None else y, np.float64)
    out = np.zeros_like(x)
    lib(libm).orc_math(ctypes.c_int({"exp": 0, "log": 1, "pow": 2}[which]), ctypes.c_uint32(x.size),
                       _p(x, f64p), _p(y, f64p), _p(out, f64p))
    return out


def dc_points_trace(frozen, slots, values, warm=None, opts=None, cap=100, libm=False):
    """dc_points with every lane's gate inputs per iterate: trace
    [lanes][cap][3] = (delta score, max |rhs_i| / residual gate, limited),
    NaN past the lane's last iterate. libm=True runs the variant with the C
    library's exp, log and pow."""
    opts = opts or newton_opts()
    values = np.ascontiguousarray(values, np.float64).reshape(-1, max(1, len(slots)))
    lanes = values.shape[0]
    x = np.zeros((lanes, frozen.n))
    it = np.zeros(lanes, np.uint32)
    cv = np.zeros(lanes, np.uint8)
    tr = np.zeros((lanes, cap, 3))
    sa = frozen.slots_array(slots)
    wp = None
    if warm is not None:
        warm = np.ascontiguousarray(warm, np.float64)
        wp = _p(warm, f64p)
    rc = lib(libm).orc_dc_points_trace(ctypes.byref(frozen.struct()), sa, ctypes.c_uint32(len(slots)),
                                       _p(values, f64p), ctypes.c_uint32(lanes), wp, ctypes.byref(opts),
                                       _p(x, f64p), _p(it, u32p), _p(cv, u8p), _p(tr, f64p),
                                       ctypes.c_uint32(cap))
    assert rc == 0
    return x, it, cv, tr


def dc_sweep(frozen, slot, values, opts=None):
    """Sequential .dc sweep (dc.zig): x [points][n], iters, conv."""
    opts = opts or newton_opts()
    values = np.ascontiguousarray(values, np.float64)
    pts = len(values)
    x = np.zeros((pts, frozen.n))
    it = np.zeros(pts, np.uint32)
    cv = np.zeros(pts, np.uint8)
    rc = lib().orc_dc_sweep(ctypes.byref(frozen.struct()), slot, _p(values, f64p),
                            ctypes.c_uint32(pts), ctypes.byref(opts), _p(x, f64p),
                            _p(it, u32p), _p(cv, u8p))
    assert rc == 0
    return x, it, cv


def dc_sweep_lanes(frozen, slots, lane_values, sweep_slot, values, opts=None):
    """One sequential sweep per lane (esl_dc_sweep_device's semantics):
    x [lanes][points][n], iters [lanes][points], conv [lanes][points]."""
    opts = opts or newton_opts()
    values = np.ascontiguousarray(values, np.float64)
    lane_values = np.ascontiguousarray(lane_values, np.float64).reshape(-1, max(1, len(slots)))
    lanes, pts = lane_values.shape[0], len(values)
    sa = frozen.slots_array(slots)
    x = np.zeros((lanes, pts, frozen.n))
    it = np.zeros((lanes, pts), np.uint32)
    cv = np.zeros((lanes, pts), np.uint8)
    rc = lib().orc_dc_sweep_lanes(ctypes.byref(frozen.struct()), sa, ctypes.c_uint32(len(slots)),
                                  _p(lane_values, f64p), ctypes.c_uint32(lanes), sweep_slot,
                                  _p(values, f64p), ctypes.c_uint32(pts), ctypes.byref(opts),
                                  _p(x, f64p), _p(it, u32p), _p(cv, u8p))
    assert rc == 0
    return x, it, cv


class MeasClause(ctypes.Structure):
    _fields_ = [("unknown", ctypes.c_uint32), ("rise", ctypes.c_int32), ("fall", ctypes.c_int32),
                ("cross", ctypes.c_int32), ("val", ctypes.c_double), ("td", ctypes.c_double),
                ("from_", ctypes.c_double), ("to", ctypes.c_double), ("at", ctypes.c_double)]


class Measure(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("pad", ctypes.c_uint32), ("a", MeasClause), ("b", MeasClause)]


MEAS_WHEN, MEAS_TRIG_TARG, MEAS_FIND_AT, MEAS_MIN, MEAS_MAX, MEAS_AVG, MEAS_PP = 0, 1, 2, 3, 4, 5, 6
MEAS_INTEG, MEAS_RMS, MEAS_DERIV = 7, 8, 9
MEAS_UNSET, MEAS_LAST = -1, -2
TRAN_RESOLVED = 5


def meas_clause(unknown, val=1e99, rise=MEAS_UNSET, fall=MEAS_UNSET, cross=MEAS_UNSET, td=0.0, from_=0.0,
                to=0.0, at=1e99):
    return MeasClause(unknown, rise, fall, cross, val, td, from_, to, at)


def tran_meas(frozen, slots, values, opts, measures, early_stop=False):
    """The transient with streamed measures: (values [lanes][n_meas] (NaN:
    unresolved), stats [lanes][8], x_final [lanes][n])."""
    values = np.ascontiguousarray(values, np.float64).reshape(-1, max(1, len(slots)))
    lanes = values.shape[0]
    ms = (Measure * max(1, len(measures)))(*measures)
    out = np.zeros((lanes, max(1, len(measures))))
    stats = np.zeros((lanes, len(TS_FIELDS)), np.uint32)
    x = np.zeros((lanes, frozen.n))
    sa = frozen.slots_array(slots)
    rc = lib().orc_tran_meas(ctypes.byref(frozen.struct()), sa, ctypes.c_uint32(len(slots)),
                             _p(values, f64p), ctypes.c_uint32(lanes), ctypes.byref(opts), ms,
                             ctypes.c_uint32(len(measures)), ctypes.c_int(1 if early_stop else 0),
                             _p(out, f64p), _p(stats, u32p), _p(x, f64p))
    assert rc == 0
    return out[:, :len(measures)], stats, x


def op(frozen, opts=None):
    opts = opts or newton_opts(max_iter=100)
    x = np.zeros(frozen.n)
    it = ctypes.c_uint32(0)
    rc = lib().orc_op(ctypes.byref(frozen.struct()), ctypes.byref(opts), _p(x, f64p),
                      ctypes.byref(it))
    return x, int(it.value), rc


class TranOpts(ctypes.Structure):
    _fields_ = [("tstop", ctypes.c_double), ("tstep", ctypes.c_double), ("tmax", ctypes.c_double),
                ("reltol", ctypes.c_double), ("abstol", ctypes.c_double), ("vntol", ctypes.c_double),
                ("chgtol", ctypes.c_double), ("trtol", ctypes.c_double), ("dt_min", ctypes.c_double),
                ("max_steps", ctypes.c_uint32)]


def tran_opts(tstop, tstep, tmax=0.0, reltol=1e-3, abstol=1e-12, vntol=1e-6, chgtol=1e-14,
              trtol=7.0, dt_min=1e-18, max_steps=1_000_000_000):
    return TranOpts(tstop, tstep, tmax, reltol, abstol, vntol, chgtol, trtol, dt_min, max_steps)


TS_FIELDS = ["status", "accepted", "attempts", "nr_iters", "rej_newton", "rej_lte", "bp_landings",
             "op_iters"]


def tran(frozen, slots, values, opts, probes=(), max_pts=0):
    """Independent transient lanes (tran.zig Sim): returns (t [lanes][max_pts],
    v [lanes][max_pts][n_probes], n_pts [lanes], stats [lanes][8] in
    TS_FIELDS order, x_final [lanes][n])."""
    values = np.ascontiguousarray(values, np.float64).reshape(-1, max(1, len(slots)))
    lanes = values.shape[0]
    probes = np.ascontiguousarray(probes, np.uint32)
    npr = len(probes)
    t = np.zeros((lanes, max(max_pts, 1)))
    v = np.zeros((lanes, max(max_pts, 1), max(npr, 1)))
    npts = np.zeros(lanes, np.uint32)
    stats = np.zeros((lanes, len(TS_FIELDS)), np.uint32)
    xf = np.zeros((lanes, frozen.n))
    sa = frozen.slots_array(slots)
    rec = max_pts > 0
    rc = lib().orc_tran(ctypes.byref(frozen.struct()), sa, ctypes.c_uint32(len(slots)),
                        _p(values, f64p), ctypes.c_uint32(lanes), ctypes.byref(opts),
                        _p(probes, u32p) if npr else None, ctypes.c_uint32(npr),
                        ctypes.c_uint32(max_pts), _p(t, f64p) if rec else None,
                        _p(v, f64p) if rec else None, _p(npts, u32p), _p(stats, u32p), _p(xf, f64p))
    if rc == -2:
        raise ValueError("MOS1 with TOX: the Meyer gate capacitance is not restated (DC only)")
    assert rc == 0
    return t, v, npts, stats, xf

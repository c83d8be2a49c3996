"""Python binding of libespice_lanes.so (include/espice_lanes.h).

The host-side mirror of the reference's lane entry points: ``DcLanes`` plays
the role of ``sweep/lanes.solveBatch`` (src/analysis/sweep/lanes.zig:186-233)
on the B200: every lane is one independent DC sweep point, solved by the
fused CUDA Newton kernel, each lane bitwise its own scalar ``converger.run``.
The library must be built (``espice_b200.build``); nothing here falls back to
a CPU solve: a missing library or device raises.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from .circuit import Frozen, Slot

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libespice_lanes.so")

ESL_OK, ESL_INVALID_ARGUMENT, ESL_OUT_OF_MEMORY = 0, 1, 3
ESL_NOT_ELIGIBLE, ESL_NO_DEVICE, ESL_DEVICE_FAULT, ESL_TIMEOUT = 4, 5, 6, 7
LANE_CONVERGED, LANE_MAX_ITER, LANE_SINGULAR, LANE_NEED_SOLVE = 1, 2, 3, 4
# the rung an operating-point lane converged on (esl_op_solve)
RUNG_PLAIN, RUNG_GMIN, RUNG_SOURCE, RUNG_NONE = 0, 1, 2, 3

# Every entry point include/espice_lanes.h declares.
EXPORTS = ["esl_create", "esl_destroy", "esl_last_error", "esl_dims", "esl_set_lanes",
           "esl_dc_solve", "esl_dc_solve_device", "esl_dc_solve_device_static", "esl_tape", "esl_lu_replay_device",
           "esl_tape_size", "esl_pattern", "esl_compile_tape", "esl_tran", "esl_tran_device", "esl_lu_lanes_device",
           "esl_lu_lanes_mixed_device", "esl_group_dc_solve_device", "esl_autotune", "esl_dc_sweep_device",
           "esl_tran_meas_device", "esl_lu_lanes_compiled_device", "esl_lu_compiled_log",
           "esl_lu_compiled_source", "esl_lu_lanes_mixed_compiled_device", "esl_lu_compiled_mixed_source",
           "esl_set_mode", "esl_block_info", "esl_block_profile", "esl_peel_counts", "esl_op_solve",
           "esl_op_solve_device", "esl_tran_refinements", "esl_set_lanes_cols"]

u32p = ctypes.POINTER(ctypes.c_uint32)
f64p = ctypes.POINTER(ctypes.c_double)
u8p = ctypes.POINTER(ctypes.c_uint8)


class LaneError(RuntimeError):
    def __init__(self, code, what, paused=0):
        super().__init__(f"espice_lanes error {code}: {what}")
        self.code = code
        self.paused = paused  # esl_dc_solve_device_static: lanes left paused


class NewtonOpts(ctypes.Structure):
    _fields_ = [("reltol", ctypes.c_double), ("abstol", ctypes.c_double),
                ("vntol", ctypes.c_double), ("residual_tol", ctypes.c_double),
                ("gmin", ctypes.c_double), ("max_iter", ctypes.c_uint32),
                ("init_fix", ctypes.c_uint32), ("iter_cap", ctypes.c_uint32)]


class Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("lanes_per_block", ctypes.c_uint32)]


class Stats(ctypes.Structure):
    _fields_ = [("lanes", ctypes.c_uint32), ("converged", ctypes.c_uint32),
                ("peeled", ctypes.c_uint32), ("host_solves", ctypes.c_uint32),
                ("launches", ctypes.c_uint32), ("kernel_ms", ctypes.c_double),
                ("path", ctypes.c_uint32), ("refinements", ctypes.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


PREC_FP64, PREC_MIXED = 0, 1
PATH_AUTO, PATH_WARP, PATH_BLOCK = 0, 1, 2


class SolveMode(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_uint32), ("path", ctypes.c_uint32), ("block_threads", ctypes.c_uint32),
                ("refine_max", ctypes.c_uint32), ("refine_tol", ctypes.c_double), ("profile", ctypes.c_uint32),
                ("pad", ctypes.c_uint32), ("refine_skip", ctypes.c_double)]


BLOCK_PHASES = ["eval", "assemble", "refactor", "solve", "refine", "gates", "iterations"]


class BlockInfo(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint32) for k in ("width", "a_rows", "b_rows", "f_rows", "a_levels", "a_nops",
                                                 "b_nops", "ntv", "warp_ok")] + \
               [("lane_bytes", ctypes.c_uint32 * 2), ("in_smem", ctypes.c_uint32 * 2),
                ("ctas_per_sm", ctypes.c_uint32 * 2), ("split", ctypes.c_uint32 * 2),
                ("cold_bytes", ctypes.c_uint32 * 2), ("gather_terms", ctypes.c_uint32),
                ("gather_cells", ctypes.c_uint32)]


class TranOpts(ctypes.Structure):
    _fields_ = [("t_stop", ctypes.c_double), ("t_step", ctypes.c_double), ("t_max", ctypes.c_double),
                ("reltol", ctypes.c_double), ("abstol", ctypes.c_double), ("vntol", ctypes.c_double),
                ("chgtol", ctypes.c_double), ("trtol", ctypes.c_double), ("dt_min", ctypes.c_double),
                ("max_steps", ctypes.c_uint32)]


def tran_opts(t_stop, t_step, t_max=0.0, reltol=1e-3, abstol=1e-12, vntol=1e-6, chgtol=1e-14, trtol=7.0,
              dt_min=1e-18, max_steps=0):
    return TranOpts(t_stop, t_step, t_max, reltol, abstol, vntol, chgtol, trtol, dt_min, max_steps)


TS_FIELDS = ["status", "accepted", "attempts", "nr_iters", "rej_newton", "rej_lte", "bp_landings", "op_iters"]
TRAN_DONE, TRAN_UNDERFLOW, TRAN_OP_FAILED, TRAN_MAX_STEPS, TRAN_LEFT_TAPE = 0, 1, 2, 3, 4
SWEEP_DONE, SWEEP_LEFT_TAPE = 0, 4
TRAN_RESOLVED = 5


class MeasClause(ctypes.Structure):
    """esl_meas_clause: the probed unknown, RISE/FALL/CROSS counts (MEAS_UNSET,
    MEAS_LAST or k >= 1), VAL, TD, FROM, TO (0: none), AT."""
    _fields_ = [("unknown", ctypes.c_uint32), ("rise", ctypes.c_int32), ("fall", ctypes.c_int32),
                ("cross", ctypes.c_int32), ("val", ctypes.c_double), ("td", ctypes.c_double),
                ("from_", ctypes.c_double), ("to", ctypes.c_double), ("at", ctypes.c_double)]


class Measure(ctypes.Structure):
    """esl_measure: MEAS_TRIG_TARG (a = TRIG, b = TARG), else clause a alone."""
    _fields_ = [("kind", ctypes.c_uint32), ("pad", ctypes.c_uint32), ("a", MeasClause), ("b", MeasClause)]


MEAS_WHEN, MEAS_TRIG_TARG, MEAS_FIND_AT, MEAS_MIN, MEAS_MAX, MEAS_AVG, MEAS_PP = 0, 1, 2, 3, 4, 5, 6
MEAS_INTEG, MEAS_RMS, MEAS_DERIV = 7, 8, 9
MEAS_UNSET, MEAS_LAST = -1, -2


def meas_clause(unknown, val=1e99, rise=MEAS_UNSET, fall=MEAS_UNSET, cross=MEAS_UNSET, td=0.0, from_=0.0,
                to=0.0, at=1e99):
    return MeasClause(unknown, rise, fall, cross, val, td, from_, to, at)


def when(unknown, val, rise=MEAS_UNSET, fall=MEAS_UNSET, cross=MEAS_UNSET, td=0.0):
    return Measure(MEAS_WHEN, 0, meas_clause(unknown, val, rise, fall, cross, td), meas_clause(0))


def trig_targ(trig, targ):
    return Measure(MEAS_TRIG_TARG, 0, trig, targ)


def find_at(unknown, at):
    return Measure(MEAS_FIND_AT, 0, meas_clause(unknown, at=at), meas_clause(0))


def deriv_at(unknown, at):
    """DERIV .. AT=: the slope of the first segment holding AT."""
    return Measure(MEAS_DERIV, 0, meas_clause(unknown, at=at), meas_clause(0))


def window(kind, unknown, from_=0.0, to=0.0):
    """MIN, MAX, AVG, PP, INTEG or RMS (MEAS_*) of `unknown` over FROM..TO (TO 0: to the end)."""
    return Measure(kind, 0, meas_clause(unknown, from_=from_, to=to), meas_clause(0))


class TapeInfo(ctypes.Structure):
    _fields_ = [("nu", ctypes.c_uint32), ("nl", ctypes.c_uint32), ("ntv", ctypes.c_uint32),
                ("n_fill", ctypes.c_uint32), ("a_rows", ctypes.c_uint32),
                ("a_levels", ctypes.c_uint32), ("a_nops", ctypes.c_uint32),
                ("b_rows", ctypes.c_uint32), ("b_levels", ctypes.c_uint32),
                ("b_nops", ctypes.c_uint32), ("flops", ctypes.c_uint64),
                ("has_void", ctypes.c_uint32)]


_lib = None


def lu_compiled_mixed_source(n, cp, ri, lead):
    """The mixed form's CUDA source for lead's tape (host only)."""
    L = lib()
    cp = np.ascontiguousarray(cp, np.uint32)
    ri = np.ascontiguousarray(ri, np.uint32)
    lead = np.ascontiguousarray(lead, np.float64)
    size = ctypes.c_size_t(0)
    rc = L.esl_lu_compiled_mixed_source(ctypes.c_uint32(n), _p(cp, u32p), _p(ri, u32p), _p(lead, f64p), None,
                                        ctypes.c_size_t(0), ctypes.byref(size))
    if rc:
        raise LaneError(rc, "esl_lu_compiled_mixed_source")
    buf = ctypes.create_string_buffer(size.value + 1)
    L.esl_lu_compiled_mixed_source(ctypes.c_uint32(n), _p(cp, u32p), _p(ri, u32p), _p(lead, f64p), buf,
                                   ctypes.c_size_t(size.value + 1), ctypes.byref(size))
    return buf.value.decode()


def lu_compiled_source(n, cp, ri, lead, resident=0):
    """The CUDA source the compiled lane LU builds for lead's tape (host only)."""
    L = lib()
    cp = np.ascontiguousarray(cp, np.uint32)
    ri = np.ascontiguousarray(ri, np.uint32)
    lead = np.ascontiguousarray(lead, np.float64)
    size = ctypes.c_size_t(0)
    rc = L.esl_lu_compiled_source(ctypes.c_uint32(n), _p(cp, u32p), _p(ri, u32p), _p(lead, f64p),
                                  ctypes.c_uint32(resident), None, ctypes.c_size_t(0), ctypes.byref(size))
    if rc:
        raise LaneError(rc, "esl_lu_compiled_source")
    buf = ctypes.create_string_buffer(size.value + 1)
    L.esl_lu_compiled_source(ctypes.c_uint32(n), _p(cp, u32p), _p(ri, u32p), _p(lead, f64p),
                             ctypes.c_uint32(resident), buf, ctypes.c_size_t(size.value + 1), ctypes.byref(size))
    return buf.value.decode()


def lib():
    """Loads the in-tree library (building it first if the sources are newer)."""
    global _lib
    if _lib is None:
        from . import build
        if build.stale():
            build.build()
        if not os.path.exists(LIB_PATH):
            raise LaneError(ESL_NO_DEVICE, "libespice_lanes.so is not built")
        L = ctypes.CDLL(LIB_PATH)
        L.esl_last_error.restype = ctypes.c_char_p
        L.esl_lu_compiled_log.restype = ctypes.c_char_p
        for name in EXPORTS:
            if name not in ("esl_last_error", "esl_lu_compiled_log"):
                getattr(L, name).restype = ctypes.c_int32
        _lib = L
    return _lib


RECORD_FIELDS = {0: 1, 1: 1, 2: 138, 3: 138, 4: 15, 5: 33, 6: 88}


def record_size(frozen: Frozen) -> int:
    """Doubles of one lane's device records (csrc/host/records.cpp layout)."""
    return sum(RECORD_FIELDS[t] * nd.shape[0] for t, nd, _ in frozen.batches)


def newton_opts(reltol=1e-3, abstol=1e-12, vntol=1e-6, residual_tol=1e-9, gmin=0.0,
                max_iter=50, init_fix=False, iter_cap=0):
    return NewtonOpts(reltol, abstol, vntol, residual_tol, gmin, max_iter, int(init_fix), int(iter_cap))


def _p(a, t):
    return a.ctypes.data_as(t)


def pattern(frozen: Frozen):
    """The library's frozen CSC pattern of a circuit (host only)."""
    L = lib()
    cp = np.zeros(frozen.n + 1, np.uint32)
    nnz = ctypes.c_uint32(0)
    L.esl_pattern(ctypes.byref(frozen.struct()), _p(cp, u32p), None, ctypes.c_size_t(0),
                  ctypes.byref(nnz))
    ri = np.zeros(nnz.value, np.uint32)
    rc = L.esl_pattern(ctypes.byref(frozen.struct()), _p(cp, u32p), _p(ri, u32p),
                       ctypes.c_size_t(nnz.value), ctypes.byref(nnz))
    if rc:
        raise LaneError(rc, "esl_pattern")
    return cp, ri


def compile_tape(n, col_ptr, row_idx, lead):
    """Lead factor + compiled warp programs (host only): a dict of arrays."""
    L = lib()
    cp = np.ascontiguousarray(col_ptr, np.uint32)
    ri = np.ascontiguousarray(row_idx, np.uint32)
    lead = np.ascontiguousarray(lead, np.float64)
    info = TapeInfo()
    rc = L.esl_compile_tape(ctypes.c_uint32(n), _p(cp, u32p), _p(ri, u32p), _p(lead, f64p),
                            ctypes.byref(info), *([None] * 7))
    if rc:
        raise LaneError(rc, "esl_compile_tape")
    out = dict(q=np.zeros(n, np.uint32), pinv=np.zeros(n, np.uint32),
               amap=np.zeros(int(cp[n]), np.uint32), fill=np.zeros(info.n_fill, np.uint32),
               a_ops=np.zeros(2 * 32 * info.a_rows, np.uint32),
               b_ops=np.zeros(2 * 32 * info.b_rows, np.uint32),
               l_scaled=np.zeros(max(1, info.nl), np.uint8))
    rc = L.esl_compile_tape(ctypes.c_uint32(n), _p(cp, u32p), _p(ri, u32p), _p(lead, f64p),
                            ctypes.byref(info), _p(out["q"], u32p), _p(out["pinv"], u32p),
                            _p(out["amap"], u32p), _p(out["fill"], u32p), _p(out["a_ops"], u32p),
                            _p(out["b_ops"], u32p), _p(out["l_scaled"], u8p))
    if rc:
        raise LaneError(rc, "esl_compile_tape")
    out["info"] = {k: getattr(info, k) for k, _ in info._fields_}
    return out


class DcLanes:
    """DC sweep lanes on one B200: a frozen circuit, then lanes of swept
    parameter values, each solved from its own start point."""

    def __init__(self, frozen: Frozen, device: int = 0, lanes_per_block: int = 0):
        self.frozen = frozen
        self._L = lib()
        self._ctx = ctypes.c_void_p()
        opts = Options(device, lanes_per_block)
        rc = self._L.esl_create(ctypes.byref(frozen.struct()), ctypes.byref(opts),
                                ctypes.byref(self._ctx))
        if rc:
            self._ctx = None
            raise LaneError(rc, "esl_create")
        n = ctypes.c_uint32()
        nnz = ctypes.c_uint32()
        self._L.esl_dims(self._ctx, ctypes.byref(n), ctypes.byref(nnz))
        self.n, self.nnz = n.value, nnz.value
        self.n_lanes = 0

    def _check(self, rc, what):
        if rc:
            msg = self._L.esl_last_error(self._ctx)
            raise LaneError(rc, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if self._ctx:
            self._L.esl_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_lanes(self, slots, values, cols=None):
        """values [lanes][len(slots)]: each lane's swept parameter values; or,
        with cols (one column per slot), values [lanes][n_cols]: each lane's
        live parameter values, slot s taking column cols[s]
        (esl_set_lanes_cols). A C-contiguous float64 array (pinned memory
        included) is passed without a copy."""
        arr = (Slot * max(1, len(slots)))(*slots)
        if cols is None:
            values = np.ascontiguousarray(values, np.float64).reshape(-1, max(1, len(slots)))
            self._check(self._L.esl_set_lanes(self._ctx, arr, ctypes.c_uint32(len(slots)),
                                              _p(values, f64p), ctypes.c_uint32(values.shape[0])),
                        "esl_set_lanes")
        else:
            values = np.ascontiguousarray(values, np.float64)
            values = values.reshape(values.shape[0], -1)
            c = np.ascontiguousarray(cols, np.uint32)
            self._check(self._L.esl_set_lanes_cols(self._ctx, arr, ctypes.c_uint32(len(slots)), _p(c, u32p),
                                                   _p(values, f64p), ctypes.c_uint32(values.shape[1]),
                                                   ctypes.c_uint32(values.shape[0])),
                        "esl_set_lanes_cols")
        self.n_lanes = values.shape[0]

    def solve(self, x0=None, opts=None):
        """Host-buffer solve (copies in and out): x [lanes][n], iters, status, stats."""
        opts = opts or newton_opts()
        x = np.zeros((self.n_lanes, self.n))
        it = np.zeros(self.n_lanes, np.uint32)
        st = np.zeros(self.n_lanes, np.uint32)
        stats = Stats()
        xp = None
        if x0 is not None:
            x0 = np.ascontiguousarray(np.broadcast_to(x0, (self.n_lanes, self.n)), np.float64)
            xp = _p(x0, f64p)
        self._check(self._L.esl_dc_solve(self._ctx, ctypes.byref(opts), xp, _p(x, f64p),
                                         _p(it, u32p), _p(st, u32p), ctypes.byref(stats)),
                    "esl_dc_solve")
        return x, it, st, stats.as_dict()

    def op(self, opts=None):
        """Operating-point lanes (esl_op_solve): every lane's operating point
        from the cold start through op.zig's ladder. Returns x [lanes][n],
        iters, status, rung (RUNG_*) and stats."""
        opts = opts or newton_opts()
        x = np.zeros((self.n_lanes, self.n))
        it = np.zeros(self.n_lanes, np.uint32)
        st = np.zeros(self.n_lanes, np.uint32)
        rung = np.zeros(self.n_lanes, np.uint32)
        stats = Stats()
        self._check(self._L.esl_op_solve(self._ctx, ctypes.byref(opts), _p(x, f64p), _p(it, u32p),
                                         _p(st, u32p), _p(rung, u32p), ctypes.byref(stats)),
                    "esl_op_solve")
        return x, it, st, rung, stats.as_dict()

    def solve_device(self, d_x, d_iters, d_status, cold=False, opts=None):
        """Device-buffer solve: pointers (ints) to [lanes][n] f64 and [lanes] u32."""
        opts = opts or newton_opts()
        stats = Stats()
        self._check(self._L.esl_dc_solve_device(self._ctx, ctypes.byref(opts),
                                                ctypes.c_void_p(d_x), ctypes.c_int(int(cold)),
                                                ctypes.c_void_p(d_iters), ctypes.c_void_p(d_status),
                                                ctypes.byref(stats)),
                    "esl_dc_solve_device")
        return stats.as_dict()

    def set_mode(self, precision=PREC_FP64, path=PATH_AUTO, block_threads=0, refine_tol=0.0, refine_max=0,
                 profile=False, refine_skip=0.0):
        """esl_set_mode: FP64 or mixed precision; the warp lanes, the block
        lanes, or either (PATH_AUTO); profile: count the block lanes' phase
        cycles (block_profile); refine_skip: take mixed steps above that many
        tolerances unrefined (0: refine every step)."""
        m = SolveMode(precision, path, block_threads, refine_max, refine_tol, int(profile), 0, refine_skip)
        self._check(self._L.esl_set_mode(self._ctx, ctypes.byref(m)), "esl_set_mode")

    def block_profile(self):
        """The last profiled block-lane solve's cycles by phase (BLOCK_PHASES)."""
        c = (ctypes.c_uint64 * len(BLOCK_PHASES))()
        self._check(self._L.esl_block_profile(self._ctx, c), "esl_block_profile")
        return dict(zip(BLOCK_PHASES, [int(v) for v in c]))

    def peel_counts(self):
        """esl_peel_counts: (lanes peeled, host solves, launches) of the last
        transient or sequential sweep call."""
        a, b, c = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self._L.esl_peel_counts(self._ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
                    "esl_peel_counts")
        return a.value, b.value, c.value

    def tran_refinements(self):
        """esl_tran_refinements: the FP64 corrections of the last mixed
        block-lane transient, summed over its lanes."""
        c = ctypes.c_uint64(0)
        self._check(self._L.esl_tran_refinements(self._ctx, ctypes.byref(c)), "esl_tran_refinements")
        return c.value

    def block_info(self):
        info = BlockInfo()
        self._check(self._L.esl_block_info(self._ctx, ctypes.byref(info)), "esl_block_info")
        out = {k: getattr(info, k) for k, _ in info._fields_[:9]}
        for k in ("lane_bytes", "in_smem", "ctas_per_sm", "split", "cold_bytes"):
            out[k] = list(getattr(info, k))
        out["gather_terms"], out["gather_cells"] = info.gather_terms, info.gather_cells
        return out

    def solve_device_static(self, d_x, d_iters, d_status, cold=False, opts=None):
        """solve_device through the allocation-free entry point (fixed lane
        scratch in the library; the context's first solve must be
        solve_device). Returns the number of lanes left paused (0 on success;
        a nonzero count raises with ESL_NOT_ELIGIBLE)."""
        opts = opts or newton_opts()
        paused = ctypes.c_uint32(0)
        rc = self._L.esl_dc_solve_device_static(self._ctx, ctypes.byref(opts), ctypes.c_void_p(d_x),
                                                ctypes.c_int(int(cold)), ctypes.c_void_p(d_iters),
                                                ctypes.c_void_p(d_status), ctypes.byref(paused))
        if rc:
            raise LaneError(rc, "esl_dc_solve_device_static: " + self._L.esl_last_error(self._ctx).decode(),
                            paused=paused.value)
        return paused.value

    def tran(self, opts, probes=(), max_pts=0):
        """Transient lanes through esl_tran (host buffers): (t [lanes][max_pts],
        v [lanes][max_pts][n_probes], n_pts [lanes], stats [lanes][8] in
        TS_FIELDS order, x [lanes][n], kernel ms)."""
        N = self.n_lanes
        probes = np.ascontiguousarray(probes, np.uint32)
        npr = len(probes)
        t = np.zeros((N, max(max_pts, 1)))
        v = np.zeros((N, max(max_pts, 1), max(npr, 1)))
        npts = np.zeros(N, np.uint32)
        stats = np.zeros((N, len(TS_FIELDS)), np.uint32)
        x = np.zeros((N, self.n))
        ms = ctypes.c_float(0)
        rec = max_pts > 0
        self._check(self._L.esl_tran(self._ctx, ctypes.byref(opts), _p(probes, u32p) if npr else None,
                                     ctypes.c_uint32(npr), ctypes.c_uint32(max_pts),
                                     _p(t, f64p) if rec else None, _p(v, f64p) if rec else None,
                                     _p(npts, u32p) if rec else None, _p(stats, u32p), _p(x, f64p),
                                     ctypes.byref(ms)), "esl_tran")
        return t, v, npts, stats, x, ms.value

    def tran_device(self, opts, d_x, d_stats):
        """esl_tran_device without a trace: device pointers [lanes][n] f64 and
        [lanes][8] u32; returns the kernel's ms."""
        ms = ctypes.c_float(0)
        self._check(self._L.esl_tran_device(self._ctx, ctypes.byref(opts), ctypes.c_void_p(d_x),
                                            ctypes.c_void_p(d_stats), None, ctypes.c_uint32(0),
                                            ctypes.c_uint32(0), None, None, None, ctypes.byref(ms)),
                    "esl_tran_device")
        return ms.value

    def sweep(self, slot, values, opts=None):
        """Sequential .dc sweeps, one per lane (esl_dc_sweep_device): every
        lane sweeps the DC value of the V or I source at `slot` through
        `values`. Returns (x [lanes][points][n], iters [lanes][points],
        converged [lanes][points] bool, status [lanes], kernel ms)."""
        import torch
        opts = opts or newton_opts()
        values = np.ascontiguousarray(values, np.float64).reshape(-1)
        N, P = self.n_lanes, len(values)
        d_x = torch.empty((N, P, self.n), dtype=torch.float64, device="cuda")
        d_it = torch.empty((N, P), dtype=torch.int32, device="cuda")
        d_cv = torch.empty((N, P), dtype=torch.uint8, device="cuda")
        d_st = torch.empty(N, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        ms = ctypes.c_float(0)
        self._check(self._L.esl_dc_sweep_device(self._ctx, ctypes.byref(slot), _p(values, f64p), ctypes.c_uint32(P),
                                                ctypes.byref(opts), ctypes.c_void_p(d_x.data_ptr()),
                                                ctypes.c_void_p(d_it.data_ptr()), ctypes.c_void_p(d_cv.data_ptr()),
                                                ctypes.c_void_p(d_st.data_ptr()), ctypes.byref(ms)),
                    "esl_dc_sweep_device")
        return (d_x.cpu().numpy(), d_it.cpu().numpy().astype(np.uint32), d_cv.cpu().numpy().astype(bool),
                d_st.cpu().numpy().astype(np.uint32), ms.value)

    def tran_meas(self, opts, measures, early_stop=False):
        """esl_tran_meas_device: the transient with streamed measure cards.
        Returns (values [lanes][n_meas] (NaN: unresolved), stats [lanes][8],
        x [lanes][n], kernel ms)."""
        import torch
        N, M = self.n_lanes, len(measures)
        cards = (Measure * M)(*measures)
        d_x = torch.empty((N, self.n), dtype=torch.float64, device="cuda")
        d_st = torch.empty((N, len(TS_FIELDS)), dtype=torch.int32, device="cuda")
        d_v = torch.empty((N, M), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ms = ctypes.c_float(0)
        self._check(self._L.esl_tran_meas_device(self._ctx, ctypes.byref(opts), cards, ctypes.c_uint32(M),
                                                 ctypes.c_int(1 if early_stop else 0),
                                                 ctypes.c_void_p(d_x.data_ptr()), ctypes.c_void_p(d_st.data_ptr()),
                                                 ctypes.c_void_p(d_v.data_ptr()), ctypes.byref(ms)),
                    "esl_tran_meas_device")
        return (d_v.cpu().numpy(), d_st.cpu().numpy().astype(np.uint32), d_x.cpu().numpy(), ms.value)

    def autotune(self, x0=None, opts=None):
        """Times lanes per CTA 1/2/4/8 on the current lanes and keeps the fastest."""
        opts = opts or newton_opts()
        best = ctypes.c_uint32(0)
        xp = None
        if x0 is not None:
            x0 = np.ascontiguousarray(np.broadcast_to(x0, (self.n_lanes, self.n)), np.float64)
            xp = _p(x0, f64p)
        self._check(self._L.esl_autotune(self._ctx, ctypes.byref(opts), xp, ctypes.byref(best)), "esl_autotune")
        return best.value

    def tape(self):
        q = np.zeros(self.n, np.uint32)
        pinv = np.zeros(self.n, np.uint32)
        counts = np.zeros(4, np.uint32)
        self._check(self._L.esl_tape(self._ctx, _p(q, u32p), _p(pinv, u32p), _p(counts, u32p)),
                    "esl_tape")
        return q, pinv, counts

    def lu_replay(self, lead, d_a, d_rhs, d_dx, d_bad, n_lanes, d_tv=0):
        """Standalone device refactor + solve; returns the kernel's ms."""
        lead = np.ascontiguousarray(lead, np.float64)
        ms = ctypes.c_float(0)
        self._check(self._L.esl_lu_replay_device(self._ctx, _p(lead, f64p), ctypes.c_uint32(n_lanes),
                                                 ctypes.c_void_p(d_a), ctypes.c_void_p(d_rhs),
                                                 ctypes.c_void_p(d_dx), ctypes.c_void_p(d_bad),
                                                 ctypes.c_void_p(d_tv) if d_tv else None,
                                                 ctypes.byref(ms)),
                    "esl_lu_replay_device")
        return ms.value

    def lu_lanes(self, lead, d_a, d_rhs, d_dx, d_bad, n_lanes, d_tv=0):
        """Lane-interleaved refactor + solve (planes [entry][lane]); the kernel's ms."""
        lead = np.ascontiguousarray(lead, np.float64)
        ms = ctypes.c_float(0)
        self._check(self._L.esl_lu_lanes_device(self._ctx, _p(lead, f64p), ctypes.c_uint32(n_lanes),
                                                ctypes.c_void_p(d_a), ctypes.c_void_p(d_rhs),
                                                ctypes.c_void_p(d_dx), ctypes.c_void_p(d_bad),
                                                ctypes.c_void_p(d_tv) if d_tv else None, ctypes.byref(ms)),
                    "esl_lu_lanes_device")
        return ms.value

    def lu_lanes_compiled(self, lead, d_a, d_rhs, d_dx, d_bad, n_lanes, d_tv=0):
        """lu_lanes through the tape compiled into code (esl_lu_lanes_compiled_device,
        built with NVRTC on the first call); the kernel's ms."""
        lead = np.ascontiguousarray(lead, np.float64)
        ms = ctypes.c_float(0)
        self._check(self._L.esl_lu_lanes_compiled_device(self._ctx, _p(lead, f64p), ctypes.c_uint32(n_lanes),
                                                         ctypes.c_void_p(d_a), ctypes.c_void_p(d_rhs),
                                                         ctypes.c_void_p(d_dx), ctypes.c_void_p(d_bad),
                                                         ctypes.c_void_p(d_tv) if d_tv else None,
                                                         ctypes.byref(ms)), "esl_lu_lanes_compiled_device")
        return ms.value

    def lu_lanes_mixed_compiled(self, lead, d_a, d_rhs, d_dx, d_bad, n_lanes, d_refine=0):
        """lu_lanes_mixed through the tape compiled into code; the kernel's ms."""
        lead = np.ascontiguousarray(lead, np.float64)
        ms = ctypes.c_float(0)
        self._check(self._L.esl_lu_lanes_mixed_compiled_device(
            self._ctx, _p(lead, f64p), ctypes.c_uint32(n_lanes), ctypes.c_void_p(d_a), ctypes.c_void_p(d_rhs),
            ctypes.c_void_p(d_dx), ctypes.c_void_p(d_bad), ctypes.c_void_p(d_refine) if d_refine else None,
            ctypes.byref(ms)), "esl_lu_lanes_mixed_compiled_device")
        return ms.value

    def lu_compiled_log(self):
        """The compiler's log of the compiled LU (ptxas registers and spills)."""
        return self._L.esl_lu_compiled_log(self._ctx).decode()

    def lu_lanes_mixed(self, lead, d_a, d_rhs, d_dx, d_bad, n_lanes, d_refine=0):
        """FP32 lane-interleaved refactor + solve with FP64 refinement; the kernel's ms."""
        lead = np.ascontiguousarray(lead, np.float64)
        ms = ctypes.c_float(0)
        self._check(self._L.esl_lu_lanes_mixed_device(self._ctx, _p(lead, f64p), ctypes.c_uint32(n_lanes),
                                                      ctypes.c_void_p(d_a), ctypes.c_void_p(d_rhs),
                                                      ctypes.c_void_p(d_dx), ctypes.c_void_p(d_bad),
                                                      ctypes.c_void_p(d_refine) if d_refine else None,
                                                      ctypes.byref(ms)), "esl_lu_lanes_mixed_device")
        return ms.value

    def tape_size(self):
        nu, nl, ntv = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self._L.esl_tape_size(self._ctx, ctypes.byref(nu), ctypes.byref(nl),
                                          ctypes.byref(ntv)), "esl_tape_size")
        return nu.value, nl.value, ntv.value


def group_solve_device(ctxs, d_xs, d_iters, d_status, cold=None, opts=None):
    """One launch over the lanes of several DcLanes contexts (uneven batching);
    device pointers per context. Returns each context's stats."""
    opts = opts or newton_opts()
    k = len(ctxs)
    arr = (ctypes.c_void_p * k)(*[c._ctx for c in ctxs])
    px = (ctypes.c_void_p * k)(*d_xs)
    pi = (ctypes.c_void_p * k)(*d_iters)
    ps = (ctypes.c_void_p * k)(*d_status)
    cl = (ctypes.c_int * k)(*[int(bool(v)) for v in (cold or [False] * k)])
    stats = (Stats * k)()
    rc = ctxs[0]._L.esl_group_dc_solve_device(arr, ctypes.c_uint32(k), ctypes.byref(opts), px, cl, pi, ps, stats)
    ctxs[0]._check(rc, "esl_group_dc_solve_device")
    return [s.as_dict() for s in stats]

"""Python binding of the points API (include/espice_points.h).

``Points`` mirrors the reference's espice_append_points /
espice_copy_point_measures / espice_release_points / espice_lane_width
(include/espice.h:286-360, src/c_api.zig:599-667): a template circuit, its
live parameters and one analysis; points appended in batches; their named
results copied with a per-point reason. The points run as lanes of the
device kernels, up to ``lane_width`` a launch, when their results are first
copied. Errors raise ``PointsError`` with the reference's espice_status code.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from . import lanes
from .circuit import Frozen, Slot

PTS_OK, PTS_INVALID_ARGUMENT, PTS_OUT_OF_MEMORY, PTS_INVALID_QUERY = 0, 1, 3, 4
PTS_RESULT_UNAVAILABLE, PTS_FAILED, PTS_ABI_MISMATCH = 5, 6, 7
REASON_OK, REASON_NO_CONVERGENCE, REASON_TIMESTEP_TOO_SMALL, REASON_SINGULAR_MATRIX = 0, 1, 2, 3
REASON_MEASURE_UNRESOLVED, REASON_OTHER = 5, 255
OP, TRAN = 0, 1
RESULT_MEASURE, RESULT_UNKNOWN = 0, 1

# Every entry point include/espice_points.h declares.
EXPORTS = ["esl_points_create", "esl_points_destroy", "esl_points_error", "esl_points_append",
           "esl_points_copy_measures", "esl_points_release", "esl_points_lane_width"]


class PointsError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"espice points error {code}: {what}")
        self.code = code


class Result(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("kind", ctypes.c_uint32), ("index", ctypes.c_uint32)]


class Bytes(ctypes.Structure):
    _fields_ = [("data", ctypes.c_char_p), ("len", ctypes.c_size_t)]


class Config(ctypes.Structure):
    _fields_ = [("circuit", ctypes.c_void_p), ("live", ctypes.POINTER(Slot)), ("n_live", ctypes.c_uint32),
                ("analysis", ctypes.c_uint32), ("newton", lanes.NewtonOpts), ("tran", lanes.TranOpts),
                ("measures", ctypes.POINTER(lanes.Measure)), ("n_measures", ctypes.c_uint32),
                ("results", ctypes.POINTER(Result)), ("n_results", ctypes.c_uint32),
                ("device", ctypes.c_int), ("lane_width", ctypes.c_uint32)]


class Options(ctypes.Structure):
    """espice_points_options: 40 bytes through warm_start, then tangent_step."""
    _fields_ = [("struct_size", ctypes.c_size_t), ("abort_measure", Bytes), ("abort_after", ctypes.c_double),
                ("measures_only", ctypes.c_uint8), ("early_stop", ctypes.c_uint8), ("warm_start", ctypes.c_uint8),
                ("tangent_step", ctypes.c_double)]


def options(early_stop=False, warm_start=False, measures_only=False, abort_after=math.nan, tangent_step=0.0,
            struct_size=None):
    return Options(ctypes.sizeof(Options) if struct_size is None else struct_size, Bytes(None, 0), abort_after,
                   int(measures_only), int(early_stop), int(warm_start), tangent_step)


def _lib():
    L = lanes.lib()
    if not getattr(L, "_points_bound", False):
        for name in EXPORTS:
            getattr(L, name).restype = ctypes.c_int32
        L.esl_points_error.restype = ctypes.c_char_p
        L._points_bound = True
    return L


class Points:
    """A points problem: ``results`` is a list of (name, kind, index) with
    kind RESULT_MEASURE (card index of ``measures``, transient) or
    RESULT_UNKNOWN (unknown index, operating point)."""

    def __init__(self, frozen: Frozen, live, analysis, results, newton=None, tran=None, measures=(), device=0,
                 lane_width=0):
        self._L = _lib()
        self.frozen = frozen
        self.n_live = len(live)
        self._keep = [frozen.struct(), (Slot * max(1, len(live)))(*live),
                      (lanes.Measure * max(1, len(measures)))(*measures),
                      (Result * max(1, len(results)))(*[Result(n.encode(), k, i) for n, k, i in results])]
        cfg = Config(ctypes.cast(ctypes.pointer(self._keep[0]), ctypes.c_void_p), self._keep[1], len(live), analysis,
                     newton or lanes.newton_opts(), tran or lanes.tran_opts(1e-9, 1e-11), self._keep[2],
                     len(measures), self._keep[3], len(results), device, lane_width)
        self._p = ctypes.c_void_p()
        rc = self._L.esl_points_create(ctypes.byref(cfg), ctypes.byref(self._p))
        if rc:
            self._p = None
            raise PointsError(rc, "esl_points_create")

    def _check(self, rc, what):
        if rc:
            msg = self._L.esl_points_error(self._p)
            raise PointsError(rc, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if self._p:
            self._L.esl_points_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def append(self, values, opts=None):
        """values [count][n_live]; returns the first point's id."""
        values = np.ascontiguousarray(values, np.float64).reshape(-1, max(1, self.n_live))
        first = ctypes.c_uint32()
        self._check(self._L.esl_points_append(self._p, values.ctypes.data_as(lanes.f64p),
                                              ctypes.c_size_t(values.shape[0]),
                                              ctypes.byref(opts) if opts is not None else None, ctypes.byref(first)),
                    "esl_points_append")
        return first.value

    def copy_measures(self, first_id, count, names):
        """(values [count][len(names)], reasons [count])."""
        enc = [n.encode() for n in names]
        arr = (Bytes * max(1, len(enc)))(*[Bytes(e, len(e)) for e in enc])
        out = np.zeros((count, len(names)))
        reasons = np.zeros(count, np.uint32)
        self._check(self._L.esl_points_copy_measures(self._p, ctypes.c_uint32(first_id), ctypes.c_size_t(count), arr,
                                                     ctypes.c_size_t(len(names)), out.ctypes.data_as(lanes.f64p),
                                                     reasons.ctypes.data_as(lanes.u32p)),
                    "esl_points_copy_measures")
        return out, reasons

    def release(self, first_id, count):
        self._check(self._L.esl_points_release(self._p, ctypes.c_uint32(first_id), ctypes.c_size_t(count)),
                    "esl_points_release")

    def lane_width(self):
        w = ctypes.c_uint32()
        self._check(self._L.esl_points_lane_width(self._p, ctypes.byref(w)), "esl_points_lane_width")
        return w.value

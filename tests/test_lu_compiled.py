"""The tape-compiled lane LU's generator, checked on the CPU.

esl_lu_compiled_source turns a lead tape into straight-line CUDA (one
statement per op of the warp programs). Here that source is compiled as
plain C++, with the CUDA rounding intrinsics defined as the IEEE operations
they are (__ddiv_rn = a / b, __dmul_rn = a * b, __dsub_rn = a - b; g++ with
-ffp-contract=off), run over lanes in [entry][lane] planes, and compared
bitwise with the oracle's replay of the reference's refactor and solve:
dx, the U and L tape values, and the peel verdicts. NVRTC then compiles the
same source for sm_100a (no GPU needed), as the library does at run time.
"""

import ctypes
import subprocess

import numpy as np
import pytest

from espice_b200 import decks, lanes
from oracle import oracle

PRELUDE = r"""
#define ESL_LU_HOST_EMULATION
static double stage_mem[2][64];
static inline void stage_copy(unsigned, unsigned b, unsigned i, const double* src) { stage_mem[b][i] = *src; }
static inline void stage_commit() {}
template <int P> static inline void stage_wait() {}
static inline double stage_read(unsigned, unsigned b, unsigned i) { return stage_mem[b][i]; }
#define __shared__ static
#define __align__(x)
static inline unsigned long __cvta_generic_to_shared(const void*) { return 0; }
#include <cmath>
#include <cstddef>
#include <cstring>
#define __device__
#define __forceinline__ inline
#define __global__
#define __launch_bounds__(...)
#define __restrict__
struct Dim { unsigned x, y, z; };
static Dim blockIdx, threadIdx;
static inline double __ddiv_rn(double a, double b) { return a / b; }
static inline double __dmul_rn(double a, double b) { return a * b; }
static inline double __dsub_rn(double a, double b) { return a - b; }
static inline double __ldg(const double* p) { return *p; }
static inline double __ldcg(const double* p) { return *p; }
static inline float __ldcg(const float* p) { return *p; }
static inline float __fdiv_rn(float a, float b) { return a / b; }
static inline float __fmul_rn(float a, float b) { return a * b; }
static inline float __fsub_rn(float a, float b) { return a - b; }
static inline float __int_as_float(int x) { float f; std::memcpy(&f, &x, 4); return f; }
using std::fmax;
static inline double __longlong_as_double(long long x) { double d; std::memcpy(&d, &x, 8); return d; }
static inline long long __double_as_longlong(double d) { long long x; std::memcpy(&x, &d, 8); return x; }
using std::fabs;
"""

DRIVER = r"""
extern "C" void run_lanes(const double* a, const double* rhs, double* tv, double* dx, unsigned char* bad,
                          unsigned n_lanes) {
  for (unsigned l = 0; l < n_lanes; ++l) {
    blockIdx.x = l / 128;
    threadIdx.x = l % 128;
    lu_tape(a, rhs, tv, dx, bad, n_lanes);
  }
}
"""


def _case(deck, seed, n_lanes=67):
    fr = decks.grid_diodes(seed=seed + 1)[0] if deck == "grid" else decks.ring_oscillator(lanes=2)[0]
    cp, ri = oracle.pattern(fr)
    n, nnz = fr.n, len(ri)
    rng = np.random.default_rng(seed)
    lead = rng.uniform(0.5, 2.0, nnz) * np.where(rng.random(nnz) < 0.5, 1, -1)
    diag = np.array([np.searchsorted(ri[cp[j]:cp[j + 1]], j) + cp[j] for j in range(n)])
    lead[diag] += 8.0
    vals = np.stack([lead * rng.uniform(0.8, 1.2, nnz) for _ in range(n_lanes)])
    vals[0] = lead
    vals[5, diag[3]] = 0.0  # a dead pivot: the lane peels
    vals[7] *= 1e-9
    rhs = rng.normal(size=(n_lanes, n))
    return fr, cp, ri, lead, vals, rhs


@pytest.mark.parametrize("deck,seed,resident", [("ring", 1, 0), ("ring", 2, 0), ("grid", 0, 0), ("ring", 1, 4),
                                                ("grid", 3, 8)])
def test_compiled_source_matches_oracle_replay(deck, seed, resident, tmp_path):
    """resident: the register budget in values (0: the library's default);
    small ones make most reads come back from the tape-value plane."""
    fr, cp, ri, lead, vals, rhs = _case(deck, seed)
    n, n_lanes = fr.n, vals.shape[0]
    src = lanes.lu_compiled_source(n, cp, ri, lead, resident=resident)
    cpp = tmp_path / "lu_tape.cpp"
    cpp.write_text(PRELUDE + src + DRIVER)
    so = tmp_path / "lu_tape.so"
    subprocess.run(["g++", "-O1", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC", "-o", str(so),
                    str(cpp)], check=True)
    lib = ctypes.CDLL(str(so))
    ref = oracle.lane_refactor_solve(n, cp, ri, lead, vals, rhs)
    tape = ref["tape"]
    nu, nl = len(tape["ui"]), len(tape["li"])
    ntv = nu + n + nl + 1
    a = np.ascontiguousarray(vals.T)
    r = np.ascontiguousarray(rhs.T)
    tv = np.zeros((ntv, n_lanes))
    dx = np.zeros((n, n_lanes))
    bad = np.zeros(n_lanes, np.uint8)
    f64p = ctypes.POINTER(ctypes.c_double)
    lib.run_lanes(a.ctypes.data_as(f64p), r.ctypes.data_as(f64p), tv.ctypes.data_as(f64p),
                  dx.ctypes.data_as(f64p), bad.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                  ctypes.c_uint32(n_lanes))
    assert np.array_equal(bad, ref["bad"])
    good = bad == 0
    assert good.sum() > n_lanes // 2
    assert np.array_equal(dx.T[good].view(np.uint64), ref["dx"][good].view(np.uint64))
    assert np.array_equal(tv.T[good, :nu].view(np.uint64), ref["ux"][good].view(np.uint64))
    assert np.array_equal(tv.T[good, nu:nu + n].view(np.uint64), ref["udiag"][good].view(np.uint64))
    assert np.array_equal(tv.T[good, nu + n:nu + n + nl].view(np.uint64), ref["lx"][good].view(np.uint64))


def _nvrtc():
    for name in ("libnvrtc.so.12", "libnvrtc.so"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            pass
    return None


def test_compiled_source_builds_for_sm100a():
    nv = _nvrtc()
    if nv is None:
        pytest.skip("NVRTC is not installed here")
    fr, cp, ri, lead, vals, rhs = _case("ring", 1)
    src = lanes.lu_compiled_source(fr.n, cp, ri, lead)
    prog = ctypes.c_void_p()
    assert nv.nvrtcCreateProgram(ctypes.byref(prog), src.encode(), b"lu_tape.cu", 0, None, None) == 0
    opts = [b"--gpu-architecture=sm_100a", b"--fmad=false", b"-std=c++17"]
    rc = nv.nvrtcCompileProgram(prog, len(opts), (ctypes.c_char_p * len(opts))(*opts))
    size = ctypes.c_size_t()
    nv.nvrtcGetProgramLogSize(prog, ctypes.byref(size))
    log = ctypes.create_string_buffer(size.value + 1)
    nv.nvrtcGetProgramLog(prog, log)
    cubin = ctypes.c_size_t()
    nv.nvrtcGetCUBINSize(prog, ctypes.byref(cubin))
    nv.nvrtcDestroyProgram(ctypes.byref(prog))
    assert rc == 0, log.value.decode()
    assert cubin.value > 0


MIXED_DRIVER = r"""
extern "C" void run_lanes(const double* a, const double* rhs, float* tf, double* dx, unsigned char* bad,
                          unsigned char* refine, unsigned n_lanes) {
  for (unsigned l = 0; l < n_lanes; ++l) {
    blockIdx.x = l / 128;
    threadIdx.x = l % 128;
    lu_tape_mixed(a, rhs, tf, dx, bad, refine, n_lanes);
  }
}
"""


@pytest.mark.parametrize("deck,seed", [("ring", 1), ("grid", 0)])
def test_compiled_mixed_source_refines_to_fp64(deck, seed, tmp_path):
    """The mixed form (FP32 factors and solves, FP64 refinement), compiled
    as C++: the same peel verdicts as the FP64 replay (these lanes sit far
    from the FP32 thresholds) and dx within 1e-9 of the oracle's FP64 dx on
    every lane that refined to the 1e-12 residual."""
    fr, cp, ri, lead, vals, rhs = _case(deck, seed)
    n, n_lanes = fr.n, vals.shape[0]
    src = lanes.lu_compiled_mixed_source(n, cp, ri, lead)
    cpp = tmp_path / "lu_mixed.cpp"
    cpp.write_text(PRELUDE + src + MIXED_DRIVER)
    so = tmp_path / "lu_mixed.so"
    subprocess.run(["g++", "-O1", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC", "-o", str(so),
                    str(cpp)], check=True)
    lib = ctypes.CDLL(str(so))
    ref = oracle.lane_refactor_solve(n, cp, ri, lead, vals, rhs)
    tape = ref["tape"]
    ntv = len(tape["ui"]) + n + len(tape["li"]) + 1
    a = np.ascontiguousarray(vals.T)
    r = np.ascontiguousarray(rhs.T)
    tf = np.zeros((ntv, n_lanes), np.float32)
    dx = np.zeros((n, n_lanes))
    bad = np.zeros(n_lanes, np.uint8)
    refine = np.zeros(n_lanes, np.uint8)
    f64p, f32p, u8p = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint8)
    lib.run_lanes(a.ctypes.data_as(f64p), r.ctypes.data_as(f64p), tf.ctypes.data_as(f32p), dx.ctypes.data_as(f64p),
                  bad.ctypes.data_as(u8p), refine.ctypes.data_as(u8p), ctypes.c_uint32(n_lanes))
    assert np.array_equal(bad, ref["bad"])
    good = (bad == 0) & (refine < 6)
    assert good.sum() > n_lanes // 2
    want = ref["dx"][good]
    got = dx.T[good]
    assert np.all(np.abs(got - want) <= 1e-9 * np.abs(want).max(axis=1, keepdims=True))

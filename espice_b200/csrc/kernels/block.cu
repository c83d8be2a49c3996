// Block lanes for sm_100a: the DC Newton solve of circuits whose lane working
// set is too large for one warp's share of shared memory (hundreds to
// thousands of unknowns). One CTA owns a lane for its whole solve, every
// phase in one persistent launch, as the warp lanes do (newton.cu); what
// changes is the width: eval strides over the CTA's threads, the tape
// programs are rows of one op per thread (a CTA barrier between rows), and
// reductions run across the CTA. Nothing per topology is staged: the
// programs (L2-resident, shared by every lane of the topology) stream in,
// each thread copying its own op words 4 rows ahead
// into a private ring in shared memory with cp.async, and the assembly is a
// per-thread stream of staging indices read eight terms ahead, so neither
// waits on an L2 round trip per row or per term.
//
// Where the working set lives: x | rhs | diag | dx | limited images |
// (mixed: the FP64 matrix) | v = [tape values | y | 0.0 | 1.0 | sink] |
// xo | staging, in the CTA's shared memory when it fits; or its hot part
// (up to v) there and xo and the staging cells (written once and read once
// an iteration, by the evaluation and the assembly) in a per-CTA slab of
// global memory, when that lets more CTAs share an SM; else all of it in
// the slab (L2-resident for the lane's solve; one CTA writes and reads it,
// ordered by its barriers).
//
// Two precisions. FP64: the refactor and solves are bitwise the CPU replay
// (sparse_lu.zig refactor + solve), as the warp programs are. Mixed: the
// tape values and y are FP32 (the refactor and both triangular solves in
// FP32), the assembled matrix is kept in FP64, and each Newton step is
// refined in FP64 on the residual -rhs - A dx (A and rhs FP64, corrections
// solved on the FP32 factors) until max |res| <= tol * max |rhs|. Device
// evaluation, assembly, the refinement residual, the update and the Newton
// gates stay FP64 in both.
//
// Reference path: src/solver/lane_kernels.zig:49-143 (refactor, solveNeg),
// sparse_lu.zig:918-1184, converger.zig newtonLanes / finalizeStep
// (:199-522); the refinement has no reference counterpart (the reference's
// lane LU is FP64 only).
#include <cuda_runtime.h>
#include <math_constants.h>

#include "block.h"
#include "lane_eval.cuh"
#include "ladder.cuh"
#include "tran_core.cuh"

namespace esl {

namespace {

__device__ __forceinline__ uint64_t warp_max_bits(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t w = __shfl_xor_sync(kFull, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// Maximum over the CTA of a non-negative double's bit pattern (the order of
// non-negative doubles); red holds one word per warp.
template <uint32_t kW>
__device__ __forceinline__ uint64_t block_max_bits(uint64_t v, uint64_t* red) {
  v = warp_max_bits(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  uint64_t r = 0;
#pragma unroll
  for (uint32_t w = 0; w < kW / 32; ++w) r = red[w] > r ? red[w] : r;
  __syncthreads();
  return r;
}

template <uint32_t kW>
__device__ __forceinline__ double block_max_abs(double v, uint64_t* red) {
  return from_bits(block_max_bits<kW>(dbits(fabs(v)), red));
}

// fmax over the CTA (NaN ignored, as fmax does).
template <uint32_t kW>
__device__ __forceinline__ double block_fmax(double v, uint64_t* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dbits(v);
  __syncthreads();
  double r = from_bits(red[0]);
#pragma unroll
  for (uint32_t w = 1; w < kW / 32; ++w) r = fmax(r, from_bits(red[w]));
  __syncthreads();
  return r;
}

// The op's arithmetic in the lane's precision, rounded as the CPU replay
// rounds (FP64: bitwise; FP32: the same order in FP32).
__device__ __forceinline__ double op_div(double b, double a) { return div_rn(b, a); }
__device__ __forceinline__ float op_div(float b, float a) { return __fdiv_rn(b, a); }
__device__ __forceinline__ double op_msub(double d, double a, double b) { return __dsub_rn(d, __dmul_rn(a, b)); }
__device__ __forceinline__ float op_msub(float d, float a, float b) { return __fsub_rn(d, __fmul_rn(a, b)); }
__device__ __forceinline__ double growth(double) { return 1e-12; }
__device__ __forceinline__ float growth(float) { return 1e-12f; }
__device__ __forceinline__ double inf_of(double) { return CUDART_INF; }
__device__ __forceinline__ float inf_of(float) { return CUDART_INF_F; }

// One op of a row (thread-local): a division with its pivot checks, or a
// multiply-subtract (the solves skip a zero multiplier, the refactor never
// does); no-ops pad the row. Returns true on a failed pivot test.
template <typename V>
__device__ __forceinline__ bool run_op(const uint4& op, V* v) {
  const uint32_t kind = op.x >> 28;
  if (kind == kOpNop) return false;
  V* pd = v + (op.x & 0x0fffffffu);
  const V a = v[op.y], b = v[op.z];
  if (kind == kOpDivGrowth || kind == kOpDivScaled || kind == kOpDivY) {
    const V q = op_div(b, a);
    *pd = q;
    if (kind == kOpDivGrowth) return !(fabs(a) >= growth(a) * fabs(b));
    if (kind == kOpDivScaled) return !(fabs(q) < inf_of(q));
    return false;
  }
  const V d = *pd;
  if (kind == kOpFlop || b != V(0)) *pd = op_msub(d, a, b);
  return false;
}

// K independent ops of one row: every operand loaded first, then the
// results computed and stored in op order (run_op's arithmetic and checks).
template <typename V, uint32_t K>
__device__ __forceinline__ bool run_ops(const uint4 (&op)[K], V* v) {
  V a[K], b[K], d[K];
#pragma unroll
  for (uint32_t j = 0; j < K; ++j) {
    const uint32_t kind = op[j].x >> 28;
    if (kind != kOpNop) {
      a[j] = v[op[j].y];
      b[j] = v[op[j].z];
      d[j] = v[op[j].x & 0x0fffffffu];
    }
  }
  bool bad = false;
#pragma unroll
  for (uint32_t j = 0; j < K; ++j) {
    const uint32_t kind = op[j].x >> 28;
    if (kind == kOpNop) continue;
    V* pd = v + (op[j].x & 0x0fffffffu);
    if (kind == kOpDivGrowth || kind == kOpDivScaled || kind == kOpDivY) {
      const V q = op_div(b[j], a[j]);
      *pd = q;
      if (kind == kOpDivGrowth) bad |= !(fabs(a[j]) >= growth(a[j]) * fabs(b[j]));
      if (kind == kOpDivScaled) bad |= !(fabs(q) < inf_of(q));
    } else if (kind == kOpFlop || b[j] != V(0)) {
      *pd = op_msub(d[j], a[j], b[j]);
    }
  }
  return bad;
}

// Op words: 8 bytes {dst | kind << 28, a | b << 16} when the value space
// has 16-bit indices, 16 bytes {dst | kind << 28, a, b, 0} otherwise. A
// thread's ring holds kDepth + 1 op words (10 or 20 KB a CTA): kDepth rows
// in flight (about 1,500 cycles ahead, past an L2 round trip), and the slot
// being refilled is
// never the one being read.
template <typename OpT>
struct OpFormat;
template <>
struct OpFormat<uint2> {
  static constexpr uint32_t kDepth = 4;
  __device__ static uint4 decode(uint2 o) { return make_uint4(o.x, o.y & 0xffffu, o.y >> 16, 0u); }
};
template <>
struct OpFormat<uint4> {
  static constexpr uint32_t kDepth = 4;
  __device__ static uint4 decode(uint4 o) { return o; }
};

__device__ __forceinline__ void ring_copy(uint32_t dst, const void* src, uint32_t bytes) {
  if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
  else asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void ring_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void ring_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ uint2 ld_ring(uint32_t a, uint2*) {
  uint2 r;
  asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(r.x), "=r"(r.y) : "r"(a));
  return r;
}
__device__ __forceinline__ uint4 ld_ring(uint32_t a, uint4*) {
  uint4 r;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w) : "r"(a));
  return r;
}

// Runs a program over v: row r holds K * kW ops, this thread's are
// ops[(r * K + j) * kW + tid] for j < K; a CTA barrier after each row. The
// ops of a row are independent (no op reads or writes a value another op of
// the row writes), so a thread loads the operands of all K before it stores
// any: K loads in flight per thread, the rows' latency paid once per K ops.
// Each thread keeps its next kDepth rows of op words in flight through its
// ring (slot s at ring + s * K * kW * sizeof(OpT), op j of the slot
// j * kW * sizeof(OpT) further, one commit group per row), so a row waits
// only for its own op words, copied kDepth rows earlier. K = 1 (rows of kW
// ops, 4 rows ahead) for working sets in shared memory; K = kSlabRowOps (2
// rows ahead) for working sets in the CTA's global slab, whose operand
// loads are L2 and HBM round trips. Returns this thread's pivot-test
// failures.
template <typename V, typename OpT, uint32_t kW, uint32_t K>
__device__ bool block_rows_k(const OpT* __restrict__ ops, uint32_t rows, V* v, uint32_t ring, int tid) {
  constexpr uint32_t D = K == 1 ? OpFormat<OpT>::kDepth : 2u, kSlot = K * kW * sizeof(OpT);
  constexpr uint32_t kStep = kW * sizeof(OpT);
  for (uint32_t d = 0; d < D; ++d) {
    if (d < rows)
#pragma unroll
      for (uint32_t j = 0; j < K; ++j)
        ring_copy(ring + d * kSlot + j * kStep, ops + (size_t(d) * K + j) * kW + tid, sizeof(OpT));
    ring_commit();
  }
  bool bad = false;
  uint32_t slot = 0, fill = D;  // the slot of row r, of row r + D
  for (uint32_t r = 0; r < rows; ++r) {
    ring_wait<D - 1>();  // row r's group has landed
    if constexpr (K == 1) {
      const uint4 op = OpFormat<OpT>::decode(ld_ring(ring + slot * kSlot, static_cast<OpT*>(nullptr)));
      if (r + D < rows) ring_copy(ring + fill * kSlot, ops + size_t(r + D) * kW + tid, sizeof(OpT));
      ring_commit();
      bad |= run_op(op, v);
    } else {
      uint4 op[K];
#pragma unroll
      for (uint32_t j = 0; j < K; ++j)
        op[j] = OpFormat<OpT>::decode(ld_ring(ring + slot * kSlot + j * kStep, static_cast<OpT*>(nullptr)));
      if (r + D < rows)
#pragma unroll
        for (uint32_t j = 0; j < K; ++j)
          ring_copy(ring + fill * kSlot + j * kStep, ops + (size_t(r + D) * K + j) * kW + tid, sizeof(OpT));
      ring_commit();
      bad |= run_ops<V, K>(op, v);
    }
    slot = slot == D ? 0 : slot + 1;
    fill = fill == D ? 0 : fill + 1;
    __syncthreads();
  }
  ring_wait<0>();
  return bad;
}

// The wide rows out of line: their K operand sets would otherwise raise the
// register pressure of every kernel that inlines the one-op rows.
template <typename V, typename OpT, uint32_t kW>
__device__ __noinline__ bool block_rows_wide(const OpT* __restrict__ ops, uint32_t rows, V* v, uint32_t ring,
                                             int tid) {
  return block_rows_k<V, OpT, kW, kSlabRowOps>(ops, rows, v, ring, tid);
}

template <typename V, typename OpT, uint32_t kW>
__device__ bool block_rows(const OpT* __restrict__ ops, uint32_t rows, V* v, uint32_t ring, int tid, uint32_t k) {
  if (k == kSlabRowOps) return block_rows_wide<V, OpT, kW>(ops, rows, v, ring, tid);
  return block_rows_k<V, OpT, kW, 1>(ops, rows, v, ring, tid);
}

// The lane's views into its working set.
template <typename V>
struct BlockMem {
  LaneMem m;    // x, xo, rhs, diag, staging, limited images (the shared evaluation's view)
  double* dx;   // n: the FP64 step, in unknown order
  double* a64;  // nnz: the assembled matrix in FP64 (mixed form only)
  V* v;         // tape values | y | 0.0 | 1.0 | sink
  V* y;
  uint32_t ring;  // this thread's op ring (shared address of its slot 0)
};

// base: the working set (its hot part when split); cold: the CTA's slab
// for a split layout's cold part.
template <typename V>
__device__ __forceinline__ BlockMem<V> block_carve(const BlockDev& D, unsigned char* base, unsigned char* cold,
                                                  unsigned char* ring = nullptr, uint32_t op_bytes = 8) {
  BlockMem<V> b;
  unsigned char* cbase = D.split ? cold : base;
  b.m.base = reinterpret_cast<double*>(base);
  b.m.x = reinterpret_cast<double*>(base + D.o_x);
  b.m.xo = reinterpret_cast<double*>(cbase + D.o_xo);
  b.m.rhs = reinterpret_cast<double*>(base + D.o_rhs);
  b.m.diag = reinterpret_cast<double*>(base + D.o_diag);
  b.m.st = reinterpret_cast<double*>(cbase + D.o_st);
  b.m.lim = reinterpret_cast<double*>(base + D.o_lim);
  b.m.v = nullptr;
  b.m.y = nullptr;
  b.dx = reinterpret_cast<double*>(base + D.o_dx);
  b.a64 = reinterpret_cast<double*>(base + D.o_a64);
  b.v = reinterpret_cast<V*>(base + D.o_v);
  b.y = b.v + D.T.ntv;
  b.ring = ring ? static_cast<uint32_t>(__cvta_generic_to_shared(ring)) + threadIdx.x * op_bytes : 0u;
  return b;
}

// Assembly as one streamed gather: thread t walks its term stream
// (D.g_terms[k * kW + t], k < D.g_len) summing staging cells (the constant
// cells for x[0], 1.0 and +0.0) from +0.0 in each cell's list order (the CSR order: the same bits as
// the warp lanes' gather and the host factor's pattern copy); a term with
// kGTermEnd closes a cell, whose destinations come from the thread's cell
// stream (D.g_cells[c * kW + t]): a pattern slot (its tape value, FP32 in the
// mixed form which also keeps the FP64 sum, and the diagonal copy for the
// gates) or a residual row (rhs and y = P(-rhs)). Term words arrive two
// batches of eight ahead, staging values one batch ahead, cells two ahead.
// gmin > 0 adds loadExtras' diagonal and residual terms; gs > 0 the
// gmin-stepping rung's at the cells that carry a stamp (c.w: 1 on a stamped
// slot, the column + 1 on a stamped row). Fill-in tape values are zeroed.
template <typename V, uint32_t kW>
__device__ __forceinline__ double gather_term(const BlockMem<V>& b, uint32_t w) {
  return b.m.st[w & ~kGTermEnd];
}

template <typename V, uint32_t kW>
__device__ __forceinline__ void gather_store(const BlockDev& D, const BlockMem<V>& b, const uint4& c, double s,
                                             double gmin, double gs) {
  constexpr bool kMixed = sizeof(V) == 4;
  if (c.x & kGCellRow) {
    const uint32_t i = c.x & ~kGCellRow;
    if (gmin > 0.0) s = __dadd_rn(s, __dmul_rn(gmin, b.m.x[i]));
    if (gs > 0.0 && c.w) s = __dadd_rn(s, __dmul_rn(gs, b.m.x[c.w - 1]));
    b.m.rhs[i] = s;
    b.y[c.y] = V(-s);
  } else {
    if (c.z != kNoDiag && gmin > 0.0) s = __dadd_rn(s, gmin);
    if (gs > 0.0 && c.w) s = __dadd_rn(s, gs);
    if (c.z != kNoDiag) b.m.diag[c.z] = s;
    b.v[c.y] = V(s);
    if constexpr (kMixed) b.a64[c.x] = s;
  }
}

template <typename V, uint32_t kW>
__device__ void block_assemble(const BlockDev& D, const BlockMem<V>& b, double gmin, double gs, int tid) {
  const TopoDev& T = D.T;
  const uint32_t* terms = D.g_terms + tid;
  const uint4* cells = D.g_cells + tid;
  const uint32_t K = D.g_len, pad = T.n_stage + kGCellZero;
  // Term words two batches ahead and staging values one batch ahead: every
  // load of a batch is issued before the stores of the batch before it, so
  // none waits behind them (the staging cells are only read here).
  uint32_t w[8], nx[8];
  double val[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    w[j] = uint32_t(j) < K ? __ldg(terms + size_t(j) * kW) : pad;
    nx[j] = uint32_t(8 + j) < K ? __ldg(terms + size_t(8 + j) * kW) : pad;
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) val[j] = gather_term<V, kW>(b, w[j]);
  const uint4 none = make_uint4(0u, 0u, 0u, 0u);
  uint4 cell = D.g_ncells > 0 ? __ldg(cells) : none;
  uint4 cell1 = D.g_ncells > 1 ? __ldg(cells + kW) : none;
  uint32_t c_next = 2;
  double s = 0.0;
  for (uint32_t k0 = 0; k0 < K; k0 += 8) {
    uint32_t nnx[8];
    double nv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) nnx[j] = k0 + 16 + j < K ? __ldg(terms + size_t(k0 + 16 + j) * kW) : pad;
#pragma unroll
    for (int j = 0; j < 8; ++j) nv[j] = gather_term<V, kW>(b, nx[j]);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      s = __dadd_rn(s, val[j]);
      if (w[j] & kGTermEnd) {
        gather_store<V, kW>(D, b, cell, s, gmin, gs);
        s = 0.0;
        cell = cell1;
        cell1 = c_next < D.g_ncells ? __ldg(cells + size_t(c_next) * kW) : none;
        ++c_next;
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      w[j] = nx[j];
      nx[j] = nnx[j];
      val[j] = nv[j];
    }
  }
  for (uint32_t j = tid; j < T.n_fill; j += kW) b.v[T.fill[j]] = V(0);
}

// Refactor + forward solve (program A), then the lane kernels' peel tests on
// the finished tape values (lane_kernels.zig Bodies.refactor and
// LaneSolver.wideMultipliers). CTA-uniform verdict.
template <typename V, typename OpT, uint32_t kW>
__device__ bool block_refactor(const BlockDev& D, V* v, uint32_t ring, int tid) {
  const TopoDev& T = D.T;
  bool bad = block_rows<V, OpT, kW>(static_cast<const OpT*>(D.a_ops), D.a_rows, v, ring, tid, D.row_k);
  const uint32_t l0 = T.nu + T.n;
  for (uint32_t s = tid; s < T.nu; s += kW)
    if (!(fabs(v[s]) < inf_of(v[s]))) bad = true;
  for (uint32_t k = tid; k < T.n; k += kW) {
    const V d = v[T.nu + k];
    if (d == V(0) || !(fabs(d) < inf_of(d))) bad = true;
  }
  for (uint32_t s = tid; s < T.nl; s += kW)
    if (!T.l_scaled[s] && !(fabs(v[l0 + s]) <= V(1e3))) bad = true;
  return __syncthreads_or(bad) != 0;
}

// The mixed form's FP64 iterative refinement of the step in dx (unknown
// order): res = -rhs - A dx with A and rhs in FP64 (the pattern by rows),
// stop when max |res| <= tol * max |rhs| or after refine_max corrections;
// each correction solved on the FP32 factors (program F then program B)
// and added to dx in FP64. Returns the corrections made.
template <typename OpT, uint32_t kW>
__device__ uint32_t block_refine(const BlockDev& D, const BlockMem<float>& b, uint64_t* red, int tid) {
  const TopoDev& T = D.T;
  uint32_t made = 0;
  for (uint32_t it = 0;; ++it) {
    double rmax = 0.0, bmax = 0.0;
    for (uint32_t i = tid; i < T.n; i += kW) {
      const double rb = b.m.rhs[i];
      double res = -rb;
      for (uint32_t e = T.row_ptr[i]; e < T.row_ptr[i + 1]; ++e)
        res = __dsub_rn(res, __dmul_rn(b.a64[T.row_slot[e]], b.dx[T.row_col[e]]));
      rmax = fmax(rmax, fabs(res));
      bmax = fmax(bmax, fabs(rb));
      b.y[T.pinv[i]] = float(res);
    }
    rmax = block_max_abs<kW>(rmax, red);
    bmax = block_max_abs<kW>(bmax, red);
    if (!(rmax > D.refine_tol * bmax) || it >= D.refine_max) break;
    block_rows<float, OpT, kW>(static_cast<const OpT*>(D.f_ops), D.f_rows, b.v, b.ring, tid, D.row_k);
    block_rows<float, OpT, kW>(static_cast<const OpT*>(D.b_ops), D.b_rows, b.v, b.ring, tid, D.row_k);
    for (uint32_t j = tid; j < T.n; j += kW) {
      const uint32_t i = T.qcol[j];
      b.dx[i] = __dadd_rn(b.dx[i], double(b.y[j]));
    }
    __syncthreads();
    ++made;
  }
  return made;
}

// The mixed form's refinement of a Newton step (dx in unknown order, x the
// iterate it moves): every step, or with refine_skip > 0 only a step whose
// FP32 solution scores within refine_skip tolerances of the Newton delta
// test (a step farther out is taken as an inexact Newton step: its FP32
// error, about 1e-7 of the step, is far below what the next iterate still
// corrects). Returns the corrections made.
template <typename OpT, uint32_t kW>
__device__ uint32_t block_refine_step(const BlockDev& D, const BlockMem<float>& b, const LaneOpts& o, uint64_t* red,
                                      int tid) {
  const TopoDev& T = D.T;
  if (D.refine_skip > 0.0) {
    uint64_t q = 0;
    for (uint32_t i = tid; i < T.n; i += kW) {
      const double d = b.dx[i], xo = b.m.x[i], xn = xo + d;
      const double tol = o.reltol * fmax(fabs(xn), fabs(xo)) + (T.cur_row[i] ? o.abstol : o.vntol);
      const double s = div_rn(fabs(d), tol);
      const uint64_t bits = dbits(s == s ? s : CUDART_INF);
      q = bits > q ? bits : q;
    }
    if (from_bits(block_max_bits<kW>(q, red)) > D.refine_skip) return 0;
  }
  return block_refine<OpT, kW>(D, b, red, tid);
}

// Phase profile: thread 0 adds the cycles since `t` to prof[phase] and
// restarts the clock (nothing when profiling is off).
__device__ __forceinline__ void phase_mark(unsigned long long* prof, uint32_t phase, long long& t) {
  if (prof && threadIdx.x == 0) {
    const long long now = clock64();
    atomicAdd(prof + phase, static_cast<unsigned long long>(now - t));
    t = now;
  }
}

// One lane's DC Newton solve (converger.zig newtonLanes at W = 1 with the
// lane's own direct solver), by the CTA that owns it: the warp lanes'
// dc_solve_lane step for step, reductions across the CTA.
template <typename V, typename OpT, bool kHasB3, uint32_t kW, bool kLadder = false>
__device__ void block_lane(const BlockDev& D, const LaneDev& L, const LaneOpts& o, unsigned char* base,
                           unsigned char* cold, unsigned char* ring, uint64_t* red, uint32_t lane,
                           const LadderDev* ld = nullptr) {
  constexpr bool kMixed = sizeof(V) == 4;
  const TopoDev& T = D.T;
  const int tid = threadIdx.x;
  const uint32_t status = L.status[lane];
  const bool resuming = L.resume && status == kNeedSolve;
  if (!(status == kRunning || resuming)) return;

  const uint32_t n = T.n;
  const BlockMem<V> b = block_carve<V>(D, base, cold, ring, sizeof(OpT));
  const LaneMem& m = b.m;
  const double* rec = L.rec + size_t(lane) * T.rec_size;
  for (uint32_t i = tid; i < n; i += kW) m.x[i] = L.x[size_t(lane) * n + i];
  for (uint32_t i = tid; i < T.nlim; i += kW) m.lim[i] = L.lim[size_t(lane) * T.nlim + i];
  if (tid == 0) {
    b.v[T.ntv + n] = V(0);
    b.v[T.ntv + n + 1] = V(1);
    b.v[T.ntv + n + 2] = V(0);
    m.st[T.n_stage + kGCellZero] = 0.0;
    m.st[T.n_stage + kGCellOne] = 1.0;
  }
  bool lim_active = L.lim_active[lane] != 0;
  uint32_t flags = L.flags[lane];
  uint32_t iter = L.iters[lane];
  double limit = L.limit[lane];
  const LadderRun run = ladder_run(o, kLadder ? ld : nullptr);
  const uint32_t max_iter = run.max_iter;
  uint32_t refinements = 0;
  SimDev sim;
  sim.t = 0.0;
  sim.src_scale = run.src;
  sim.kind = 0;
  sim.gmin = run.gmin_dev;
  bool have_step = false;
  if (resuming) {
    for (uint32_t i = tid; i < n; i += kW) {
      m.rhs[i] = L.rhs[size_t(lane) * n + i];
      m.diag[i] = L.diag[size_t(lane) * n + i];
      b.dx[i] = L.dx[size_t(lane) * n + i];
    }
    have_step = true;
  }
  __syncthreads();

  long long t0 = D.prof && tid == 0 ? clock64() : 0;
  for (; iter < max_iter; ++iter) {
    if (D.prof && tid == 0) atomicAdd(D.prof + kBlockPhaseIters, 1ull);
    if (!have_step) {
      eval_all<kHasB3, kW>(T, rec, m, lim_active, sim, tid, false, nullptr, true);
      if (tid == 0) m.st[T.n_stage + kGCellX0] = m.x[0];
      __syncthreads();
      phase_mark(D.prof, kBlockPhaseEval, t0);
      block_assemble<V, kW>(D, b, o.gmin, run.gs, tid);
      __syncthreads();
      phase_mark(D.prof, kBlockPhaseAssemble, t0);
      if (iter == 0) {
        // plausibleLimit: 1e3 x the start's scale, at least x_plausible
        double g = 1.0;
        uint64_t xm = 0, fm = 0;
        for (uint32_t i = tid; i < n; i += kW) {
          g = fmax(g, fabs(m.diag[i]));
          const uint64_t bx = dbits(fabs(m.x[i])), bf = dbits(fabs(m.rhs[i]));
          xm = bx > xm ? bx : xm;
          fm = bf > fm ? bf : fm;
        }
        const double gd = block_fmax<kW>(g, red);
        xm = block_max_bits<kW>(xm, red);
        fm = block_max_bits<kW>(fm, red);
        const double scale = fmin(fmax(from_bits(xm), from_bits(fm) * gd), 1e18);
        limit = !(1e3 * scale > kXPlausible) ? kXPlausible : 1e3 * scale;
      }
      const bool host_mode = (flags & 2u) != 0;
      bool bad = true;
      if (!host_mode) bad = block_refactor<V, OpT, kW>(D, b.v, b.ring, tid);
      phase_mark(D.prof, kBlockPhaseRefactor, t0);
      if (bad) {
        // Pause: the host factors this lane with its own FP64 direct solver.
        const size_t at = size_t(lane) * n;
        gather_pattern<kW>(T, m, L.a_vals + size_t(lane) * T.nnz, tid);
        for (uint32_t i = tid; i < n; i += kW) {
          L.x[at + i] = m.x[i];
          L.rhs[at + i] = m.rhs[i];
          L.diag[at + i] = m.diag[i];
        }
        for (uint32_t i = tid; i < T.nlim; i += kW) L.lim[size_t(lane) * T.nlim + i] = m.lim[i];
        if (tid == 0) {
          L.lim_active[lane] = lim_active;
          L.flags[lane] = flags | 2u;
          L.iters[lane] = iter;
          L.limit[lane] = limit;
          L.status[lane] = kNeedSolve;
          if (D.refine_out) D.refine_out[lane] += refinements;
          atomicAdd(L.n_paused, 1u);
        }
        return;
      }
      block_rows<V, OpT, kW>(static_cast<const OpT*>(D.b_ops), D.b_rows, b.v, b.ring, tid, D.row_k);
      for (uint32_t j = tid; j < n; j += kW) b.dx[T.qcol[j]] = double(b.y[j]);
      __syncthreads();
      phase_mark(D.prof, kBlockPhaseSolve, t0);
      if constexpr (kMixed) {
        refinements += block_refine_step<OpT, kW>(D, b, o, red, tid);
        phase_mark(D.prof, kBlockPhaseRefine, t0);
      }
    }
    have_step = false;

    // finalizeStep: x_old = x, x += dx, delta score (updateAndNorm)
    uint64_t worst = 0;
    for (uint32_t i = tid; i < n; i += kW) {
      const double d = b.dx[i];
      const double xold = m.x[i];
      const double xn = xold + d;
      m.xo[i] = xold;
      m.x[i] = xn;
      const double tol = o.reltol * fmax(fabs(xn), fabs(xold)) + (T.cur_row[i] ? o.abstol : o.vntol);
      const bool finite = fabs(xn) < CUDART_INF && fabs(d) < CUDART_INF;
      const double qv = div_rn(fabs(d), tol);
      const double score = !finite ? CUDART_INF : (qv == qv ? qv : 0.0);
      const uint64_t sb = dbits(score);
      worst = sb > worst ? sb : worst;
    }
    worst = block_max_bits<kW>(worst, red);
    const bool limited = __syncthreads_or(apply_limits<kHasB3, kW>(T, rec, m, lim_active, tid)) != 0;
    if (T.nlim) lim_active = true;

    bool ok = !limited && iter != 0 && !(from_bits(worst) >= 1.0);
    if (ok) {
      bool p = true;
      for (uint32_t i = tid; i < n; i += kW) p &= fabs(m.x[i]) <= limit;
      ok = __syncthreads_and(p) != 0;
    }
    if (ok) {
      bool p = true;
      for (uint32_t i = tid; i < n; i += kW) p &= fabs(m.rhs[i]) <= residual_gate(o, m.diag[i], m.x[i]);
      ok = __syncthreads_and(p) != 0;
    }
    phase_mark(D.prof, kBlockPhaseGates, t0);
    if (ok) {
      if (flags & 1u) {
        flags &= ~1u;  // INITFIX -> INITFLOAT: one more passing iterate
      } else {
        for (uint32_t i = tid; i < n; i += kW) L.x[size_t(lane) * n + i] = m.xo[i];
        if (tid == 0) {
          L.iters[lane] = iter + 1;
          L.status[lane] = kConverged;
          L.lim_active[lane] = 0;
          if (D.refine_out) D.refine_out[lane] += refinements;
        }
        return;
      }
    }
    __syncthreads();
  }
  for (uint32_t i = tid; i < n; i += kW) L.x[size_t(lane) * n + i] = m.x[i];
  if (tid == 0) {
    L.iters[lane] = max_iter;
    L.status[lane] = kMaxIter;
    L.lim_active[lane] = 0;
    if (D.refine_out) D.refine_out[lane] += refinements;
  }
}

// Persistent grid: each CTA takes lanes blockIdx.x, + gridDim.x, ...; its
// working set in dynamic shared memory, split between shared memory and its
// slab of D.slab, or all in its slab. Dynamic shared memory: the working set
// (its hot part when split; nothing when all in the slab), then the op ring.
// Two CTAs an SM by registers (the BSIM3 instantiation spills a few words
// of its evaluation for it), as many as shared memory then allows.
template <typename V, typename OpT, bool kHasB3, uint32_t kW, bool kLadder>
__global__ void __launch_bounds__(kW, 2) dc_block_kernel(BlockDev D, LaneDev L, LaneOpts o) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint64_t red[kW / 32];
  unsigned char* own = D.slab + size_t(blockIdx.x) * (D.split ? D.cold_bytes : D.lane_bytes);
  unsigned char* base = D.in_smem ? smem_raw : own;
  unsigned char* ring = smem_raw + (D.in_smem ? D.lane_bytes : 0u);
  for (uint32_t lane = blockIdx.x; lane < L.n_lanes; lane += gridDim.x) {
    if constexpr (!kLadder) {
      block_lane<V, OpT, kHasB3, kW>(D, L, o, base, own, ring, red, lane);
    } else {
      // an operating-point lane runs Newton until the ladder is done or the
      // lane pauses for a host factor (a singular host factor ends a run)
      for (;;) {
        const uint32_t st = *(volatile uint32_t*)(L.status + lane);
        if (st == kRunning || (L.resume && st == kNeedSolve)) {
          block_lane<V, OpT, kHasB3, kW, true>(D, L, o, base, own, ring, red, lane, L.ladder + lane);
          __syncthreads();
          if (*(volatile uint32_t*)(L.status + lane) == kNeedSolve) break;
        } else if (!(st == kSingular && L.ladder[lane].rung != kRungDone)) {
          break;
        }
        if (!ladder_step(D.T, L, lane, threadIdx.x, kW)) break;
      }
    }
    __syncthreads();
  }
}

// Uneven batching on the block lanes: the lanes of several topologies in one
// persistent launch. Work items are (topology, lane) pairs; each CTA takes
// the next item from a counter (items ordered largest topology first, so
// the long solves start early and the short ones fill in behind them),
// copies that topology's tables into shared memory and solves the lane with
// its working set in dynamic shared memory (when the topology's fits) or in
// the CTA's slab. Every topology of a group runs in one precision and width.
template <typename V, typename OpT, bool kHasB3, uint32_t kW>
__global__ void __launch_bounds__(kW, 2) dc_block_group_kernel(const BlockDev* __restrict__ Ds,
                                                            const LaneDev* __restrict__ Ls, const uint2* items,
                                                            uint32_t n_items, uint32_t* next, LaneOpts o,
                                                            unsigned char* slab, size_t slab_stride,
                                                            uint32_t ring_at) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint64_t red[kW / 32];
  __shared__ BlockDev D;
  __shared__ LaneDev L;
  __shared__ uint32_t item;
  unsigned char* own_slab = slab + size_t(blockIdx.x) * slab_stride;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(next, 1u);
    __syncthreads();
    const uint32_t it = item;
    if (it >= n_items) break;
    const uint2 w = items[it];
    if (threadIdx.x == 0) {
      D = Ds[w.x];
      L = Ls[w.x];
    }
    __syncthreads();
    block_lane<V, OpT, kHasB3, kW>(D, L, o, D.in_smem ? smem_raw : own_slab, own_slab, smem_raw + ring_at, red,
                                   w.y, nullptr);
    __syncthreads();
  }
}

template <typename V, bool kHasB3, uint32_t kW>
cudaError_t launch_group_t(const BlockDev* Ds, const LaneDev* Ls, const uint2* items, uint32_t n_items,
                           uint32_t* next, const LaneOpts& o, unsigned char* slab, size_t slab_stride, size_t smem,
                           uint32_t grid, cudaStream_t s) {
  auto* k = dc_block_group_kernel<V, kHasB3, kW>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(next, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  k<<<grid, kW, smem, s>>>(Ds, Ls, items, n_items, next, o, slab, slab_stride);
  return cudaGetLastError();
}

template <typename V, bool kHasB3, uint32_t kW>
int group_occupancy_t(size_t smem) {
  int per_sm = 0;
  auto* k = dc_block_group_kernel<V, kHasB3, kW>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, int(kW), smem);
  return per_sm;
}

// The lead lane's first Jacobian in pattern order (its device evaluation at
// the lane's start point), with the working set in global scratch: the
// block lanes' counterpart of assemble_kernel, for any circuit size.
template <bool kHasB3, uint32_t kW>
__global__ void __launch_bounds__(kW) block_lead_kernel(BlockDev D, LaneDev L, uint32_t lane, double* out) {
  const TopoDev& T = D.T;
  const int tid = threadIdx.x;
  const BlockMem<double> b = block_carve<double>(D, D.slab, D.slab);
  for (uint32_t i = tid; i < T.n; i += kW) b.m.x[i] = L.x[size_t(lane) * T.n + i];
  for (uint32_t i = tid; i < T.nlim; i += kW) b.m.lim[i] = L.lim[size_t(lane) * T.nlim + i];
  SimDev sim;
  sim.t = 0.0;
  sim.src_scale = 1.0;
  sim.kind = 0;
  __syncthreads();
  eval_all<kHasB3, kW>(T, L.rec + size_t(lane) * T.rec_size, b.m, L.lim_active[lane] != 0, sim, tid, false, nullptr,
                       true);
  __syncthreads();
  gather_pattern<kW>(T, b.m, out, tid);
}

template <typename V, typename OpT, bool kHasB3>
cudaError_t launch_t(const BlockDev& D, const LaneDev& L, const LaneOpts& o, cudaStream_t s) {
  // operating-point lanes: the FP64 form with the ladder between runs
  auto* k = dc_block_kernel<V, OpT, kHasB3, kBlockThreads, false>;
  if (o.ladder) {
    if constexpr (sizeof(V) == 8)
      k = dc_block_kernel<V, OpT, kHasB3, kBlockThreads, true>;
    else
      return cudaErrorNotSupported;
  }
  const size_t smem = (D.in_smem ? D.lane_bytes : 0) + D.ring_bytes;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  const uint32_t grid = D.grid < L.n_lanes ? D.grid : L.n_lanes;
  k<<<grid > 0 ? grid : 1, kBlockThreads, smem, s>>>(D, L, o);
  return cudaGetLastError();
}

template <typename V, typename OpT, bool kHasB3>
int occupancy_t(size_t smem) {
  int per_sm = 0;
  auto* k = dc_block_kernel<V, OpT, kHasB3, kBlockThreads, false>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, int(kBlockThreads), smem);
  return per_sm;
}

template <typename V, typename OpT, bool kHasB3>
cudaError_t launch_group_t(const BlockDev* Ds, const LaneDev* Ls, const uint2* items, uint32_t n_items,
                           uint32_t* next, const LaneOpts& o, unsigned char* slab, size_t slab_stride, size_t smem,
                           uint32_t ring_at, uint32_t grid, cudaStream_t s) {
  auto* k = dc_block_group_kernel<V, OpT, kHasB3, kBlockThreads>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(next, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  k<<<grid, kBlockThreads, smem, s>>>(Ds, Ls, items, n_items, next, o, slab, slab_stride, ring_at);
  return cudaGetLastError();
}

template <typename V, typename OpT, bool kHasB3>
int group_occupancy_t(size_t smem) {
  int per_sm = 0;
  auto* k = dc_block_group_kernel<V, OpT, kHasB3, kBlockThreads>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, int(kBlockThreads), smem);
  return per_sm;
}

// ---------------------------------------------------------------------------
// Transient block lanes (tran.zig Sim.begin / Sim.end and the integrator.zig
// kernels on a CTA per lane): the warp transient lanes' run, step for step,
// for circuits whose working set leaves a warp's share of shared memory, and
// for few lanes (a lane's rows spread over the CTA's 256 threads). FP64, or
// mixed precision: the FP32 refactor and solves with the step refined in
// FP64 on the FP64 residual (evaluation, assembly, the companion, the gates
// and the LTE control stay FP64). No streamed measures; a lane whose factor
// leaves the lead tape stops with kTranLeftTape (no host factor).
// ---------------------------------------------------------------------------

// The transient's row charges (q of every row that carries charge cells,
// summed from +0.0 in stamp order) into q.
template <uint32_t kW>
__device__ void block_row_charges(const TopoDev& T, const double* st, double* q, int tid) {
  for (uint32_t i = tid; i < T.n; i += kW) {
    const uint32_t e0 = T.q_ptr[i], e1 = T.q_ptr[i + 1];
    if (e0 == e1) continue;
    double s = 0.0;
    for (uint32_t e = e0; e < e1; ++e) s = __dadd_rn(s, st[T.q_src[e]]);
    q[i] = s;
  }
}

// integrator.companionAt (accumulate) and Circuit.combineGC on the
// assembled G: rows with charge get ag0 (q - q1) (less ag1 ip on a
// trapezoidal step), slots with capacitance ag0 C.
struct BlockCompanion {
  double ag0, ag1;
  bool trap;
  const double* q1;
  const double* ip;
};

template <typename V, uint32_t kW>
__device__ void block_companion(const TopoDev& T, const BlockMem<V>& b, const BlockCompanion& c, int tid) {
  constexpr bool kMixed = sizeof(V) == 4;
  const double* st = b.m.st;
  for (uint32_t i = tid; i < T.n; i += kW) {
    const uint32_t e0 = T.q_ptr[i], e1 = T.q_ptr[i + 1];
    if (e0 == e1) continue;
    double s = 0.0;
    for (uint32_t e = e0; e < e1; ++e) s = __dadd_rn(s, st[T.q_src[e]]);
    const double dq = c.ag0 * (s - c.q1[i]);
    const double base = b.m.rhs[i] + dq;
    const double r = c.trap ? base - c.ag1 * c.ip[i] : base;
    b.m.rhs[i] = r;
    b.y[T.pinv[i]] = V(-r);
  }
  // the mixed form adds to the FP64 matrix (the refinement's) and rounds the
  // sum into the FP32 tape value, so both hold G + ag0 C of the FP64 form
  for (uint32_t p = tid; p < T.nnz; p += kW) {
    const uint32_t e0 = T.c_ptr[p], e1 = T.c_ptr[p + 1];
    if (e0 == e1) continue;
    double s = 0.0;
    for (uint32_t e = e0; e < e1; ++e) s = __dadd_rn(s, st[T.c_src[e]]);
    const uint32_t at = T.amap[p], dr = T.slot_row[p];
    double v;
    if constexpr (kMixed) {
      v = b.a64[p] + c.ag0 * s;
      b.a64[p] = v;
    } else {
      v = b.v[at] + c.ag0 * s;
    }
    b.v[at] = V(v);
    if (dr != kNoDiag) b.m.diag[dr] = v;
  }
}

// One Newton solve of a block transient lane (converger.newton at W = 1,
// the warp lanes' lane_newton): the companion when cp is given, the
// gmin-stepping stamps at o.gstamp. Returns 0 converged (x holds the
// published iterate), 1 out of iterations, 2 a factor left the lead tape.
// The mixed form (V = float) refactors and solves in FP32 and refines the
// step in FP64 as the DC block lanes do (block_refine, refine_skip), adding
// the corrections made to `refinements`.
template <typename V, typename OpT, bool kHasB3, uint32_t kW>
__device__ int block_tran_newton(const BlockDev& D, const BlockMem<V>& b, const double* rec, const LaneOpts& o,
                                 const SimDev& sim, const BlockCompanion* cp, bool& lim_active, bool init_fix,
                                 uint32_t& iters, const double* vsrc, uint64_t* red, int tid,
                                 uint32_t& refinements) {
  constexpr bool kMixed = sizeof(V) == 4;
  const TopoDev& T = D.T;
  const LaneMem& m = b.m;
  const uint32_t n = T.n;
  uint32_t max_iter = o.max_iter < 100 ? 100 : o.max_iter;
  if (o.iter_cap && o.iter_cap < max_iter) max_iter = o.iter_cap;
  double limit = kXPlausible;
  for (uint32_t iter = 0; iter < max_iter; ++iter) {
    eval_all<kHasB3, kW>(T, rec, m, lim_active, sim, tid, false, vsrc);
    if (tid == 0) m.st[T.n_stage + kGCellX0] = m.x[0];
    __syncthreads();
    block_assemble<V, kW>(D, b, o.gmin, o.gstamp, tid);
    __syncthreads();
    if (cp) {
      block_companion<V, kW>(T, b, *cp, tid);
      __syncthreads();
    }
    if (iter == 0) {
      // plausibleLimit: 1e3 x the start's scale, at least x_plausible
      double g = 1.0;
      uint64_t xm = 0, fm = 0;
      for (uint32_t i = tid; i < n; i += kW) {
        g = fmax(g, fabs(m.diag[i]));
        const uint64_t bx = dbits(fabs(m.x[i])), bf = dbits(fabs(m.rhs[i]));
        xm = bx > xm ? bx : xm;
        fm = bf > fm ? bf : fm;
      }
      const double gd = block_fmax<kW>(g, red);
      xm = block_max_bits<kW>(xm, red);
      fm = block_max_bits<kW>(fm, red);
      const double scale = fmin(fmax(from_bits(xm), from_bits(fm) * gd), 1e18);
      limit = !(1e3 * scale > kXPlausible) ? kXPlausible : 1e3 * scale;
    }
    if (block_refactor<V, OpT, kW>(D, b.v, b.ring, tid)) {
      iters = iter + 1;
      return 2;
    }
    block_rows<V, OpT, kW>(static_cast<const OpT*>(D.b_ops), D.b_rows, b.v, b.ring, tid, D.row_k);
    for (uint32_t j = tid; j < n; j += kW) b.dx[T.qcol[j]] = double(b.y[j]);
    __syncthreads();
    if constexpr (kMixed) refinements += block_refine_step<OpT, kW>(D, b, o, red, tid);
    // finalizeStep: x_old = x, x += dx, delta score (updateAndNorm)
    uint64_t worst = 0;
    for (uint32_t i = tid; i < n; i += kW) {
      const double d = b.dx[i];
      const double xold = m.x[i];
      const double xn = xold + d;
      m.xo[i] = xold;
      m.x[i] = xn;
      const double tol = o.reltol * fmax(fabs(xn), fabs(xold)) + (T.cur_row[i] ? o.abstol : o.vntol);
      const bool finite = fabs(xn) < CUDART_INF && fabs(d) < CUDART_INF;
      const double qv = div_rn(fabs(d), tol);
      const double score = !finite ? CUDART_INF : (qv == qv ? qv : 0.0);
      const uint64_t sb = dbits(score);
      worst = sb > worst ? sb : worst;
    }
    worst = block_max_bits<kW>(worst, red);
    const bool limited = __syncthreads_or(apply_limits<kHasB3, kW>(T, rec, m, lim_active, tid)) != 0;
    if (T.nlim) lim_active = true;
    bool ok = !limited && iter != 0 && !(from_bits(worst) >= 1.0);
    if (ok) {
      bool p = true;
      for (uint32_t i = tid; i < n; i += kW) p &= fabs(m.x[i]) <= limit;
      ok = __syncthreads_and(p) != 0;
    }
    if (ok) {
      bool p = true;
      for (uint32_t i = tid; i < n; i += kW) p &= fabs(m.rhs[i]) <= residual_gate(o, m.diag[i], m.x[i]);
      ok = __syncthreads_and(p) != 0;
    }
    if (ok) {
      if (init_fix) {
        init_fix = false;  // INITFIX -> INITFLOAT: one more passing iterate
      } else {
        for (uint32_t i = tid; i < n; i += kW) m.x[i] = m.xo[i];
        __syncthreads();
        iters = iter + 1;
        return 0;
      }
    }
    __syncthreads();
  }
  iters = max_iter;
  return 1;
}

// A block transient lane's run state, in its CTA's part of the transient
// slab (global memory): the accepted point and the one before (n each),
// the row-charge ring (4 slots of n) and its currents (n), the LTE-state
// ring (4 slots of nq) and its currents (nq), the sources' values (n_src)
// and their PULSE timers (8 n_src).
__host__ __device__ inline size_t tran_block_slab_doubles(const TopoDev& T) {
  return (7 * size_t(T.n) + 5 * size_t(T.n_qt) + 9 * size_t(T.n_src) + 1) & ~size_t(1);
}

// One lane's whole transient on the CTA (tran_lane's run): the operating
// point through op.zig's ladder, then the trapezoidal steps with the
// predictor, LTE control, order promotion and source breakpoints.
template <typename V, typename OpT, bool kHasB3, uint32_t kW>
__device__ void block_tran_lane(const BlockDev& D, const LaneDev& L, const TranDev& P, const LaneOpts& o,
                                unsigned char* base, unsigned char* cold, unsigned char* ring, double* tslab,
                                uint64_t* red, uint32_t lane) {
  const TopoDev& T = D.T;
  const int tid = threadIdx.x;
  const uint32_t n = T.n, nq = T.n_qt;
  const BlockMem<V> b = block_carve<V>(D, base, cold, ring, sizeof(OpT));
  uint32_t refinements = 0;
  const LaneMem& m = b.m;
  double* cur = tslab;
  double* prev = cur + n;
  double* qh = prev + n;  // 4 slots of n: the row-charge ring
  double* ipr = qh + 4 * size_t(n);
  double* qt = ipr + n;   // 4 slots of nq: the LTE-state ring
  double* ipt = qt + 4 * size_t(nq);
  double* vsrc = ipt + nq;  // the V and I sources at the current time point
  double* tmr = vsrc + T.n_src;  // 8 n_src: the PULSE corner timers
  const double* rec = L.rec + size_t(lane) * T.rec_size;
  const size_t at = size_t(lane) * n;
  uint32_t stat[kTsN];
  for (int k = 0; k < kTsN; ++k) stat[k] = 0;
  if (tid == 0) {
    b.v[T.ntv + n] = V(0);
    b.v[T.ntv + n + 1] = V(1);
    b.v[T.ntv + n + 2] = V(0);
    m.st[T.n_stage + kGCellZero] = 0.0;
    m.st[T.n_stage + kGCellOne] = 1.0;
  }

  const double dt_max = P.dt_max;
  const double delmin = 1e-11 * dt_max;
  const double min_break = 10.0 * delmin;
  double dt = 0.0, t = 0.0, bp_next = 0.0, bp_save_dt = div_rn(P.t_stop, 50.0);
  double dt_old[6];
  for (int k = 0; k < 6; ++k) dt_old[k] = dt_max;
  int order = 1;
  uint32_t steps = 0, hb = 0, n_rec = 0;
  bool have_bp = false, bp_clamped = false, lim_active = false;
  SimDev sim;
  sim.t = 0.0;
  sim.src_scale = 1.0;
  sim.kind = 2;
  __syncthreads();

  auto record = [&](double tr) {
    if (P.out_t && n_rec < P.max_pts) {
      if (tid == 0) P.out_t[size_t(lane) * P.max_pts + n_rec] = tr;
      for (uint32_t k = tid; k < P.n_probes; k += kW)
        P.out_v[(size_t(lane) * P.max_pts + n_rec) * P.n_probes + k] = m.x[P.probes[k]];
      ++n_rec;
    }
  };

  // operating point (op.solve with tran_op): op.zig's ladder from the cold
  // start, the source waves at t = 0 (kind 2), every run through one call
  // site, the ladder's state in L.ladder
  int rc = 0;
  {
    LadderMove mv{kStartCold, false, false, true, 3u, 0u};
    LadderDev ls{kRungPlain};
    LaneOpts op = o;
    op.residual_tol = 1e-9;
    op.gmin = 0.0;
    op.max_iter = 100;
    bool left = false;
    for (;;) {
      if (mv.done) break;
      if (mv.save)
        for (uint32_t i = tid; i < n; i += kW) L.x_good[at + i] = m.x[i];
      if (mv.start == kStartGood)
        for (uint32_t i = tid; i < n; i += kW) m.x[i] = L.x_good[at + i];
      if (mv.start == kStartCold) {
        for (uint32_t i = tid; i < n; i += kW) m.x[i] = 0.0;
        cold_images(T, rec, m.lim, tid, kW);
      }
      __syncthreads();
      lim_active = mv.start == kStartCold && T.nlim != 0;
      const LadderRun run = ladder_run(op, &ls);
      LaneOpts ro = op;
      ro.gstamp = run.gs;
      ro.max_iter = run.max_iter;
      SimDev rs = sim;
      rs.src_scale = run.src;
      rs.gmin = run.gmin_dev;
      fill_sources<kW>(T, rec, rs, vsrc, tid);
      uint32_t it = 0;
      const int r = block_tran_newton<V, OpT, kHasB3, kW>(D, b, rec, ro, rs, nullptr, lim_active, mv.init_fix, it,
                                                           vsrc, red, tid, refinements);
      if (r == 2) {
        left = true;
        break;
      }
      mv = ladder_decide(ls, r == 0, it);
    }
    lim_active = false;
    stat[kTsOpIters] = mv.report;
    if (left) {
      stat[kTsStatus] = kTranLeftTape;
      rc = 2;
    } else {
      rc = mv.result < 3 ? 0 : 1;
    }
  }
  if (rc == 1) {
    stat[kTsStatus] = kTranOpFailed;
  } else if (rc == 0) {
    const bool has_charge = T.q_ptr[n] != 0 || T.c_ptr[T.nnz] != 0;
    auto slot = [&](double* base_, uint32_t len, uint32_t r) { return base_ + size_t((hb + r) & 3u) * len; };
    for (uint32_t i = tid; i < n; i += kW) {
      cur[i] = m.x[i];
      prev[i] = m.x[i];
    }
    // charge histories, flat at q(x_op); no dynamic current yet
    sim.kind = 1;
    eval_all<kHasB3, kW>(T, rec, m, false, sim, tid, true);
    for (uint32_t i = tid; i < 4 * n; i += kW) qh[i] = 0.0;
    __syncthreads();
    block_row_charges<kW>(T, m.st, qh + n, tid);
    state_charges<kW>(T, rec, m.x, qt + nq, tid);
    __syncthreads();
    for (uint32_t i = tid; i < n; i += kW) {
      qh[2 * n + i] = qh[n + i];
      qh[3 * n + i] = qh[n + i];
      ipr[i] = 0.0;
    }
    for (uint32_t j = tid; j < nq; j += kW) {
      qt[2 * nq + j] = qt[nq + j];
      qt[3 * nq + j] = qt[nq + j];
      ipt[j] = 0.0;
    }
    __syncthreads();
    pulse_timers<kW>(T, rec, tmr, tid);
    dt = fmin(div_rn(fmin(P.t_step, div_rn(P.t_stop, 100.0)), 10.0), dt_max);
    double bp0;
    if (next_bp<kW>(T, rec, tmr, min_break, bp0, tid, red)) dt = fmin(dt, 0.1 * bp0);
    dt = div_rn(dt, 10.0);
    record(0.0);
    LaneOpts nr = o;
    nr.residual_tol = CUDART_INF;
    nr.gmin = 0.0;
    nr.max_iter = 100;
    for (;;) {
      if (!(t < P.t_stop && !almost_equal_ulps(t, P.t_stop, 100) && steps < P.max_steps)) break;
      const double t_dev = t + dt;
      sim.kind = 1;
      sim.t = t_dev;
      const bool trap = order == 2;
      const double ag0 = trap ? div_rn(div_rn(1.0, dt), 1.0 - 0.5) : div_rn(1.0, dt);
      const double ag1 = trap ? div_rn(0.5, 1.0 - 0.5) : 1.0;
      // predictor, limited against the accepted point
      const double xfact = div_rn(dt, dt_old[0]);
      for (uint32_t i = tid; i < n; i += kW) {
        m.x[i] = cur[i] + xfact * (cur[i] - prev[i]);
        m.xo[i] = cur[i];
      }
      __syncthreads();
      apply_limits<kHasB3, kW>(T, rec, m, false, tid);
      lim_active = T.nlim != 0;
      __syncthreads();
      const BlockCompanion c{ag0, ag1, trap, slot(qh, n, 1), ipr};
      uint32_t iters = 0;
      fill_sources<kW>(T, rec, sim, vsrc, tid);
      rc = block_tran_newton<V, OpT, kHasB3, kW>(D, b, rec, nr, sim, &c, lim_active, false, iters, vsrc, red, tid,
                                                 refinements);
      lim_active = false;
      if (rc == 2) {
        stat[kTsStatus] = kTranLeftTape;
        break;
      }
      stat[kTsAttempts] += 1;
      stat[kTsNrIters] += iters;
      if (rc != 0) {
        stat[kTsRejNewton] += 1;
        order = 1;
        dt = div_rn(dt, 8.0);
        if (dt < P.dt_min) {
          stat[kTsStatus] = kTranUnderflow;
          break;
        }
        continue;
      }
      double dt_next = steps == 0 ? dt : fmin(dt * 2.0, dt_max);
      if (has_charge) {
        eval_all<kHasB3, kW>(T, rec, m, false, sim, tid, true);
        __syncthreads();
        block_row_charges<kW>(T, m.st, slot(qh, n, 0), tid);
        state_charges<kW>(T, rec, m.x, slot(qt, nq, 0), tid);
        __syncthreads();
      }
      const double dt1 = dt_old[0], dt2 = dt_old[1];
      if (has_charge && steps > 0) {
        const int mth = trap ? 2 : 1;
        const double del = step_bound<kW>(mth, mth, nq, slot(qt, nq, 0), slot(qt, nq, 1), slot(qt, nq, 2),
                                          slot(qt, nq, 3), ipt, ag0, ag1, dt, dt1, dt2, P, tid, red);
        if (!(del >= 0.9 * dt)) {
          stat[kTsRejLte] += 1;
          if (del != del) {
            order = 1;
            dt = div_rn(dt, 8.0);
          } else {
            dt = del;
          }
          if (dt < P.dt_min) {
            stat[kTsStatus] = kTranUnderflow;
            break;
          }
          continue;
        }
        dt_next = fmin(fmin(fmax(del, P.dt_min), 2.0 * dt), dt_max);
      }
      if (has_charge) {
        if (steps > 0 && order == 1) {
          const double trial_del = step_bound<kW>(2, 1, nq, slot(qt, nq, 0), slot(qt, nq, 1), slot(qt, nq, 2),
                                                  slot(qt, nq, 3), ipt, ag0, ag1, dt, dt1, dt2, P, tid, red);
          if (trial_del == trial_del) {
            const double nd2 = fmin(2.0 * dt, trial_del);
            if (nd2 > 1.05 * dt) order = 2;
            dt_next = fmin(fmax(nd2, P.dt_min), dt_max);
          }
        }
        // integrator.advanceCurrent over rows and states, then the rotation
        const double* q0 = slot(qh, n, 0);
        const double* q1 = slot(qh, n, 1);
        for (uint32_t i = tid; i < n; i += kW) {
          const double d = ag0 * (q0[i] - q1[i]);
          ipr[i] = trap ? d - ag1 * ipr[i] : d;
        }
        const double* s0 = slot(qt, nq, 0);
        const double* s1 = slot(qt, nq, 1);
        for (uint32_t j = tid; j < nq; j += kW) {
          const double d = ag0 * (s0[j] - s1[j]);
          ipt[j] = trap ? d - ag1 * ipt[j] : d;
        }
        hb = (hb + 3u) & 3u;
      }
      for (int k = 5; k > 0; --k) dt_old[k] = dt_old[k - 1];
      dt_old[0] = dt;
      for (uint32_t i = tid; i < n; i += kW) {
        prev[i] = cur[i];
        cur[i] = m.x[i];
      }
      __syncthreads();
      t = t + dt;
      steps += 1;
      stat[kTsAccepted] += 1;
      const double t_new = t;
      if (have_bp) {
        const bool landed = bp_clamped ? fabs(t_new - bp_next) <= min_break
                                       : (bp_next - t_new <= delmin || almost_equal_ulps(t_new, bp_next, 100));
        if (landed) {
          stat[kTsBpLandings] += 1;
          order = 1;
          double shrink = bp_save_dt, nb;
          if (next_bp<kW>(T, rec, tmr, t_new + min_break, nb, tid, red)) shrink = fmin(shrink, nb - t_new);
          dt_next = fmin(dt_next, 0.1 * shrink);
        }
        have_bp = false;
      }
      record(t_new);
      have_bp = next_bp<kW>(T, rec, tmr, t_new + min_break, bp_next, tid, red);
      bp_clamped = false;
      if (have_bp) {
        const double dt_to_bp = bp_next - t_new;
        if (dt_to_bp < dt_next) {
          bp_save_dt = dt_next;
          dt_next = dt_to_bp;
          bp_clamped = true;
        }
      }
      dt = dt_next;
      if (t_new + dt > P.t_stop) dt = P.t_stop - t_new;
    }
    if (stat[kTsStatus] == kTranDone && steps >= P.max_steps && !(t >= P.t_stop || almost_equal_ulps(t, P.t_stop, 100)))
      stat[kTsStatus] = kTranMaxSteps;
    for (uint32_t i = tid; i < n; i += kW) m.x[i] = cur[i];
    __syncthreads();
  }
  for (uint32_t i = tid; i < n; i += kW) L.x[at + i] = m.x[i];
  if (tid < kTsN) P.stats[size_t(lane) * kTsN + tid] = stat[tid];
  if (tid == 0) {
    if (P.n_pts) P.n_pts[lane] = n_rec;
    L.status[lane] = kConverged;
    if (D.refine_out) D.refine_out[lane] = refinements;
  }
}

// Persistent grid over the lanes, one CTA per lane at a time; the working
// set placed as the DC block lanes place it (shared memory, split or slab),
// the run state in the CTA's part of tslab.
template <typename V, typename OpT, bool kHasB3, uint32_t kW>
__global__ void __launch_bounds__(kW, 2) tran_block_kernel(BlockDev D, LaneDev L, TranDev P, LaneOpts o,
                                                          double* tslab, size_t tslab_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint64_t red[kW / 32];
  unsigned char* own = D.slab + size_t(blockIdx.x) * (D.split ? D.cold_bytes : D.lane_bytes);
  unsigned char* base = D.in_smem ? smem_raw : own;
  unsigned char* ring = smem_raw + (D.in_smem ? D.lane_bytes : 0u);
  double* ts = tslab + size_t(blockIdx.x) * tslab_stride;
  for (uint32_t lane = blockIdx.x; lane < L.n_lanes; lane += gridDim.x) {
    block_tran_lane<V, OpT, kHasB3, kW>(D, L, P, o, base, own, ring, ts, red, lane);
    __syncthreads();
  }
}

template <typename V, typename OpT, bool kHasB3>
cudaError_t launch_tran_t(const BlockDev& D, const LaneDev& L, const TranDev& P, const LaneOpts& o, double* tslab,
                          size_t tslab_stride, cudaStream_t s) {
  auto* k = tran_block_kernel<V, OpT, kHasB3, kBlockThreads>;
  const size_t smem = (D.in_smem ? D.lane_bytes : 0) + D.ring_bytes;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  const uint32_t grid = D.grid < L.n_lanes ? D.grid : L.n_lanes;
  k<<<grid > 0 ? grid : 1, kBlockThreads, smem, s>>>(D, L, P, o, tslab, tslab_stride);
  return cudaGetLastError();
}

// The eight instantiations: precision x op format x BSIM3.
#define ESL_BLOCK_DISPATCH(F, ...)                                                     \
  do {                                                                                 \
    if (mixed) {                                                                       \
      if (long_ops) return has_b3 ? F<float, uint4, true>(__VA_ARGS__) : F<float, uint4, false>(__VA_ARGS__); \
      return has_b3 ? F<float, uint2, true>(__VA_ARGS__) : F<float, uint2, false>(__VA_ARGS__);               \
    }                                                                                  \
    if (long_ops) return has_b3 ? F<double, uint4, true>(__VA_ARGS__) : F<double, uint4, false>(__VA_ARGS__); \
    return has_b3 ? F<double, uint2, true>(__VA_ARGS__) : F<double, uint2, false>(__VA_ARGS__);               \
  } while (0)

}  // namespace

cudaError_t launch_dc_block(const BlockDev& D, const LaneDev& L, const LaneOpts& o, bool mixed, bool has_b3,
                            cudaStream_t s) {
  const bool long_ops = D.op_bytes == 16;
  ESL_BLOCK_DISPATCH(launch_t, D, L, o, s);
}

size_t tran_block_slab(const TopoDev& T) { return tran_block_slab_doubles(T); }

cudaError_t launch_tran_block(const BlockDev& D, const LaneDev& L, const TranDev& P, const LaneOpts& o, bool mixed,
                              bool has_b3, double* tslab, cudaStream_t s) {
  const size_t stride = tran_block_slab_doubles(D.T);
  const bool long_ops = D.op_bytes == 16;
  ESL_BLOCK_DISPATCH(launch_tran_t, D, L, P, o, tslab, stride, s);
}

int block_occupancy(bool mixed, bool long_ops, bool has_b3, size_t smem) {
  ESL_BLOCK_DISPATCH(occupancy_t, smem);
}

cudaError_t launch_dc_block_group(const BlockDev* d_Ds, const LaneDev* d_Ls, const uint2* d_items, uint32_t n_items,
                                  uint32_t* d_next, const LaneOpts& o, unsigned char* slab, size_t slab_stride,
                                  size_t smem, uint32_t ring_at, uint32_t grid, bool mixed, bool long_ops, bool has_b3,
                                  cudaStream_t s) {
  ESL_BLOCK_DISPATCH(launch_group_t, d_Ds, d_Ls, d_items, n_items, d_next, o, slab, slab_stride, smem, ring_at, grid,
                     s);
}

int block_group_occupancy(bool mixed, bool long_ops, bool has_b3, size_t smem) {
  ESL_BLOCK_DISPATCH(group_occupancy_t, smem);
}

#undef ESL_BLOCK_DISPATCH

cudaError_t launch_block_lead(const BlockDev& D, const LaneDev& L, uint32_t lane, double* out, bool has_b3,
                              cudaStream_t s) {
  if (has_b3) block_lead_kernel<true, kBlockThreads><<<1, kBlockThreads, 0, s>>>(D, L, lane, out);
  else block_lead_kernel<false, kBlockThreads><<<1, kBlockThreads, 0, s>>>(D, L, lane, out);
  return cudaGetLastError();
}

}  // namespace esl

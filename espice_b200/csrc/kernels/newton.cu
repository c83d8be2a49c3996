// Fused sweep-lane Newton kernel for sm_100a: one warp per lane, the lane's
// whole working set in shared memory, every phase of a Newton iteration in
// one launch (eval + stamp -> assemble -> refactor on the lead lane's frozen
// pivot tape with the forward solve merged in -> back solve -> update ->
// limiting -> gates), looping on the device until the lane converges, runs
// out of iterations, or needs the host (a pivot the frozen tape cannot stand
// in for).
//
// Reference path this replaces (src/analysis/gpu_lanes.zig:758-845 and the
// 12 kernels of src/solver/lane_device.zig, bodies in
// src/solver/lane_kernels.zig:49-301): there, each Newton tick is eight or
// more launches of one thread per lane over lane-major HBM planes plus two
// host syncs. Here one launch runs every tick of every lane.
//
// Shared memory of a CTA: the topology's program blob (warp programs and
// the assembly gather program, staged once per CTA), then one block per
// lane (warp): x | xo | rhs | diag | v | staging | limited images, where
// v = [tape values | y | 0.0 | 1.0 | sink] is the value space of the warp
// programs. The hot loops address shared memory explicitly (32-bit shared
// addresses, ld.shared / st.shared).
//
// Bitwise contract: the refactor and solve ops use __dmul_rn / __dsub_rn /
// __ddiv_rn in the reference's operation order per value, so a lane's L, U
// and dx are bitwise the CPU replay (sparse_lu.zig refactor + solve) on the
// same matrix. The file builds with --fmad=false so the stamp and gates
// round as the reference's strict-float code does.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <mutex>

#include "launch.h"
#include "lanes.cuh"
#include "models.cuh"
#include "bsim3.cuh"
#include "lane_eval.cuh"
#include "ladder.cuh"
#include "tran_core.cuh"

namespace esl {

namespace {

__device__ __forceinline__ double lds(uint32_t a) {
  double r;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(r) : "r"(a));
  return r;
}
__device__ __forceinline__ void sts(uint32_t a, double x) {
  asm volatile("st.shared.f64 [%0], %1;" ::"r"(a), "d"(x) : "memory");
}
__device__ __forceinline__ uint32_t lds_u32(uint32_t a) {
  uint32_t r;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(r) : "r"(a));
  return r;
}
__device__ __forceinline__ uint2 lds_u2(uint32_t a) {
  uint2 r;
  asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(r.x), "=r"(r.y) : "r"(a));
  return r;
}
__device__ __forceinline__ uint32_t saddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t w = __shfl_xor_sync(kFull, v, o);
    v = w > v ? w : v;
  }
  return v;
}

__device__ __forceinline__ double warp_fmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}


// Copies the program blob into the CTA's shared memory (every thread takes
// part) and returns the lanes' area that follows it.
__device__ __forceinline__ double* stage_programs(const TopoDev& T, unsigned char* smem) {
  const uint4* src = reinterpret_cast<const uint4*>(T.prog);
  uint4* dst = reinterpret_cast<uint4*>(smem);
  for (uint32_t i = threadIdx.x; i < T.prog_bytes / 16; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  return reinterpret_cast<double*>(smem + T.prog_bytes);
}


// Assembly: every residual row and pattern slot sums its staging cells in
// the reference's stamp order (batch, instance, local row, local column),
// the ground pin last; slots land in their tape values, the diagonal is
// copied for the gates, y = P(-rhs) is loaded and fill-in zeroed, all in
// one gather program (groups of 32 cells; a cell t of group g sums
// src[off + k * 32 + t], lane-block indices, then writes three places).
// One gather cell's sum: +0.0 plus the d values at lane-block indices
// src[k * 32] (shared addresses), added in list order (d is the same for
// the whole warp). Software-pipelined in blocks of four: while a block's
// four additions run, the next block's values and the indices of the block
// after it are in flight, so a long list (a supply node's row sums one cell
// per device on it) costs about its chain of additions, not a
// shared-memory round trip per term.
__device__ __forceinline__ double gather_sum(uint32_t src, uint32_t d, uint32_t lb) {
  double s = 0.0;
  const uint32_t nb = d >> 2;
  uint32_t k = 0;
  if (nb >= 2) {
    uint32_t i0 = lds_u32(src), i1 = lds_u32(src + 128), i2 = lds_u32(src + 256), i3 = lds_u32(src + 384);
    double v0 = lds(lb + 8 * i0), v1 = lds(lb + 8 * i1), v2 = lds(lb + 8 * i2), v3 = lds(lb + 8 * i3);
    i0 = lds_u32(src + 512);
    i1 = lds_u32(src + 640);
    i2 = lds_u32(src + 768);
    i3 = lds_u32(src + 896);
    for (uint32_t b = 1; b < nb; ++b) {
      const double w0 = lds(lb + 8 * i0), w1 = lds(lb + 8 * i1), w2 = lds(lb + 8 * i2), w3 = lds(lb + 8 * i3);
      if (b + 1 < nb) {
        const uint32_t at = src + 512 * (b + 1);
        i0 = lds_u32(at);
        i1 = lds_u32(at + 128);
        i2 = lds_u32(at + 256);
        i3 = lds_u32(at + 384);
      }
      s = __dadd_rn(s, v0);
      s = __dadd_rn(s, v1);
      s = __dadd_rn(s, v2);
      s = __dadd_rn(s, v3);
      v0 = w0;
      v1 = w1;
      v2 = w2;
      v3 = w3;
    }
    s = __dadd_rn(s, v0);
    s = __dadd_rn(s, v1);
    s = __dadd_rn(s, v2);
    s = __dadd_rn(s, v3);
    k = nb << 2;
  }
  for (; k < d; ++k) s = __dadd_rn(s, lds(lb + 8 * lds_u32(src + 128 * k)));
  return s;
}

// Assembly: the segmented gather. Every thread sums its column's terms,
// software-pipelined in blocks of eight: while a block's additions run, the
// next block's values and the indices of the block after it are in flight.
// At each segment's end a thread whose cell ends there stores it and starts
// over; the next segment's destinations are loaded a segment ahead.
__device__ void assemble(const TopoDev& T, uint32_t prog, const LaneMem& m, int tid) {
  const uint32_t lb = saddr(m.base);
  const uint32_t sb = T.g_seg_blocks, nblk = T.g_nseg * sb;
  if (nblk == 0) return;
  const uint32_t src = prog + T.o_g_src + 4 * tid;
  uint32_t dp = prog + T.o_g_dst + 4 * tid;
  uint32_t d0 = lds_u32(dp), d1 = lds_u32(dp + 128), d2 = lds_u32(dp + 256);
  dp += 384;
  uint32_t i[kGatherBlock];
  double v[kGatherBlock];
#pragma unroll
  for (int j = 0; j < kGatherBlock; ++j) i[j] = lds_u32(src + 128 * j);
#pragma unroll
  for (int j = 0; j < kGatherBlock; ++j) v[j] = lds(lb + 8 * i[j]);
  {
    const uint32_t at = src + 128 * kGatherBlock * (nblk > 1 ? 1u : 0u);
#pragma unroll
    for (int j = 0; j < kGatherBlock; ++j) i[j] = lds_u32(at + 128 * j);
  }
  double s = 0.0;
  uint32_t left = sb;
  for (uint32_t b = 0; b < nblk; ++b) {
    double w[kGatherBlock];
#pragma unroll
    for (int j = 0; j < kGatherBlock; ++j) w[j] = lds(lb + 8 * i[j]);
    if (b + 2 < nblk) {
      const uint32_t at = src + 128 * kGatherBlock * (b + 2);
#pragma unroll
      for (int j = 0; j < kGatherBlock; ++j) i[j] = lds_u32(at + 128 * j);
    }
#pragma unroll
    for (int j = 0; j < kGatherBlock; ++j) s = __dadd_rn(s, v[j]);
#pragma unroll
    for (int j = 0; j < kGatherBlock; ++j) v[j] = w[j];
    if (--left == 0) {
      left = sb;
      const uint32_t e0 = lds_u32(dp), e1 = lds_u32(dp + 128), e2 = lds_u32(dp + 256);
      dp += 384;
      if (d0 & kGatherEnd) {
        sts(lb + 8 * (d0 & ~kGatherEnd), s);
        sts(lb + 8 * d1, s);
        sts(lb + 8 * d2, -s);
        s = 0.0;
      }
      d0 = e0;
      d1 = e1;
      d2 = e2;
    }
  }
}


// Runs one warp program over v (shared address vb): rows of 32 ops, each
// row divisions only or multiply-subtracts only (warp-uniform branches),
// thread t taking op t, the next row's op fetched while this one runs.
// Padding ops move 1.0 / 0.0 into the sink. Returns true when a division
// failed its pivot test (thread-local). Compiled out of line: the loop's
// own register allocation measured about 1% faster on the transient than
// inlined into the fused kernels.
__device__ __noinline__ bool run_rows(uint32_t ops, uint32_t rows, uint32_t vb, int tid) {
  bool bad = false;
  if (rows == 0) return false;
  uint2 op = lds_u2(ops + 8 * tid);
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t rn = r + 1 < rows ? r + 1 : r;
    const uint2 next = lds_u2(ops + 8 * (rn * 32 + tid));
    const uint32_t kind = op.x >> 28;
    const uint32_t pd = vb + 8 * (op.x & 0x0fffffffu);
    const uint32_t pa = vb + 8 * (op.y & 0xffffu), pb = vb + 8 * (op.y >> 16);
    // Two warp-uniform paths (a switch here compiles to an indirect jump
    // that costs more than the op): the divisions with their checks
    // predicated on the kind, and the multiply-subtracts (the solves skip a
    // zero multiplier, the refactor never does).
    const double a = lds(pa), b = lds(pb);
    if (kind == kOpDivGrowth || kind == kOpDivScaled || kind == kOpDivY) {
      // dividend at b (the op's own value; 1.0 on padding)
      const double q = div_rn(b, a);
      if (kind == kOpDivGrowth && !(fabs(a) >= __dmul_rn(kGrowth, fabs(b)))) bad = true;
      if (kind == kOpDivScaled && !(fabs(q) < CUDART_INF)) bad = true;
      sts(pd, q);
    } else {
      const double d = lds(pd);
      if (kind == kOpFlop || b != 0.0) sts(pd, __dsub_rn(d, __dmul_rn(a, b)));
    }
    __syncwarp();
    op = next;
  }
  return bad;
}

// Refactor on the frozen tape with the forward solve merged in (program A),
// then the lane kernel's peel tests (lane_kernels.zig Bodies.refactor and
// LaneSolver.wideMultipliers): U entries finite, pivots alive, L multipliers
// within 1 / pivot_tol. y must hold P(-rhs). Warp-uniform verdict.
__device__ bool refactor_forward(const TopoDev& T, uint32_t prog, double* v, int tid) {
  bool bad = run_rows(prog + T.o_a_ops, T.a_rows, saddr(v), tid);
  const uint32_t l0 = T.nu + T.n;
  for (uint32_t s = tid; s < T.nu; s += 32)
    if (dbits(v[s] - v[s]) != 0) bad = true;
  for (uint32_t k = tid; k < T.n; k += 32) {
    const double d = v[T.nu + k];
    if (d == 0.0 || !(fabs(d) < CUDART_INF)) bad = true;
  }
  for (uint32_t s = tid; s < T.nl; s += 32)
    if (!T.l_scaled[s] && !(fabs(v[l0 + s]) <= kWide)) bad = true;
  return __any_sync(kFull, bad);
}

__device__ __forceinline__ void back_solve(const TopoDev& T, uint32_t prog, double* v, int tid) {
  run_rows(prog + T.o_b_ops, T.b_rows, saddr(v), tid);
}

__device__ __forceinline__ void load_y(const TopoDev& T, const double* rhs, double* y, int tid) {
  for (uint32_t r = tid; r < T.n; r += 32) y[T.pinv[r]] = -rhs[r];
}

__device__ __forceinline__ void init_consts(const TopoDev& T, double* v, int tid) {
  if (tid == 0) {
    v[T.ntv + T.n] = 0.0;
    v[T.ntv + T.n + 1] = 1.0;
    v[T.ntv + T.n + 2] = 0.0;
  }
}



}  // namespace

// One lane's DC Newton solve (converger.zig newtonLanes at W = 1 with the
// lane's own direct solver), by the warp that owns it.
// `ld`: an operating-point lane's ladder state (the run's gmin stamps,
// source factor and cap), null for a plain DC solve.
template <bool kHasB3, bool kLadder = false>
__device__ void dc_solve_lane(const TopoDev& T, const LaneDev& L, const LaneOpts& o, uint32_t prog, double* block,
                              uint32_t lane, int tid, const LadderDev* ld = nullptr) {
  const uint32_t status = L.status[lane];
  const bool resuming = L.resume && status == kNeedSolve;
  if (!(status == kRunning || resuming)) return;

  const uint32_t n = T.n;
  LaneMem m = carve(T, block);
  const double* rec = L.rec + size_t(lane) * T.rec_size;
  for (uint32_t i = tid; i < n; i += 32) m.x[i] = L.x[size_t(lane) * n + i];
  for (uint32_t i = tid; i < T.nlim; i += 32) m.lim[i] = L.lim[size_t(lane) * T.nlim + i];
  init_consts(T, m.v, tid);
  bool lim_active = L.lim_active[lane] != 0;
  uint32_t flags = L.flags[lane];
  uint32_t iter = L.iters[lane];
  double limit = L.limit[lane];
  const LadderRun run = ladder_run(o, kLadder ? ld : nullptr);
  const uint32_t max_iter = run.max_iter;
  SimDev sim;
  sim.t = 0.0;
  sim.src_scale = run.src;
  sim.kind = 0;
  sim.gmin = run.gmin_dev;
  bool have_step = false;
  if (resuming) {
    for (uint32_t i = tid; i < n; i += 32) {
      m.rhs[i] = L.rhs[size_t(lane) * n + i];
      m.diag[i] = L.diag[size_t(lane) * n + i];
    }
    // the host's dx, permuted as the device solve leaves it
    for (uint32_t j = tid; j < n; j += 32) m.y[j] = L.dx[size_t(lane) * n + T.qcol[j]];
    have_step = true;
  }
  __syncwarp();

  for (; iter < max_iter; ++iter) {
    if (!have_step) {
      eval_all<kHasB3>(T, rec, m, lim_active, sim, tid);
      __syncwarp();
      assemble(T, prog, m, tid);
      __syncwarp();
      if (o.gmin > 0) {
        // loadExtras: diagonal gmin and its residual form
        for (uint32_t p = tid; p < T.nnz; p += 32) {
          const uint32_t row = T.slot_row[p];
          if (row != kNoDiag) {
            const double d = m.diag[row] + o.gmin;
            m.diag[row] = d;
            m.v[T.amap[p]] = d;
          }
        }
        for (uint32_t i = tid; i < n; i += 32) m.rhs[i] += o.gmin * m.x[i];
        __syncwarp();
        load_y(T, m.rhs, m.y, tid);
        __syncwarp();
      }
      if (run.gs > 0.0) {
        // loadGmin at the gmin-stepping stamps (converger.zig:696-713);
        // every stamp its own row and slot
        for (uint32_t k = tid; k < T.n_gst; k += 32) {
          const uint32_t slot = T.gst[3 * k], row = T.gst[3 * k + 1], col = T.gst[3 * k + 2];
          const uint32_t at = T.amap[slot], dr = T.slot_row[slot];
          const double d = m.v[at] + run.gs;
          m.v[at] = d;
          if (dr != kNoDiag) m.diag[dr] = d;
          m.rhs[row] += run.gs * m.x[col];
        }
        __syncwarp();
        load_y(T, m.rhs, m.y, tid);
        __syncwarp();
      }
      if (iter == 0) {
        // plausibleLimit: 1e3 x the start's scale, at least x_plausible
        double g = 1.0;
        uint64_t xm = 0, fm = 0;
        for (uint32_t i = tid; i < n; i += 32) {
          g = fmax(g, fabs(m.diag[i]));
          const uint64_t bx = dbits(fabs(m.x[i])), bf = dbits(fabs(m.rhs[i]));
          xm = bx > xm ? bx : xm;
          fm = bf > fm ? bf : fm;
        }
        g = warp_fmax(g);
        xm = warp_max_u64(xm);
        fm = warp_max_u64(fm);
        const double scale = fmin(fmax(from_bits(xm), from_bits(fm) * g), 1e18);
        limit = !(1e3 * scale > kXPlausible) ? kXPlausible : 1e3 * scale;
      }
      const bool host_mode = (flags & 2u) != 0;
      bool bad = true;
      if (!host_mode) bad = refactor_forward(T, prog, m.v, tid);
      if (bad) {
        // Pause: the host factors this lane with its own direct solver.
        const size_t base = size_t(lane) * n;
        gather_pattern(T, m, L.a_vals + size_t(lane) * T.nnz, tid);
        for (uint32_t i = tid; i < n; i += 32) {
          L.x[base + i] = m.x[i];
          L.rhs[base + i] = m.rhs[i];
          L.diag[base + i] = m.diag[i];
        }
        for (uint32_t i = tid; i < T.nlim; i += 32) L.lim[size_t(lane) * T.nlim + i] = m.lim[i];
        if (tid == 0) {
          L.lim_active[lane] = lim_active;
          L.flags[lane] = flags | 2u;
          L.iters[lane] = iter;
          L.limit[lane] = limit;
          L.status[lane] = kNeedSolve;
          atomicAdd(L.n_paused, 1u);
        }
        return;
      }
      back_solve(T, prog, m.v, tid);
    }
    have_step = false;
    __syncwarp();

    // finalizeStep: x_old = x, x += dx, delta score (updateAndNorm)
    uint64_t worst = 0;
    for (uint32_t j = tid; j < n; j += 32) {
      const uint32_t i = T.qcol[j];
      const double d = m.y[j];
      const double xold = m.x[i];
      const double xn = xold + d;
      m.xo[i] = xold;
      m.x[i] = xn;
      const double tol = o.reltol * fmax(fabs(xn), fabs(xold)) + (T.cur_row[i] ? o.abstol : o.vntol);
      const bool finite = fabs(xn) < CUDART_INF && fabs(d) < CUDART_INF;
      const double qv = div_rn(fabs(d), tol);
      const double score = !finite ? CUDART_INF : (qv == qv ? qv : 0.0);
      const uint64_t b = dbits(score);
      worst = b > worst ? b : worst;
    }
    worst = warp_max_u64(worst);
    __syncwarp();
    const bool limited = apply_limits<kHasB3>(T, rec, m, lim_active, tid);
    if (T.nlim) lim_active = true;

    bool ok = !limited && iter != 0 && !(from_bits(worst) >= 1.0);
    if (ok) {
      bool p = true;
      for (uint32_t i = tid; i < n; i += 32) p &= fabs(m.x[i]) <= limit;
      ok = __all_sync(kFull, p);
    }
    if (ok) {
      bool p = true;
      for (uint32_t i = tid; i < n; i += 32) p &= fabs(m.rhs[i]) <= residual_gate(o, m.diag[i], m.x[i]);
      ok = __all_sync(kFull, p);
    }
    if (ok) {
      if (flags & 1u) {
        flags &= ~1u;  // INITFIX -> INITFLOAT: one more passing iterate
      } else {
        for (uint32_t i = tid; i < n; i += 32) L.x[size_t(lane) * n + i] = m.xo[i];
        if (tid == 0) {
          L.iters[lane] = iter + 1;
          L.status[lane] = kConverged;
          L.lim_active[lane] = 0;
        }
        return;
      }
    }
    __syncwarp();
  }
  for (uint32_t i = tid; i < n; i += 32) L.x[size_t(lane) * n + i] = m.x[i];
  if (tid == 0) {
    L.iters[lane] = max_iter;
    L.status[lane] = kMaxIter;
    L.lim_active[lane] = 0;
  }
}

// DC Newton over independent sweep points (sweep/lanes.zig solveBatch:
// each lane bitwise its own converger.run), one warp per lane; a persistent
// grid, each CTA staging the programs once and taking lanes in turn.
template <bool kHasB3, bool kLadder>
__global__ void __launch_bounds__(256) dc_newton_kernel(TopoDev T, LaneDev L, LaneOpts o) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* lanes_smem = stage_programs(T, smem_raw);
  const uint32_t prog = saddr(smem_raw);
  const int tid = threadIdx.x & 31;
  const uint32_t warps = blockDim.x >> 5, w = threadIdx.x >> 5;
  double* block = lanes_smem + size_t(w) * T.smem_doubles;
  for (uint32_t lane = blockIdx.x * warps + w; lane < L.n_lanes; lane += gridDim.x * warps) {
    if constexpr (!kLadder) {
      dc_solve_lane<kHasB3>(T, L, o, prog, block, lane, tid);
    } else {
      // an operating-point lane: Newton runs until the ladder is done or the
      // lane pauses for a host factor (a singular host factor ends a run)
      for (;;) {
        const uint32_t st = *(volatile uint32_t*)(L.status + lane);
        if (st == kRunning || (L.resume && st == kNeedSolve)) {
          dc_solve_lane<kHasB3, true>(T, L, o, prog, block, lane, tid, L.ladder + lane);
          __syncwarp();
          if (*(volatile uint32_t*)(L.status + lane) == kNeedSolve) break;
        } else if (!(st == kSingular && L.ladder[lane].rung != kRungDone)) {
          break;
        }
        if (!ladder_step(T, L, lane, tid, 32)) break;
      }
    }
    __syncwarp();
  }
}

// Standalone lane refactor + solve on the frozen tape (the reference's
// arp_lane_refactor + arp_lane_solve): A [lane][nnz] and rhs [lane][n] in
// HBM, the tape values (U, diagonal, L) [lane][ntv], dx [lane][n] and the
// peel verdict out. One warp per lane; the tape values stay in shared
// memory between the scatter, the factor and the solves.
__global__ void __launch_bounds__(256) lu_replay_kernel(TopoDev T, uint32_t n_lanes, const double* a,
                                                         const double* rhs, double* tv_out, double* dx,
                                                         uint8_t* bad_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* lanes_smem = stage_programs(T, smem_raw);
  const uint32_t prog = saddr(smem_raw);
  const int tid = threadIdx.x & 31;
  const uint32_t warps = blockDim.x >> 5, w = threadIdx.x >> 5;
  double* v = lanes_smem + size_t(w) * (T.nv + T.n + 1);
  double* y = v + T.ntv;
  double* r = v + T.nv;
  for (uint32_t lane = blockIdx.x * warps + w; lane < n_lanes; lane += gridDim.x * warps) {
    init_consts(T, v, tid);
    for (uint32_t j = tid; j < T.n_fill; j += 32) v[T.fill[j]] = 0.0;
    const double* al = a + size_t(lane) * T.nnz;
    for (uint32_t p = tid; p < T.nnz; p += 32) v[T.amap[p]] = al[p];
    for (uint32_t i = tid; i < T.n; i += 32) r[i] = rhs[size_t(lane) * T.n + i];
    __syncwarp();
    load_y(T, r, y, tid);
    __syncwarp();
    const bool bad = refactor_forward(T, prog, v, tid);
    back_solve(T, prog, v, tid);
    for (uint32_t j = tid; j < T.n; j += 32) dx[size_t(lane) * T.n + T.qcol[j]] = y[j];
    if (tv_out)
      for (uint32_t s = tid; s < T.ntv; s += 32) tv_out[size_t(lane) * T.ntv + s] = v[s];
    if (tid == 0) bad_out[lane] = bad;
    __syncwarp();
  }
}

// The matrix of one lane at its start point, in pattern order: the lead
// lane's first Jacobian, which the host factors into the pivot tape
// (gpu_lanes.zig:361-372 factors lane 0 on the host the same way).
template <bool kHasB3>
__global__ void assemble_kernel(TopoDev T, LaneDev L, uint32_t lane, double* out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* smem = reinterpret_cast<double*>(smem_raw);
  const int tid = threadIdx.x & 31;
  if (threadIdx.x >= 32) return;
  LaneMem m = carve(T, smem);
  for (uint32_t i = tid; i < T.n; i += 32) m.x[i] = L.x[size_t(lane) * T.n + i];
  for (uint32_t i = tid; i < T.nlim; i += 32) m.lim[i] = L.lim[size_t(lane) * T.nlim + i];
  SimDev sim;
  sim.t = 0.0;
  sim.src_scale = 1.0;
  sim.kind = 0;
  __syncwarp();
  eval_all<kHasB3>(T, L.rec + size_t(lane) * T.rec_size, m, L.lim_active[lane] != 0, sim, tid);
  __syncwarp();
  gather_pattern(T, m, out, tid);
}

size_t lane_smem_bytes(const TopoDev& T) { return size_t(T.smem_doubles) * sizeof(double); }

// CTAs for a persistent launch: enough for every lane, at most as many as
// the device holds at once (SMs x resident CTAs at this shared memory).
template <class K>
static uint32_t persistent_grid(K kernel, uint32_t n_lanes, uint32_t lanes_per_block, size_t smem) {
  const uint32_t need = (n_lanes + lanes_per_block - 1) / lanes_per_block;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, int(32 * lanes_per_block), smem);
  const uint32_t cap = uint32_t(sms) * uint32_t(per_sm > 0 ? per_sm : 1);
  return need < cap ? need : cap;
}

// Every lane kernel comes in two instantiations: without BSIM3 (the
// register budget of the MOS1, diode and passive models) and with it (the
// BSIM3 dual-number chain raises the per-thread register need). The launch
// takes the second only for a topology that has a BSIM3 batch.
bool topo_has_b3(const TopoDev& T) {
  for (uint32_t b = 0; b < T.n_batches; ++b)
    if (T.b[b].type == kB3) return true;
  return false;
}

template <bool kHasB3>
static cudaError_t launch_dc_newton_t(const TopoDev& T, const LaneDev& L, const LaneOpts& o, uint32_t lanes_per_block,
                                      cudaStream_t s) {
  const size_t smem = T.prog_bytes + lanes_per_block * lane_smem_bytes(T);
  auto* k = o.ladder ? dc_newton_kernel<kHasB3, true> : dc_newton_kernel<kHasB3, false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  k<<<persistent_grid(k, L.n_lanes, lanes_per_block, smem), 32 * lanes_per_block, smem, s>>>(T, L, o);
  return cudaGetLastError();
}

cudaError_t launch_dc_newton(const TopoDev& T, const LaneDev& L, const LaneOpts& o, uint32_t lanes_per_block,
                             cudaStream_t s) {
  return topo_has_b3(T) ? launch_dc_newton_t<true>(T, L, o, lanes_per_block, s)
                        : launch_dc_newton_t<false>(T, L, o, lanes_per_block, s);
}

cudaError_t launch_assemble(const TopoDev& T, const LaneDev& L, uint32_t lane, double* out, cudaStream_t s) {
  // Before the tape exists (the lead lane's first Jacobian) a lane needs no
  // tape values: x, xo, rhs, diag, staging and the limited images (nv = 0).
  const size_t smem = size_t(4 * T.n + T.nv + T.n_stage + T.nlim + 2) * sizeof(double);
  auto* k = topo_has_b3(T) ? assemble_kernel<true> : assemble_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  k<<<1, 32, smem, s>>>(T, L, lane, out);
  return cudaGetLastError();
}

cudaError_t launch_lu_replay(const TopoDev& T, uint32_t n_lanes, const double* a, const double* rhs, double* tv,
                             double* dx, uint8_t* bad, uint32_t lanes_per_block, cudaStream_t s) {
  const size_t per = size_t(T.nv + T.n + 1) * sizeof(double);
  const size_t smem = T.prog_bytes + lanes_per_block * per;
  cudaError_t e = cudaFuncSetAttribute(lu_replay_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  lu_replay_kernel<<<persistent_grid(lu_replay_kernel, n_lanes, lanes_per_block, smem), 32 * lanes_per_block, smem,
                     s>>>(T, n_lanes, a, rhs, tv, dx, bad);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Lane-interleaved refactor + solve: one thread per lane. The lane values of a
// warp sit interleaved in shared memory (value i of the warp's lane t at
// [i * 32 + t]: every access of the warp is 32 consecutive words), A, rhs and
// dx are [entry][lane] planes in HBM (coalesced), and every thread walks the
// same sequential op list (the programs' ops in row order, padding left
// out), so control flow stays uniform. This is the reference's lane layout
// (lane_kernels.zig Bodies.refactor / solveNeg over [nnz][N] planes) with the
// working set staged on chip; the ops and their order per value are those of
// the warp programs, so the results are bitwise theirs.
// ---------------------------------------------------------------------------
namespace {

// cp.async of one 8-byte value from global into shared memory (in flight
// until cp_async_wait); lanes past the end copy nothing and leave the value.
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, bool live) {
  if (live) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__global__ void __launch_bounds__(256) lu_lanes_kernel(TopoDev T, const uint2* seq, uint32_t n_seq_a, uint32_t n_seq,
                                                       uint32_t n_lanes, const double* a, const double* rhs,
                                                       double* tv_out, double* dx, uint8_t* bad_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // per CTA: the op list, the index tables (amap, pinv, qcol, fill), the
  // L entries' scaled flags, then each warp's interleaved lane values
  uint2* ops = reinterpret_cast<uint2*>(smem_raw);
  uint32_t* s_amap = reinterpret_cast<uint32_t*>(ops + n_seq);
  uint32_t* s_pinv = s_amap + T.nnz;
  uint32_t* s_qcol = s_pinv + T.n;
  uint32_t* s_fill = s_qcol + T.n;
  unsigned char* lsc = reinterpret_cast<unsigned char*>(s_fill + T.n_fill);
  for (uint32_t i = threadIdx.x; i < n_seq; i += blockDim.x) ops[i] = seq[i];
  for (uint32_t i = threadIdx.x; i < T.nnz; i += blockDim.x) s_amap[i] = T.amap[i];
  for (uint32_t i = threadIdx.x; i < T.n; i += blockDim.x) {
    s_pinv[i] = T.pinv[i];
    s_qcol[i] = T.qcol[i];
  }
  for (uint32_t i = threadIdx.x; i < T.n_fill; i += blockDim.x) s_fill[i] = T.fill[i];
  for (uint32_t i = threadIdx.x; i < T.nl; i += blockDim.x) lsc[i] = T.l_scaled[i];
  __syncthreads();
  const size_t tables = size_t(n_seq) * 8 + size_t(T.nnz + 2 * T.n + T.n_fill) * 4 + T.nl;
  const uint32_t vbase_off = uint32_t((tables + 15) & ~size_t(15));
  const uint32_t t = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t nv = T.nv;
  const uint32_t vb = saddr(smem_raw + vbase_off) + w * nv * 256 + t * 8;  // value i at vb + i * 256
  const uint32_t ob = saddr(ops);
  const uint32_t lanes_per_grid = gridDim.x * blockDim.x;
  const uint32_t l0 = blockIdx.x * blockDim.x + threadIdx.x;
  // every thread of a warp runs the loop the same number of times (lanes
  // past the end compute on stale values and store nothing)
  const uint32_t rounds = (n_lanes + lanes_per_grid - 1) / lanes_per_grid;
  for (uint32_t rd = 0; rd < rounds; ++rd) {
    const uint32_t lane = l0 + rd * lanes_per_grid;
    const bool live = lane < n_lanes;
    // A and rhs straight into their tape positions, all copies in flight at once
    for (uint32_t p = 0; p < T.nnz; ++p) cp_async8(vb + 256 * s_amap[p], a + size_t(p) * n_lanes + lane, live);
    for (uint32_t r = 0; r < T.n; ++r)
      cp_async8(vb + 256 * (T.ntv + s_pinv[r]), rhs + size_t(r) * n_lanes + lane, live);
    sts(vb + 256 * (nv - 3), 0.0);
    sts(vb + 256 * (nv - 2), 1.0);
    sts(vb + 256 * (nv - 1), 0.0);
    for (uint32_t j = 0; j < T.n_fill; ++j) sts(vb + 256 * s_fill[j], 0.0);
    cp_async_wait();
    // y = P(-rhs)
    for (uint32_t r = 0; r < T.n; ++r) {
      const uint32_t py = vb + 256 * (T.ntv + s_pinv[r]);
      sts(py, -lds(py));
    }
    bool bad = false;
    auto run = [&](uint32_t k0, uint32_t k1) {
      if (k0 >= k1) return;
      uint2 op = lds_u2(ob + 8 * k0);
      for (uint32_t k = k0; k < k1; ++k) {
        const uint2 next = lds_u2(ob + 8 * (k + 1 < k1 ? k + 1 : k));  // the same word in every thread
        const uint32_t kind = op.x >> 28;
        const uint32_t pd = vb + 256 * (op.x & 0x0fffffffu);
        const uint32_t pa = vb + 256 * (op.y & 0xffffu), pb = vb + 256 * (op.y >> 16);
        const double av = lds(pa), bv = lds(pb);
        if (kind == kOpDivGrowth || kind == kOpDivScaled || kind == kOpDivY) {
          const double q = div_rn(bv, av);
          if (kind == kOpDivGrowth && !(fabs(av) >= __dmul_rn(kGrowth, fabs(bv)))) bad = true;
          if (kind == kOpDivScaled && !(fabs(q) < CUDART_INF)) bad = true;
          sts(pd, q);
        } else {
          const double d = lds(pd);
          if (kind == kOpFlop || bv != 0.0) sts(pd, __dsub_rn(d, __dmul_rn(av, bv)));
        }
        op = next;
      }
    };
    run(0, n_seq_a);
    // the refactor's peel tests (as refactor_forward)
    const uint32_t l0v = T.nu + T.n;
    for (uint32_t sv = 0; sv < T.nu; ++sv) {
      const double u = lds(vb + 256 * sv);
      if (dbits(u - u) != 0) bad = true;
    }
    for (uint32_t kk = 0; kk < T.n; ++kk) {
      const double dg = lds(vb + 256 * (T.nu + kk));
      if (dg == 0.0 || !(fabs(dg) < CUDART_INF)) bad = true;
    }
    for (uint32_t sv = 0; sv < T.nl; ++sv)
      if (!lsc[sv] && !(fabs(lds(vb + 256 * (l0v + sv))) <= kWide)) bad = true;
    run(n_seq_a, n_seq);
    if (live) {
      for (uint32_t j = 0; j < T.n; ++j) dx[size_t(s_qcol[j]) * n_lanes + lane] = lds(vb + 256 * (T.ntv + j));
      if (tv_out)
        for (uint32_t sv = 0; sv < T.ntv; ++sv) tv_out[size_t(sv) * n_lanes + lane] = lds(vb + 256 * sv);
      bad_out[lane] = bad;
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Mixed precision: the same lane-interleaved replay with the refactor and the
// triangular solves in FP32, then FP64 iterative refinement on the residual
// (res = -rhs - A dx with A and rhs re-read in FP64, the correction solved on
// the FP32 factors) until the residual is below 1e-12 of rhs, at most
// kRefineMax corrections.
// ---------------------------------------------------------------------------
namespace {

constexpr int kRefineMax = 6;
constexpr float kGrowthF = 1e-12f;
constexpr float kWideF = 1e3f;

__device__ __forceinline__ float ldsf(uint32_t a) {
  float r;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(r) : "r"(a));
  return r;
}
__device__ __forceinline__ void stsf(uint32_t a, float x) {
  asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(x) : "memory");
}

__global__ void __launch_bounds__(256) lu_lanes_mixed_kernel(TopoDev T, const uint2* seq, uint32_t n_seq_a,
                                                             uint32_t n_seq, uint32_t n_seq_f, uint32_t n_lanes,
                                                             const double* a, const double* rhs, double* dx_out,
                                                             uint8_t* bad_out, uint8_t* refine_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // per CTA: A, B and forward-only op lists, amap, pinv, qcol, fill, the
  // CSR of the pattern (row_ptr, slot, col), the scaled flags; then per warp
  // the interleaved FP32 tape values and the FP64 dx
  const uint32_t n_ops = n_seq + n_seq_f;
  uint2* ops = reinterpret_cast<uint2*>(smem_raw);
  uint32_t* s_amap = reinterpret_cast<uint32_t*>(ops + n_ops);
  uint32_t* s_pinv = s_amap + T.nnz;
  uint32_t* s_qcol = s_pinv + T.n;
  uint32_t* s_fill = s_qcol + T.n;
  uint32_t* s_rptr = s_fill + T.n_fill;
  uint32_t* s_rslot = s_rptr + T.n + 1;
  uint32_t* s_rcol = s_rslot + T.nnz;
  unsigned char* lsc = reinterpret_cast<unsigned char*>(s_rcol + T.nnz);
  for (uint32_t i = threadIdx.x; i < n_ops; i += blockDim.x) ops[i] = seq[i];
  for (uint32_t i = threadIdx.x; i < T.nnz; i += blockDim.x) {
    s_amap[i] = T.amap[i];
    s_rslot[i] = T.row_slot[i];
    s_rcol[i] = T.row_col[i];
  }
  for (uint32_t i = threadIdx.x; i < T.n; i += blockDim.x) {
    s_pinv[i] = T.pinv[i];
    s_qcol[i] = T.qcol[i];
  }
  for (uint32_t i = threadIdx.x; i <= T.n; i += blockDim.x) s_rptr[i] = T.row_ptr[i];
  for (uint32_t i = threadIdx.x; i < T.n_fill; i += blockDim.x) s_fill[i] = T.fill[i];
  for (uint32_t i = threadIdx.x; i < T.nl; i += blockDim.x) lsc[i] = T.l_scaled[i];
  __syncthreads();
  const size_t tables = size_t(n_ops) * 8 + size_t(3 * T.nnz + 3 * T.n + 1 + T.n_fill) * 4 + T.nl;
  const uint32_t base = uint32_t((tables + 15) & ~size_t(15));
  const uint32_t t = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t nv = T.nv;
  const uint32_t per_warp = (nv * 128 + T.n * 256 + 15) & ~15u;
  const uint32_t vb = saddr(smem_raw + base) + w * per_warp + t * 4;                 // float value i at vb + i * 128
  const uint32_t xb = saddr(smem_raw + base) + w * per_warp + nv * 128 + t * 8;      // FP64 dx_i at xb + i * 256
  const uint32_t ob = saddr(ops);
  const uint32_t lanes_per_grid = gridDim.x * blockDim.x;
  const uint32_t l0 = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t rounds = (n_lanes + lanes_per_grid - 1) / lanes_per_grid;
  for (uint32_t rd = 0; rd < rounds; ++rd) {
    const uint32_t lane = l0 + rd * lanes_per_grid;
    const bool live = lane < n_lanes;
    const size_t ls = live ? lane : 0;  // dead lanes read lane 0 and store nothing
    for (uint32_t p = 0; p < T.nnz; ++p) stsf(vb + 128 * s_amap[p], float(a[size_t(p) * n_lanes + ls]));
    for (uint32_t r = 0; r < T.n; ++r) stsf(vb + 128 * (T.ntv + s_pinv[r]), float(-rhs[size_t(r) * n_lanes + ls]));
    stsf(vb + 128 * (nv - 3), 0.0f);
    stsf(vb + 128 * (nv - 2), 1.0f);
    stsf(vb + 128 * (nv - 1), 0.0f);
    for (uint32_t j = 0; j < T.n_fill; ++j) stsf(vb + 128 * s_fill[j], 0.0f);
    bool bad = false;
    auto run = [&](uint32_t k0, uint32_t k1) {
      if (k0 >= k1) return;
      uint2 op = lds_u2(ob + 8 * k0);
      for (uint32_t k = k0; k < k1; ++k) {
        const uint2 next = lds_u2(ob + 8 * (k + 1 < k1 ? k + 1 : k));
        const uint32_t kind = op.x >> 28;
        const uint32_t pd = vb + 128 * (op.x & 0x0fffffffu);
        const uint32_t pa = vb + 128 * (op.y & 0xffffu), pb = vb + 128 * (op.y >> 16);
        const float av = ldsf(pa), bv = ldsf(pb);
        if (kind == kOpDivGrowth || kind == kOpDivScaled || kind == kOpDivY) {
          const float q = __fdiv_rn(bv, av);
          if (kind == kOpDivGrowth && !(fabsf(av) >= __fmul_rn(kGrowthF, fabsf(bv)))) bad = true;
          if (kind == kOpDivScaled && !(fabsf(q) < CUDART_INF_F)) bad = true;
          stsf(pd, q);
        } else {
          const float d = ldsf(pd);
          if (kind == kOpFlop || bv != 0.0f) stsf(pd, __fsub_rn(d, __fmul_rn(av, bv)));
        }
        op = next;
      }
    };
    run(0, n_seq_a);
    const uint32_t l0v = T.nu + T.n;
    for (uint32_t sv = 0; sv < T.nu; ++sv) {
      const float u = ldsf(vb + 128 * sv);
      if (!(fabsf(u) < CUDART_INF_F)) bad = true;
    }
    for (uint32_t kk = 0; kk < T.n; ++kk) {
      const float dg = ldsf(vb + 128 * (T.nu + kk));
      if (dg == 0.0f || !(fabsf(dg) < CUDART_INF_F)) bad = true;
    }
    for (uint32_t sv = 0; sv < T.nl; ++sv)
      if (!lsc[sv] && !(fabsf(ldsf(vb + 128 * (l0v + sv))) <= kWideF)) bad = true;
    run(n_seq_a, n_seq);
    for (uint32_t j = 0; j < T.n; ++j) sts(xb + 256 * s_qcol[j], double(ldsf(vb + 128 * (T.ntv + j))));
    // refinement: res = -rhs - A dx in FP64, corrections on the FP32 factors
    uint32_t refined = 0;
    for (int it = 0; it <= kRefineMax; ++it) {
      double rmax = 0.0, bmax = 0.0;
      for (uint32_t i = 0; i < T.n; ++i) {
        const double b = rhs[size_t(i) * n_lanes + ls];
        double res = -b;
        for (uint32_t e = s_rptr[i]; e < s_rptr[i + 1]; ++e)
          res = res - a[size_t(s_rslot[e]) * n_lanes + ls] * lds(xb + 256 * s_rcol[e]);
        rmax = fmax(rmax, fabs(res));
        bmax = fmax(bmax, fabs(b));
        stsf(vb + 128 * (T.ntv + s_pinv[i]), float(res));
      }
      if (!(rmax > 1e-12 * bmax) || it == kRefineMax) break;
      run(n_seq, n_seq + n_seq_f);  // forward through L
      run(n_seq_a, n_seq);          // back through U
      for (uint32_t j = 0; j < T.n; ++j) {
        const uint32_t px = xb + 256 * s_qcol[j];
        sts(px, lds(px) + double(ldsf(vb + 128 * (T.ntv + j))));
      }
      ++refined;
    }
    if (live) {
      for (uint32_t i = 0; i < T.n; ++i) dx_out[size_t(i) * n_lanes + lane] = lds(xb + 256 * i);
      bad_out[lane] = bad;
      if (refine_out) refine_out[lane] = uint8_t(refined);
    }
  }
}

}  // namespace

uint32_t lu_lanes_mixed_smem(const TopoDev& T, uint32_t n_ops, uint32_t warps) {
  const size_t tables = size_t(n_ops) * 8 + size_t(3 * T.nnz + 3 * T.n + 1 + T.n_fill) * 4 + T.nl;
  const uint32_t per_warp = (T.nv * 128 + T.n * 256 + 15) & ~15u;
  return uint32_t(((tables + 15) & ~size_t(15)) + size_t(warps) * per_warp);
}

cudaError_t launch_lu_lanes_mixed(const TopoDev& T, const uint2* seq, uint32_t n_seq_a, uint32_t n_seq,
                                  uint32_t n_seq_f, uint32_t n_lanes, const double* a, const double* rhs, double* dx,
                                  uint8_t* bad, uint8_t* refine, uint32_t warps, cudaStream_t s) {
  const size_t smem = lu_lanes_mixed_smem(T, n_seq + n_seq_f, warps);
  cudaError_t e = cudaFuncSetAttribute(lu_lanes_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lu_lanes_mixed_kernel, int(32 * warps), smem);
  const uint32_t per_cta = 32 * warps;
  const uint32_t need = (n_lanes + per_cta - 1) / per_cta;
  const uint32_t cap = uint32_t(sms) * uint32_t(per_sm > 0 ? per_sm : 1);
  lu_lanes_mixed_kernel<<<need < cap ? need : cap, per_cta, smem, s>>>(T, seq, n_seq_a, n_seq, n_seq_f, n_lanes, a,
                                                                       rhs, dx, bad, refine);
  return cudaGetLastError();
}

uint32_t lu_lanes_smem(const TopoDev& T, uint32_t n_seq, uint32_t warps) {
  const size_t tables = size_t(n_seq) * 8 + size_t(T.nnz + 2 * T.n + T.n_fill) * 4 + T.nl;
  return uint32_t(((tables + 15) & ~size_t(15)) + size_t(warps) * T.nv * 256);
}

cudaError_t launch_lu_lanes(const TopoDev& T, const uint2* seq, uint32_t n_seq_a, uint32_t n_seq, uint32_t n_lanes,
                            const double* a, const double* rhs, double* tv, double* dx, uint8_t* bad,
                            uint32_t warps, cudaStream_t s) {
  const size_t smem = lu_lanes_smem(T, n_seq, warps);
  cudaError_t e = cudaFuncSetAttribute(lu_lanes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lu_lanes_kernel, int(32 * warps), smem);
  const uint32_t per_cta = 32 * warps;
  const uint32_t need = (n_lanes + per_cta - 1) / per_cta;
  const uint32_t cap = uint32_t(sms) * uint32_t(per_sm > 0 ? per_sm : 1);
  lu_lanes_kernel<<<need < cap ? need : cap, per_cta, smem, s>>>(T, seq, n_seq_a, n_seq, n_lanes, a, rhs, tv, dx,
                                                                 bad);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fixed lane scratch for the allocation-free DC entry point
// (esl_dc_solve_device_static). The per-lane Newton state and the paused-lane
// hand-off buffers the fused kernel keeps in HBM live in one file-scope device
// array instead of context-owned allocations. The array is created with the
// module (zero-filled by the loader) and is reached through its symbol
// address, looked up once per device.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_lane_scratch[kStaticScratchBytes];

cudaError_t static_scratch(void** ptr) {
  constexpr int kMaxDevices = 64;
  static void* addr[kMaxDevices] = {};
  static std::mutex mu;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_lane_scratch);
    if (e != cudaSuccess) return e;
    addr[dev] = p;
  }
  *ptr = addr[dev];
  return cudaSuccess;
}

// Start state of every lane (the host-side set-up of esl_dc_solve_device done
// on the device): iteration 0, running, limit 1e9, INITFIX from the options;
// a cold lane starts at x = 0 with its junction images at the seeds the
// records carry (diode vcrit; MOSFET vgs, vds = 0, vbs = -1) and limiting live, a warm lane at its x with
// limiting off. The first thread also clears the paused-lane counter.
__global__ void lane_init_kernel(TopoDev T, LaneDev L, uint32_t cold, uint32_t init_fix) {
  const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
  if (lane == 0) *L.n_paused = 0;
  if (lane >= L.n_lanes) return;
  L.status[lane] = kRunning;
  L.iters[lane] = 0;
  L.flags[lane] = init_fix ? 1u : 0u;
  L.lim_active[lane] = cold && T.nlim ? 1u : 0u;
  L.limit[lane] = 1e9;
  double* lim = L.lim + size_t(lane) * T.nlim;
  for (uint32_t i = 0; i < T.nlim; ++i) lim[i] = 0.0;
  if (L.ladder) {
    LadderDev z{};
    z.rung = kRungPlain;
    L.ladder[lane] = z;
  }
  if (!cold) return;
  for (uint32_t i = 0; i < T.n; ++i) L.x[size_t(lane) * T.n + i] = 0.0;
  cold_images(T, L.rec + size_t(lane) * T.rec_size, lim, 0, 1);
}

cudaError_t launch_lane_init(const TopoDev& T, const LaneDev& L, bool cold, bool init_fix, cudaStream_t s) {
  const uint32_t threads = 128, blocks = (L.n_lanes + threads - 1) / threads;
  lane_init_kernel<<<blocks > 0 ? blocks : 1, threads, 0, s>>>(T, L, cold ? 1u : 0u, init_fix ? 1u : 0u);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Transient lanes (src/analysis/tran/tran.zig Sim.begin / Sim.end with the
// integrator.zig kernels): one warp runs one lane's whole transient, its
// operating point included, without returning to the host between steps.
// ---------------------------------------------------------------------------
namespace {


// One companion step's terms (integrator.zig Hook): rhs += ag0 * (q - q1)
// (- ag1 * ip for trap), matrix G + ag0 * C.
struct Companion {
  double ag0, ag1;
  bool trap;
  const double* q1;  // n: accepted row charges
  const double* ip;  // n: accepted dynamic currents
};

// Row charge sums and capacitance slot sums from the staging cells, in
// stamp order (the companion gather program in shared memory); the
// companion folded into rhs, y and the tape values. Rows and slots without
// charge or capacitance cells have exactly zero terms and are not visited.
__device__ void companion(const TopoDev& T, uint32_t prog, const LaneMem& m, const Companion& c, int tid) {
  const uint32_t lb = saddr(m.base);
  const uint32_t depth = prog + T.o_k_depth, koff = prog + T.o_k_off;
  const uint32_t ksrc = prog + T.o_k_src, kdst = prog + T.o_k_dst;
  const uint32_t ng = T.n_kr_groups + T.n_ks_groups;
  for (uint32_t g = 0; g < ng; ++g) {
    const double s = gather_sum(ksrc + 4 * (lds_u32(koff + 4 * g) + tid), lds_u32(depth + 4 * g), lb);
    const uint2 d = lds_u2(kdst + 8 * (g * 32 + tid));
    if (g < T.n_kr_groups) {
      if (d.x != kNoDiag) {
        const double dq = c.ag0 * (s - c.q1[d.x]);
        const double base = m.rhs[d.x] + dq;
        const double r = c.trap ? base - c.ag1 * c.ip[d.x] : base;
        m.rhs[d.x] = r;
        sts(lb + 8 * d.y, -r);
      }
    } else {
      const double v = lds(lb + 8 * d.x) + c.ag0 * s;
      sts(lb + 8 * d.x, v);
      sts(lb + 8 * d.y, v);
    }
  }
}

// Row charges of the last evaluation (the q plane) for the rows with charge
// cells, from the companion program's row part; the other rows' charges are
// zero in every slot of the ring from the start and stay so.
__device__ __forceinline__ void row_charges(const TopoDev& T, uint32_t prog, const LaneMem& m, double* q, int tid) {
  const uint32_t lb = saddr(m.base);
  const uint32_t depth = prog + T.o_k_depth, koff = prog + T.o_k_off;
  const uint32_t ksrc = prog + T.o_k_src, kdst = prog + T.o_k_dst;
  for (uint32_t g = 0; g < T.n_kr_groups; ++g) {
    const double s = gather_sum(ksrc + 4 * (lds_u32(koff + 4 * g) + tid), lds_u32(depth + 4 * g), lb);
    const uint32_t row = lds_u32(kdst + 8 * (g * 32 + tid));
    if (row != kNoDiag) q[row] = s;
  }
}

// The LTE charge states at x (capacitor charges, diode junction charges,
// MOS1 overlap gate charges).

// The V and I sources' values at `sim` (they depend on the time point and
// the source scale alone), once for all the Newton iterations there.

// Newton on one lane (converger.newton at W = 1 on the frozen tape), for
// the transient's operating point (no companion) and its steps, and for the
// points of a sequential sweep. `vcache` holds the sources' values
// (fill_sources). Returns 0 converged (x holds the published iterate), 1
// out of iterations, 2 the factor left the tape.
template <bool kHasB3>
__device__ int lane_newton(const TopoDev& T, uint32_t prog, const LaneMem& m, const double* rec, const LaneOpts& o,
                           const SimDev& sim, const Companion* cp, bool& lim_active, bool init_fix,
                           uint32_t& iters, const double* vcache, int tid, NewtonCarry* carry = nullptr) {
  const uint32_t n = T.n;
  const uint32_t max_iter = o.max_iter < 100 ? 100 : o.max_iter;
  double limit = kXPlausible;
  uint32_t iter0 = 0;
  bool have_step = false;
  if (carry && carry->resume) {
    // resumed after a host factor: the step for iteration `iter` is the host's
    iter0 = carry->iter;
    limit = carry->limit;
    init_fix = carry->init_fix != 0;
    if (carry->resume == 2) {
      iters = iter0 + 1;
      return 2;
    }
    have_step = true;
  }
  for (uint32_t iter = iter0; iter < max_iter; ++iter) {
   if (!have_step) {
    eval_all<kHasB3>(T, rec, m, lim_active, sim, tid, false, vcache);
    __syncwarp();
    assemble(T, prog, m, tid);
    __syncwarp();
    if (cp) {
      companion(T, prog, m, *cp, tid);
      __syncwarp();
    }
    if (o.gmin > 0) {
      // loadExtras (converger.zig:321-330): diagonal gmin and its residual form
      for (uint32_t p = tid; p < T.nnz; p += 32) {
        const uint32_t row = T.slot_row[p];
        if (row != kNoDiag) {
          const double d = m.diag[row] + o.gmin;
          m.diag[row] = d;
          m.v[T.amap[p]] = d;
        }
      }
      for (uint32_t i = tid; i < n; i += 32) m.rhs[i] += o.gmin * m.x[i];
      __syncwarp();
      load_y(T, m.rhs, m.y, tid);
      __syncwarp();
    }
    if (o.gstamp > 0.0) {
      // loadGmin at the gmin-stepping stamps (converger.zig:696-713)
      for (uint32_t k = tid; k < T.n_gst; k += 32) {
        const uint32_t slot = T.gst[3 * k], row = T.gst[3 * k + 1], col = T.gst[3 * k + 2];
        const uint32_t at = T.amap[slot], dr = T.slot_row[slot];
        const double d = m.v[at] + o.gstamp;
        m.v[at] = d;
        if (dr != kNoDiag) m.diag[dr] = d;
        m.rhs[row] += o.gstamp * m.x[col];
      }
      __syncwarp();
      load_y(T, m.rhs, m.y, tid);
      __syncwarp();
    }
    if (iter == 0) {
      double g = 1.0;
      uint64_t xm = 0, fm = 0;
      for (uint32_t i = tid; i < n; i += 32) {
        g = fmax(g, fabs(m.diag[i]));
        const uint64_t bx = dbits(fabs(m.x[i])), bf = dbits(fabs(m.rhs[i]));
        xm = bx > xm ? bx : xm;
        fm = bf > fm ? bf : fm;
      }
      g = warp_fmax(g);
      xm = warp_max_u64(xm);
      fm = warp_max_u64(fm);
      const double scale = fmin(fmax(from_bits(xm), from_bits(fm) * g), 1e18);
      limit = !(1e3 * scale > kXPlausible) ? kXPlausible : 1e3 * scale;
    }
    const bool bad = (carry && carry->host_mode) || refactor_forward(T, prog, m.v, tid);
    if (bad) {
      if (carry) {
        // pause: the caller hands the lane to the host at this iteration
        carry->iter = iter;
        carry->limit = limit;
        carry->init_fix = init_fix;
        return 3;
      }
      iters = iter + 1;
      return 2;
    }
    back_solve(T, prog, m.v, tid);
   }
    have_step = false;
    __syncwarp();
    uint64_t worst = 0;
    for (uint32_t j = tid; j < n; j += 32) {
      const uint32_t i = T.qcol[j];
      const double d = m.y[j];
      const double xold = m.x[i];
      const double xn = xold + d;
      m.xo[i] = xold;
      m.x[i] = xn;
      const double tol = o.reltol * fmax(fabs(xn), fabs(xold)) + (T.cur_row[i] ? o.abstol : o.vntol);
      const bool finite = fabs(xn) < CUDART_INF && fabs(d) < CUDART_INF;
      const double qv = div_rn(fabs(d), tol);
      const double score = !finite ? CUDART_INF : (qv == qv ? qv : 0.0);
      const uint64_t b = dbits(score);
      worst = b > worst ? b : worst;
    }
    worst = warp_max_u64(worst);
    __syncwarp();
    const bool limited = apply_limits<kHasB3>(T, rec, m, lim_active, tid);
    if (T.nlim) lim_active = true;
    bool ok = !limited && iter != 0 && !(from_bits(worst) >= 1.0);
    if (ok) {
      bool p = true;
      for (uint32_t i = tid; i < n; i += 32) p &= fabs(m.x[i]) <= limit;
      ok = __all_sync(kFull, p);
    }
    if (ok) {
      bool p = true;
      for (uint32_t i = tid; i < n; i += 32) p &= fabs(m.rhs[i]) <= residual_gate(o, m.diag[i], m.x[i]);
      ok = __all_sync(kFull, p);
    }
    if (ok) {
      if (init_fix) {
        init_fix = false;
      } else {
        for (uint32_t i = tid; i < n; i += 32) m.x[i] = m.xo[i];
        __syncwarp();
        iters = iter + 1;
        return 0;
      }
    }
    __syncwarp();
  }
  iters = max_iter;
  return 1;
}

// CKTterr's bound over the LTE states (integrator.zig minDel at w = 1, then
// the order-2 root): `method` 1 BE / 2 trap probed after a step integrated
// with `cur`; q0..q3 the ring slots; NaN when a read entry is not finite.


// The first PULSE corner at or after `after` over every V source with a
// PULSE wave (models/vsource.va:133-136: four periodic timers per source).
// The PULSE corner timers (vsource.va:133-136, the 4 periodic timers of
// each V source with a PULSE wave) into `tm`: timer k at tm[2 k] (start)
// and tm[2 k + 1] (period); 4 per V source, start +inf where the source has
// no PULSE wave. Each lane computes its table once.

// The first timer event at or after `after` (tran.zig nextBp), the timers
// spread over the warp and the earliest taken by a warp minimum: the PULSE
// corners from the lane's timer table, and each PWL source's one-shot
// corners (its table times plus TD, and TD itself when the table leaves
// slots unused, vsource.va:137-200) found in its record.

// Streamed measures (src/output/measure.zig, after ngspice com_measure2.c):
// Cross counts RISE/FALL/CROSS events from a clause's second sample and
// interpolates the level crossing on the last segment (:1269-1365); At
// takes the first segment holding AT (:1379-1398). Thread c runs card c.
__device__ void meas_start(const MeasDev& mc, CrossDev* x) {
  for (int k = 0; k < 2; ++k) {
    const MeasClauseDev& c = k ? mc.b : mc.a;
    CrossDev& s = x[k];
    s.td = c.td;
    s.prev = s.prev_x = 0.0;
    s.last = s.hit = CUDART_NAN;
    s.want_rise = c.rise;
    s.want_fall = c.fall;
    s.want_cross = c.cross;
    s.rise = s.fall = s.cross = 0;
    s.first = 0;
    s.above = s.pending = s.found = s.over = 0;
    if (mc.kind >= kMeasMin) {
      s.hit = 0.0;  // Extremum's m
      s.td = 0.0;   // its span
    }
  }
  if (mc.kind == kMeasInteg || mc.kind == kMeasRms) {
    IntegDev& g = *reinterpret_cast<IntegDev*>(x);
    for (int j = 0; j < 4; ++j) g.p[j][0] = g.p[j][1] = 0.0;
    g.sum[0] = g.sum[1] = g.sum[2] = 0.0;
    g.px = g.py = 0.0;
    g.first_x = g.cut_x = CUDART_NAN;
    g.rows = g.np = g.count = g.inside = g.cut = g.over = 0;
  }
}

// Extremum.feed (measure.zig:1401-1449, not DC): op 0 MIN, 1 MAX (the last
// sample reaching the extreme), 2 AVG (trapezoids over the samples' span;
// hit the sum, td the span); inside FROM..TO, no interpolated ends; true
// once past TO.
__device__ bool ext_feed(CrossDev& s, const MeasClauseDev& c, int op, double xv, double v) {
  if (s.over) return true;
  if (xv < c.from) return false;
  if (c.to != 0.0 && xv > c.to) {
    s.over = 1;
    return true;
  }
  if (!s.first) {
    s.first = 1;
    s.hit = op == 2 ? 0.0 : v;
    s.prev = v;
    s.prev_x = xv;
    return false;
  }
  if (op == 0) {
    if (v <= s.hit) s.hit = v;
  } else if (op == 1) {
    if (v >= s.hit) s.hit = v;
  } else {
    s.hit = s.hit + 0.5 * (v + s.prev) * (xv - s.prev_x);
    s.td = s.td + (xv - s.prev_x);
    s.prev = v;
    s.prev_x = xv;
  }
  return false;
}

// Cross.feed for one event; true once the scan is over (its event found,
// or past TO).
__device__ bool cross_feed(CrossDev& s, const MeasClauseDev& c, double xv, double v) {
  if (s.over) return true;
  if (xv < s.td) return false;
  if (xv < c.from) return false;
  if (c.to != 0.0 && xv > c.to) {
    s.over = 1;
    return true;
  }
  const double level = c.val, prev_level = c.val;
  if (s.first == 1) {
    s.cross = 0;
    s.above = !(v < level);
    if (!s.above && s.prev >= prev_level) {
      s.fall = 1;
      s.cross = 1;
    } else if (s.above && s.prev < prev_level) {
      s.rise = 1;
      s.cross = 1;
    }
  }
  if (s.first > 1) {
    if (!s.above && v >= level) {
      s.above = 1;
      s.cross += 1;
      s.rise += 1;
      if (c.fall != kMeasLast) s.pending = 1;
    } else if (s.above && v <= level) {
      s.above = 0;
      s.cross += 1;
      s.fall += 1;
      if (c.rise != kMeasLast) s.pending = 1;
    }
    const double hit = s.prev_x + div_rn((prev_level - s.prev) * (xv - s.prev_x), ((v - s.prev) - level) + prev_level);
    if (s.cross == s.want_cross || s.rise == s.want_rise || s.fall == s.want_fall) {
      s.hit = hit;
      s.found = 1;
      s.over = 1;
      return true;
    }
    if (s.pending) {
      if (c.cross == kMeasUnset && c.rise == kMeasUnset && c.fall == kMeasUnset) {
        s.hit = hit;
        s.found = 1;
        s.over = 1;
        return true;
      }
      if (c.cross == kMeasLast || c.rise == kMeasLast || c.fall == kMeasLast) s.last = hit;
      s.pending = 0;
    }
  }
  s.first += 1;
  s.prev = v;
  s.prev_x = xv;
  return false;
}

__device__ bool at_feed(CrossDev& s, const MeasClauseDev& c, double xv, double v) {
  if (s.over) return true;
  if (s.first > 0 && s.prev_x <= c.at && xv >= c.at) {
    s.hit = s.prev + div_rn((c.at - s.prev_x) * (v - s.prev), xv - s.prev_x);
    s.found = 1;
    s.over = 1;
    return true;
  }
  s.first += 1;
  s.prev_x = xv;
  s.prev = v;
  return false;
}

// At.feed with slope (DERIV .. AT=): the slope of the first segment
// holding AT.
__device__ bool slope_feed(CrossDev& s, const MeasClauseDev& c, double xv, double v) {
  if (s.over) return true;
  if (s.first > 0 && s.prev_x <= c.at && xv >= c.at) {
    s.hit = div_rn(v - s.prev, xv - s.prev_x);
    s.found = 1;
    s.over = 1;
    return true;
  }
  s.first += 1;
  s.prev_x = xv;
  s.prev = v;
  return false;
}

// almostEqualUlps (measure.zig:1699-1708): within 100 units in the last
// place, on the doubles' order-preserving integer images.
__device__ __forceinline__ bool almost_equal_ulps(double a, double b) {
  if (a == b) return true;
  long long ia = __double_as_longlong(a), ib = __double_as_longlong(b);
  if (ia < 0) ia = (long long)(0x8000000000000000ull - (unsigned long long)ia);
  if (ib < 0) ib = (long long)(0x8000000000000000ull - (unsigned long long)ib);
  const unsigned long long d = (unsigned long long)ia - (unsigned long long)ib;
  const unsigned long long mag = (long long)d < 0 ? 0ull - d : d;
  return mag <= 100ull;
}

// measure.zig line (:1257-1261).
__device__ __forceinline__ double line_at(double x0, double y0, double x1, double y1, double at) {
  const double slope = div_rn(y1 - y0, x1 - x0);
  const double intercept = y0 - slope * x0;
  return slope * at + intercept;
}

// Integ.panel (measure.zig:1568-1586): folds the oldest points into one
// panel by Simpson's 3/8 rule, Simpson's rule or the trapezoid, as the next
// spacings agree; `avail` of p are points, the rest read zero.
__device__ void integ_panel(IntegDev& s, uint32_t avail) {
  double p[4][2];
  for (uint32_t j = 0; j < 4; ++j) {
    p[j][0] = j < avail ? s.p[j][0] : 0.0;
    p[j][1] = j < avail ? s.p[j][1] : 0.0;
  }
  double w[3];
  for (uint32_t j = 0; j < 3; ++j) w[j] = j + 1 < avail ? p[j + 1][0] - p[j][0] : 0.0;
  uint32_t used;
  if (almost_equal_ulps(w[0], w[1]) && almost_equal_ulps(w[0], w[2])) {
    s.sum[0] = s.sum[0] + div_rn(3.0 * w[0] * (p[0][1] + 3.0 * (p[1][1] + p[2][1]) + p[3][1]), 8.0);
    used = 3;
  } else if (almost_equal_ulps(w[0], w[1])) {
    s.sum[1] = s.sum[1] + div_rn(w[0] * (p[0][1] + 4.0 * p[1][1] + p[2][1]), 3.0);
    used = 2;
  } else {
    s.sum[2] = s.sum[2] + div_rn(w[0] * (p[0][1] + p[1][1]), 2.0);
    used = 1;
  }
  s.np = avail > used ? avail - used : 0u;
  for (uint32_t j = 0; j < s.np; ++j) {
    s.p[j][0] = p[avail - s.np + j][0];
    s.p[j][1] = p[avail - s.np + j][1];
  }
}

// Integ.feed (measure.zig:1538-1563): the window's points from the first
// sample at or past FROM (read as the value at a nonzero FROM) to the first
// past a nonzero TO (read as the value at TO); true once past TO.
__device__ bool integ_feed(IntegDev& s, const MeasClauseDev& c, bool rms, double xv, double v) {
  if (s.over) return true;
  bool ret = false;
  if (s.inside || !(xv < c.from)) {
    s.inside = 1;
    s.cut = c.to != 0.0 && xv > c.to;
    double p0 = xv, p1 = v;
    if (s.cut) {
      if (s.rows > 0 && !almost_equal_ulps(xv, c.to)) {
        p0 = c.to;
        p1 = line_at(s.px, s.py, xv, v, c.to);
      }
    } else if (s.count == 0 && c.from != 0.0 && s.rows > 0 && !almost_equal_ulps(xv, c.from)) {
      p0 = c.from;
      p1 = line_at(s.px, s.py, xv, v, c.from);
    }
    if (rms) p1 = p1 * p1;
    if (s.count == 0) s.first_x = p0;
    if (s.cut) s.cut_x = p0;
    s.count += 1;
    s.p[s.np][0] = p0;
    s.p[s.np][1] = p1;
    s.np += 1;
    if (s.np == 4) integ_panel(s, s.np);
    ret = s.cut != 0;
    if (ret) s.over = 1;
  }
  s.rows += 1;
  s.px = xv;
  s.py = v;
  return ret;
}

// Integ.result (measure.zig:1588-1595): the integral, or the RMS over the
// window's span.
__device__ double integ_result(IntegDev s, bool rms) {
  if (s.rows == 0) return CUDART_NAN;
  while (s.np > 1) integ_panel(s, s.np);
  const double from = s.count > (s.cut ? 1u : 0u) ? s.first_x : CUDART_NAN;
  const double to = s.cut ? s.cut_x : s.px;
  const double total = s.sum[0] + s.sum[1] + s.sum[2];
  return rms ? sqrt(div_rn(total, to - from)) : total;
}

// Feeds the row (t, x) to card c; true once the card has resolved.
__device__ bool meas_feed(const MeasDev& mc, CrossDev* x, double t, const double* xs) {
  if (mc.kind == kMeasFindAt) return at_feed(x[0], mc.a, t, xs[mc.a.unknown]);
  if (mc.kind == kMeasDeriv) return slope_feed(x[0], mc.a, t, xs[mc.a.unknown]);
  if (mc.kind == kMeasInteg || mc.kind == kMeasRms)
    return integ_feed(*reinterpret_cast<IntegDev*>(x), mc.a, mc.kind == kMeasRms, t, xs[mc.a.unknown]);
  if (mc.kind == kMeasMin || mc.kind == kMeasMax || mc.kind == kMeasAvg)
    return ext_feed(x[0], mc.a, int(mc.kind - kMeasMin), t, xs[mc.a.unknown]);
  if (mc.kind == kMeasPp) {
    const bool d0 = ext_feed(x[0], mc.a, 0, t, xs[mc.a.unknown]);
    const bool d1 = ext_feed(x[1], mc.a, 1, t, xs[mc.a.unknown]);
    return d0 && d1;
  }
  if (mc.kind == kMeasWhen) return cross_feed(x[0], mc.a, t, xs[mc.a.unknown]);
  const bool da = cross_feed(x[0], mc.a, t, xs[mc.a.unknown]);
  const bool db = cross_feed(x[1], mc.b, t, xs[mc.b.unknown]);
  return da && db;
}

// A card's value at the end: WHEN the event time (else a LAST count's last
// event, else NaN), TRIG/TARG targ - trig, FIND the interpolated value,
// MIN/MAX the extreme, AVG the trapezoidal mean, PP max - min.
__device__ double meas_value(const MeasDev& mc, const CrossDev* x) {
  double v;
  if (mc.kind == kMeasFindAt || mc.kind == kMeasDeriv) {
    v = x[0].found ? x[0].hit : CUDART_NAN;
  } else if (mc.kind == kMeasInteg || mc.kind == kMeasRms) {
    v = integ_result(*reinterpret_cast<const IntegDev*>(x), mc.kind == kMeasRms);
  } else if (mc.kind == kMeasMin || mc.kind == kMeasMax) {
    v = x[0].hit;  // 0 when no sample fell in the window
  } else if (mc.kind == kMeasAvg) {
    v = div_rn(x[0].hit, x[0].first ? x[0].td : 1.0);
  } else if (mc.kind == kMeasPp) {
    v = x[1].hit - x[0].hit;
  } else if (mc.kind == kMeasWhen) {
    v = x[0].found ? x[0].hit : x[0].last;
  } else {
    const double trig = x[0].found ? x[0].hit : x[0].last, targ = x[1].found ? x[1].hit : x[1].last;
    v = isfinite(trig) && isfinite(targ) ? targ - trig : CUDART_NAN;
  }
  return isfinite(v) ? v : CUDART_NAN;
}

}  // namespace

// A paused transient lane's matrix for the host factor: every pattern slot's
// G from the staging cells, plus ag0 C on the slots with capacitance cells
// (the same sums in the same order as the assembly and the companion
// gather, so the same bits as the lane's own assembled matrix).
__device__ void gather_pattern_tran(const TopoDev& T, const LaneMem& m, double ag0, bool dynamic, double* out,
                                    int tid) {
  for (uint32_t p = tid; p < T.nnz; p += 32) {
    double g = 0.0;
    for (uint32_t e = T.a_ptr[p]; e < T.a_ptr[p + 1]; ++e) {
      const uint32_t src = T.a_src[e];
      g = __dadd_rn(g, src == kSrcOne ? 1.0 : src == kSrcX0 ? m.x[0] : m.st[src]);
    }
    if (dynamic && T.c_ptr[p + 1] != T.c_ptr[p]) {
      double c = 0.0;
      for (uint32_t e = T.c_ptr[p]; e < T.c_ptr[p + 1]; ++e) c = __dadd_rn(c, m.st[T.c_src[e]]);
      g = __dadd_rn(g, __dmul_rn(ag0, c));
    }
    out[p] = g;
  }
}

template <bool kHasB3>
__device__ void tran_lane(const TopoDev& T, const LaneDev& L, const TranDev& P, const LaneOpts& o, uint32_t prog,
                          double* block, uint32_t lane, int tid) {
  const uint32_t lstat = L.status[lane];
  const bool resuming = L.resume && (lstat == kNeedSolve || lstat == kSingular);
  if (!(lstat == kRunning || resuming)) return;
  const uint32_t n = T.n, nq = T.n_qt;
  LaneMem m = carve(T, block);
  double* cur = block + T.smem_doubles;
  double* prev = cur + n;
  double* qh = prev + n;   // 4 slots of n: the row-charge ring
  double* ipr = qh + 4 * n;
  double* qt = ipr + n;    // 4 slots of nq: the LTE-state ring
  double* ipt = qt + 4 * nq;
  double* vsrc = ipt + nq;  // T.n_src: the V and I sources at the current time point
  double* tmr = vsrc + T.n_src;  // 8 T.n_src: the PULSE corner timers
  // past the lane's tran_doubles: kMeasDoubles per measure card
  CrossDev* mstate = reinterpret_cast<CrossDev*>(block + T.tran_doubles) + 2 * tid;
  const bool card = P.meas && uint32_t(tid) < P.n_meas;
  const uint32_t bd = T.tran_doubles + kMeasDoubles * P.n_meas;  // the lane's shared-memory doubles
  uint32_t* ts = P.tstate + size_t(lane) * kTranStateN;
  double* sv = P.tsave + size_t(lane) * (size_t(bd) + kTranSaveRegs);
  const double* rec = L.rec + size_t(lane) * T.rec_size;
  const size_t at = size_t(lane) * n;
  uint32_t stat[kTsN];
  for (int k = 0; k < kTsN; ++k) stat[k] = 0;

  // The run's state outside shared memory (saved with it on a pause).
  const double dt_max = P.dt_max;
  const double delmin = 1e-11 * dt_max;
  const double min_break = 10.0 * delmin;
  double dt = 0.0, t = 0.0, bp_next = 0.0, bp_save_dt = div_rn(P.t_stop, 50.0);
  double dt_old[6];
  for (int k = 0; k < 6; ++k) dt_old[k] = dt_max;
  int order = 1;
  uint32_t steps = 0, hb = 0, n_rec = 0;
  bool have_bp = false, bp_clamped = false, lim_active = false;
  NewtonCarry carry{0u, kXPlausible, 0u, 0u, (L.flags[lane] & 2u) ? 1u : 0u};
  uint32_t phase0 = 0;  // 0 a fresh lane, 1 resumed in the operating point, 2 in a step

  SimDev sim;
  sim.t = 0.0;
  sim.src_scale = 1.0;
  sim.kind = 2;
  if (resuming) {
    for (uint32_t i = tid; i < bd; i += 32) block[i] = sv[i];
    phase0 = ts[kTrPhase];
    carry.iter = ts[kTrIter];
    carry.init_fix = ts[kTrInitFix];
    carry.limit = L.limit[lane];
    carry.resume = lstat == kSingular ? 2u : 1u;
    order = int(ts[kTrOrder]);
    steps = ts[kTrSteps];
    have_bp = ts[kTrHaveBp] != 0;
    bp_clamped = ts[kTrBpClamped] != 0;
    hb = ts[kTrHb];
    n_rec = ts[kTrNRec];
    lim_active = ts[kTrLimActive] != 0;
    for (int k = 0; k < kTsN; ++k) stat[k] = ts[kTrStat + k];
    const double* r = sv + bd;
    t = r[0];
    dt = r[1];
    bp_next = r[2];
    bp_save_dt = r[3];
    for (int k = 0; k < 6; ++k) dt_old[k] = r[4 + k];
    __syncwarp();
    // the host's step for the iteration the lane paused in
    if (carry.resume == 1)
      for (uint32_t j = tid; j < n; j += 32) m.y[j] = L.dx[at + T.qcol[j]];
  } else {
    if (card) meas_start(P.meas[tid], mstate);
    init_consts(T, m.v, tid);
  }
  // Pause: the host factors this lane's matrix (G, plus ag0 C in a step)
  // with the lane's own direct solver; the resume launch restores the
  // lane's shared memory and state and continues the Newton solve with the
  // host's step (lane_solver.zig's per-lane peel).
  auto pause = [&](uint32_t phase, double ag0) {
    gather_pattern_tran(T, m, ag0, phase == 2, L.a_vals + size_t(lane) * T.nnz, tid);
    for (uint32_t i = tid; i < n; i += 32) {
      L.x[at + i] = m.x[i];
      L.rhs[at + i] = m.rhs[i];
      L.diag[at + i] = m.diag[i];
    }
    __syncwarp();
    for (uint32_t i = tid; i < bd; i += 32) sv[i] = block[i];
    if (tid == 0) {
      double* r = sv + bd;
      r[0] = t;
      r[1] = dt;
      r[2] = bp_next;
      r[3] = bp_save_dt;
      for (int k = 0; k < 6; ++k) r[4 + k] = dt_old[k];
      ts[kTrPhase] = phase;
      ts[kTrIter] = carry.iter;
      ts[kTrInitFix] = carry.init_fix;
      ts[kTrOrder] = uint32_t(order);
      ts[kTrSteps] = steps;
      ts[kTrHaveBp] = have_bp;
      ts[kTrBpClamped] = bp_clamped;
      ts[kTrHb] = hb;
      ts[kTrNRec] = n_rec;
      ts[kTrLimActive] = lim_active;
      for (int k = 0; k < kTsN; ++k) ts[kTrStat + k] = stat[k];
      L.limit[lane] = carry.limit;
      L.flags[lane] |= 2u;
      // the lane's first factor of all is its own fresh factor; a later
      // one continues the lead tape's history
      L.iters[lane] = (phase == 1 && carry.iter == 0 && L.ladder[lane].rung == kRungPlain) ? 0u : 1u;
      L.status[lane] = kNeedSolve;
      atomicAdd(L.n_paused, 1u);
    }
  };
  // Records the row (t, m.x) and feeds it to the measure cards; true while
  // a card is still open.
  auto record = [&](double tr) {
    bool open = false;
    if (P.meas) {
      const bool done = card ? meas_feed(P.meas[tid], mstate, tr, m.x) : true;
      open = __any_sync(kFull, !done);
    }
    if (P.out_t && n_rec < P.max_pts) {
      if (tid == 0) P.out_t[size_t(lane) * P.max_pts + n_rec] = tr;
      for (uint32_t k = tid; k < P.n_probes; k += 32)
        P.out_v[(size_t(lane) * P.max_pts + n_rec) * P.n_probes + k] = m.x[P.probes[k]];
      ++n_rec;
    }
    return open;
  };

  // operating point (op.solve with tran_op): op.zig's ladder from the cold
  // start (the junction seeds, MODEINITFIX), the source waves at t = 0
  // (kind 2: vsource.va:214-219); every run through one call site, the
  // ladder's state in L.ladder (across pauses too). in_run: resumed inside a
  // paused run.
  int rc = 0;
  if (phase0 != 2) {
    bool in_run = phase0 == 1;
    LadderMove mv{kStartCold, false, false, true, 3u, 0u};
    if (phase0 == 0 && tid == 0) L.ladder[lane] = LadderDev{kRungPlain};
    __syncwarp();
    LaneOpts op = o;
    op.residual_tol = 1e-9;
    op.gmin = 0.0;
    op.max_iter = 100;
    for (;;) {
      if (!in_run) {
        if (mv.done) break;
        if (mv.save)
          for (uint32_t i = tid; i < n; i += 32) L.x_good[at + i] = m.x[i];
        if (mv.start == kStartGood)
          for (uint32_t i = tid; i < n; i += 32) m.x[i] = L.x_good[at + i];
        if (mv.start == kStartCold) {
          for (uint32_t i = tid; i < n; i += 32) m.x[i] = 0.0;
          cold_images(T, rec, m.lim, tid, 32);
        }
        __syncwarp();
        lim_active = mv.start == kStartCold && T.nlim != 0;
        carry.iter = 0;
        carry.init_fix = mv.init_fix ? 1u : 0u;
        carry.resume = 0;
      }
      in_run = false;
      // the rung's gmin stamps, junction gmin and source factor
      const LadderRun run = ladder_run(op, L.ladder + lane);
      LaneOpts ro = op;
      ro.gstamp = run.gs;
      ro.max_iter = run.max_iter;
      SimDev rs = sim;
      rs.src_scale = run.src;
      rs.gmin = run.gmin_dev;
      fill_sources<32>(T, rec, rs, vsrc, tid);
      uint32_t it = 0;
      const int r = lane_newton<kHasB3>(T, prog, m, rec, ro, rs, nullptr, lim_active, carry.init_fix != 0, it, vsrc,
                                        tid, &carry);
      if (r == 3) {
        pause(1, 0.0);
        return;
      }
      carry.resume = 0;
      LadderDev ls = L.ladder[lane];
      mv = ladder_decide(ls, r == 0, r == 2 ? 0u : it);
      __syncwarp();
      if (tid == 0) L.ladder[lane] = ls;
      __syncwarp();
    }
    lim_active = false;
    stat[kTsOpIters] = mv.report;
    rc = mv.result < 3 ? 0 : 1;
  }
  if (rc != 0) {
    stat[kTsStatus] = kTranOpFailed;
  } else {
    const bool has_charge = T.q_ptr[n] != 0 || T.c_ptr[T.nnz] != 0;
    auto slot = [&](double* base, uint32_t len, uint32_t r) { return base + size_t((hb + r) & 3u) * len; };
    if (phase0 != 2) {
      // the operating point converged here (fresh, or resumed in it): the
      // run's start
      for (uint32_t i = tid; i < n; i += 32) {
        cur[i] = m.x[i];
        prev[i] = m.x[i];
      }
      // charge histories, flat at q(x_op); no dynamic current yet
      sim.kind = 1;
      eval_all<kHasB3>(T, rec, m, false, sim, tid, true);
      __syncwarp();
      for (uint32_t i = tid; i < 4 * n; i += 32) qh[i] = 0.0;
      __syncwarp();
      row_charges(T, prog, m, qh + n, tid);
      state_charges<32>(T, rec, m.x, qt + nq, tid);
      __syncwarp();
      for (uint32_t i = tid; i < n; i += 32) {
        qh[2 * n + i] = qh[n + i];
        qh[3 * n + i] = qh[n + i];
        ipr[i] = 0.0;
      }
      for (uint32_t j = tid; j < nq; j += 32) {
        qt[2 * nq + j] = qt[nq + j];
        qt[3 * nq + j] = qt[nq + j];
        ipt[j] = 0.0;
      }
      __syncwarp();
      pulse_timers<32>(T, rec, tmr, tid);
      dt = fmin(div_rn(fmin(P.t_step, div_rn(P.t_stop, 100.0)), 10.0), dt_max);
      double bp0;
      if (next_bp<32>(T, rec, tmr, min_break, bp0, tid, nullptr)) dt = fmin(dt, 0.1 * bp0);
      dt = div_rn(dt, 10.0);
      record(0.0);
    }
    LaneOpts nr = o;
    nr.residual_tol = CUDART_INF;
    nr.gmin = 0.0;
    nr.max_iter = 100;
    bool res_step = phase0 == 2;  // the first pass continues the paused step's Newton solve
    for (;;) {
      if (!res_step && !(t < P.t_stop && !almost_equal_ulps(t, P.t_stop, 100) && steps < P.max_steps)) break;
      const double t_dev = t + dt;
      sim.kind = 1;
      sim.t = t_dev;
      const bool trap = order == 2;
      const double ag0 = trap ? div_rn(div_rn(1.0, dt), 1.0 - 0.5) : div_rn(1.0, dt);
      const double ag1 = trap ? div_rn(0.5, 1.0 - 0.5) : 1.0;
      if (!res_step) {
        // predictor, limited against the accepted point
        const double xfact = div_rn(dt, dt_old[0]);
        for (uint32_t i = tid; i < n; i += 32) {
          m.x[i] = cur[i] + xfact * (cur[i] - prev[i]);
          m.xo[i] = cur[i];
        }
        __syncwarp();
        apply_limits<kHasB3>(T, rec, m, false, tid);
        lim_active = T.nlim != 0;
        carry.iter = 0;
        carry.init_fix = 0;
        carry.resume = 0;
        __syncwarp();
      }
      res_step = false;
      Companion c{ag0, ag1, trap, slot(qh, n, 1), ipr};
      uint32_t iters = 0;
      fill_sources<32>(T, rec, sim, vsrc, tid);
      rc = lane_newton<kHasB3>(T, prog, m, rec, nr, sim, &c, lim_active, false, iters, vsrc, tid, &carry);
      if (rc == 3) {
        pause(2, ag0);
        return;
      }
      carry.resume = 0;
      lim_active = false;
      stat[kTsAttempts] += 1;
      stat[kTsNrIters] += iters;
      if (rc != 0) {
        // out of iterations, or the host's factor of this lane was singular
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
        eval_all<kHasB3>(T, rec, m, false, sim, tid, true);
        __syncwarp();
        row_charges(T, prog, m, slot(qh, n, 0), tid);
        state_charges<32>(T, rec, m.x, slot(qt, nq, 0), tid);
        __syncwarp();
      }
      const double dt1 = dt_old[0], dt2 = dt_old[1];
      if (has_charge && steps > 0) {
        const int mth = trap ? 2 : 1;
        const double del = step_bound<32>(mth, mth, nq, slot(qt, nq, 0), slot(qt, nq, 1), slot(qt, nq, 2),
                                      slot(qt, nq, 3), ipt, ag0, ag1, dt, dt1, dt2, P, tid, nullptr);
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
          const double trial_del = step_bound<32>(2, 1, nq, slot(qt, nq, 0), slot(qt, nq, 1), slot(qt, nq, 2),
                                              slot(qt, nq, 3), ipt, ag0, ag1, dt, dt1, dt2, P, tid, nullptr);
          if (trial_del == trial_del) {
            const double nd2 = fmin(2.0 * dt, trial_del);
            if (nd2 > 1.05 * dt) order = 2;
            dt_next = fmin(fmax(nd2, P.dt_min), dt_max);
          }
        }
        // integrator.advanceCurrent over rows and states, then the rotation
        const double* q0 = slot(qh, n, 0);
        const double* q1 = slot(qh, n, 1);
        for (uint32_t i = tid; i < n; i += 32) {
          const double d = ag0 * (q0[i] - q1[i]);
          ipr[i] = trap ? d - ag1 * ipr[i] : d;
        }
        const double* s0 = slot(qt, nq, 0);
        const double* s1 = slot(qt, nq, 1);
        for (uint32_t j = tid; j < nq; j += 32) {
          const double d = ag0 * (s0[j] - s1[j]);
          ipt[j] = trap ? d - ag1 * ipt[j] : d;
        }
        hb = (hb + 3u) & 3u;
      }
      for (int k = 5; k > 0; --k) dt_old[k] = dt_old[k - 1];
      dt_old[0] = dt;
      for (uint32_t i = tid; i < n; i += 32) {
        prev[i] = cur[i];
        cur[i] = m.x[i];
      }
      __syncwarp();
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
          if (next_bp<32>(T, rec, tmr, t_new + min_break, nb, tid, nullptr)) shrink = fmin(shrink, nb - t_new);
          dt_next = fmin(dt_next, 0.1 * shrink);
        }
        have_bp = false;
      }
      const bool open = record(t_new);
      if (P.meas && P.early_stop && !open) {
        // tran.zig:1060-1063: every card resolved, the run ends here
        stat[kTsStatus] = kTranResolved;
        break;
      }
      have_bp = next_bp<32>(T, rec, tmr, t_new + min_break, bp_next, tid, nullptr);
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
    for (uint32_t i = tid; i < n; i += 32) m.x[i] = cur[i];
    __syncwarp();
  }
  for (uint32_t i = tid; i < n; i += 32) L.x[size_t(lane) * n + i] = m.x[i];
  if (card) P.meas_out[size_t(lane) * P.n_meas + tid] = meas_value(P.meas[tid], mstate);
  if (tid < kTsN) P.stats[size_t(lane) * kTsN + tid] = stat[tid];
  if (tid == 0) {
    if (P.n_pts) P.n_pts[lane] = n_rec;
    L.status[lane] = kConverged;  // done: a resume launch passes it by
  }
}

// One lane's sequential .dc sweep over the points of one swept source
// (dc.zig Sweep, :163-386): per point the MODEINITPRED predictor
// 2 last - prev (:330-337), limited against the last point (prepareWarm,
// :342-347), and a warm Newton; when that fails, or before any point has
// converged, a cold start (op.zig coldStart: zero x and the junction seeds)
// and Newton with MODEINITFIX at the operating point's 100 iterations, the
// ladder's plain rung (endPoint, dc.zig:361-365). Point 0, once converged,
// is also `prev` (dc.zig:376-379, after dctrcurv.c). A factor that leaves
// the lead tape pauses the lane for the host (sweep_lane below).
//
// The cold start of a sweep point (op.zig coldStart): x = 0, every junction
// image at its seed.
template <bool kHasB3>
__device__ void sweep_seed(const TopoDev& T, const double* rec, const LaneMem& m, int tid) {
  for (uint32_t i = tid; i < T.n; i += 32) m.x[i] = 0.0;
  cold_images(T, rec, m.lim, tid, 32);
}

// A sweep lane (dc.zig Sweep, one per lane): per point, the predictor
// limited against the last point and a warm Newton; on its failure, or
// before any point has converged, the cold rung (op.zig's plain rung at 100
// iterations with MODEINITFIX). A factor the lead tape cannot stand in for
// pauses the lane (the DC lanes' protocol: the matrix, residual and
// diagonal to the hand-off planes, L.status kNeedSolve); the host factors it
// on the lane's own direct solver and a resume launch continues the lane at
// that point, phase and iteration with the host's step (or its singular
// verdict). The lane keeps pausing before every factor until its own factor
// is the lead tape again (the host clears the host-mode flag).
template <bool kHasB3>
__device__ void sweep_lane(const TopoDev& T, const LaneDev& L, const SweepDev& P, const LaneOpts& o, uint32_t prog,
                           double* block, uint32_t lane, int tid) {
  const uint32_t n = T.n;
  const uint32_t lstat = L.status[lane];
  const bool resuming = L.resume && (lstat == kNeedSolve || lstat == kSingular);
  if (!(lstat == kRunning || resuming)) return;
  LaneMem m = carve(T, block);
  double* sol = block + T.smem_doubles;
  double* prev = sol + n;
  double* vsrc = prev + n;  // T.n_src
  const double* rec = L.rec + size_t(lane) * T.rec_size;
  uint32_t* sw = P.state + size_t(lane) * kSweepStateN;
  init_consts(T, m.v, tid);
  SimDev sim;
  sim.t = 0.0;
  sim.src_scale = 1.0;
  sim.kind = 0;
  fill_sources<32>(T, rec, sim, vsrc, tid);
  LaneOpts cold_o = o;
  cold_o.max_iter = 100;
  uint32_t status = kSweepDone;
  bool cold = true;
  uint32_t pt0 = 0, phase0 = 0, it_total0 = 0;
  bool lim_active = false;
  NewtonCarry carry{0u, kXPlausible, 0u, 0u, (L.flags[lane] & 2u) ? 1u : 0u};
  if (resuming) {
    pt0 = sw[kSwPoint];
    phase0 = sw[kSwPhase];
    it_total0 = sw[kSwItTotal];
    cold = sw[kSwCold] != 0;
    lim_active = sw[kSwLimActive] != 0;
    carry.iter = sw[kSwIter];
    carry.init_fix = sw[kSwInitFix];
    carry.limit = L.limit[lane];
    carry.resume = lstat == kSingular ? 2u : 1u;
    const size_t at = size_t(lane) * n;
    for (uint32_t i = tid; i < n; i += 32) {
      sol[i] = P.rows[2 * at + i];
      prev[i] = P.rows[2 * at + n + i];
      m.x[i] = L.x[at + i];
      m.rhs[i] = L.rhs[at + i];
      m.diag[i] = L.diag[at + i];
    }
    for (uint32_t i = tid; i < T.nlim; i += 32) m.lim[i] = L.lim[size_t(lane) * T.nlim + i];
    for (uint32_t j = tid; j < n; j += 32) m.y[j] = L.dx[at + T.qcol[j]];
  } else {
    for (uint32_t i = tid; i < n; i += 32) {
      sol[i] = 0.0;
      prev[i] = 0.0;
    }
  }
  // Pause: the lane's state for the host and for the resume launch.
  auto pause = [&](uint32_t pt, uint32_t phase, uint32_t it_total, bool fresh) {
    const size_t at = size_t(lane) * n;
    gather_pattern(T, m, L.a_vals + size_t(lane) * T.nnz, tid);
    for (uint32_t i = tid; i < n; i += 32) {
      L.x[at + i] = m.x[i];
      L.rhs[at + i] = m.rhs[i];
      L.diag[at + i] = m.diag[i];
      P.rows[2 * at + i] = sol[i];
      P.rows[2 * at + n + i] = prev[i];
    }
    for (uint32_t i = tid; i < T.nlim; i += 32) L.lim[size_t(lane) * T.nlim + i] = m.lim[i];
    if (tid == 0) {
      sw[kSwPoint] = pt;
      sw[kSwPhase] = phase;
      sw[kSwItTotal] = it_total;
      sw[kSwCold] = cold;
      sw[kSwIter] = carry.iter;
      sw[kSwInitFix] = carry.init_fix;
      sw[kSwLimActive] = lim_active;
      L.limit[lane] = carry.limit;
      L.flags[lane] |= 2u;
      // the lane's first factor of all is its own fresh factor; a later
      // one continues the lead tape's history
      L.iters[lane] = fresh ? 0u : 1u;
      L.status[lane] = kNeedSolve;
      atomicAdd(L.n_paused, 1u);
    }
  };
  __syncwarp();
  for (uint32_t pt = pt0; pt < P.n_pts; ++pt) {
    const size_t row = size_t(lane) * P.n_pts + pt;
    const bool res_here = resuming && pt == pt0;
    if (tid == 0) vsrc[P.src] = P.values[pt];
    uint32_t it_total = res_here ? it_total0 : 0u;
    if (!res_here) {
      for (uint32_t i = tid; i < n; i += 32) {
        const double last = sol[i];
        sol[i] = 2.0 * last - prev[i];
        prev[i] = last;
      }
    }
    __syncwarp();
    // The point's Newton runs through one call site: the warm run (stage 0)
    // and, when it fails or no point has converged yet, the cold ladder's
    // runs (stage 2; dc.zig endPoint: op.nodesetLadder from the cold start,
    // rung 1 first). in_run: resumed inside a paused run.
    // The ladder's state stays in L.ladder (across pauses too).
    uint32_t stage = res_here ? phase0 : (cold ? 2u : 0u);
    bool in_run = res_here;
    LadderMove mv{kStartCold, false, false, true, 3u, 0u};
    if (stage == 2 && !res_here && tid == 0) L.ladder[lane] = LadderDev{kRungPlain};
    __syncwarp();
    bool scaled = false;  // the sources hold a source-stepping factor
    int rc = 1;
    const size_t at = size_t(lane) * n;
    for (;;) {
      LaneOpts ro = o;
      SimDev rs = sim;
      if (stage == 2) {
        if (!in_run) {
          if (mv.done) break;
          // the next run's start: its own end point, the last good
          // stepping point or the cold start
          if (mv.save)
            for (uint32_t i = tid; i < n; i += 32) L.x_good[at + i] = m.x[i];
          if (mv.start == kStartGood)
            for (uint32_t i = tid; i < n; i += 32) m.x[i] = L.x_good[at + i];
          if (mv.start == kStartCold) sweep_seed<kHasB3>(T, rec, m, tid);
          __syncwarp();
          lim_active = mv.start == kStartCold && T.nlim != 0;
          carry.iter = 0;
          carry.init_fix = mv.init_fix ? 1u : 0u;
          carry.resume = 0;
        }
        // the rung's gmin stamps, junction gmin and source factor (the
        // swept source's value scaled with the others)
        const LadderRun run = ladder_run(cold_o, L.ladder + lane);
        ro = cold_o;
        ro.gstamp = run.gs;
        ro.max_iter = run.max_iter;
        rs.src_scale = run.src;
        rs.gmin = run.gmin_dev;
        if (scaled || run.src != 1.0) {
          fill_sources<32>(T, rec, rs, vsrc, tid);
          if (tid == 0) vsrc[P.src] = P.values[pt] * run.src;
          __syncwarp();
          scaled = run.src != 1.0;
        }
      } else if (!in_run) {
        // the warm start: the predictor limited against the last point
        for (uint32_t i = tid; i < n; i += 32) {
          m.x[i] = sol[i];
          m.xo[i] = prev[i];
        }
        __syncwarp();
        apply_limits<kHasB3>(T, rec, m, false, tid);
        lim_active = T.nlim != 0;
        carry.iter = 0;
        carry.resume = 0;
        __syncwarp();
      }
      in_run = false;
      uint32_t it = 0;
      const int r = lane_newton<kHasB3>(T, prog, m, rec, ro, rs, nullptr, lim_active,
                                        stage == 2 && carry.init_fix != 0, it, vsrc, tid, &carry);
      if (r == 3) {
        pause(pt, stage, it_total, pt == 0 && carry.iter == 0 && (stage == 0 || L.ladder[lane].rung == kRungPlain));
        return;
      }
      carry.resume = 0;
      if (stage == 0) {
        it_total += it;
        for (uint32_t i = tid; i < n; i += 32) sol[i] = m.x[i];
        __syncwarp();
        if (r == 0) {
          rc = 0;
          break;
        }
        stage = 2;
        if (tid == 0) L.ladder[lane] = LadderDev{kRungPlain};
        __syncwarp();
        mv = LadderMove{kStartCold, false, false, true, 3u, 0u};
        continue;
      }
      LadderDev ls = L.ladder[lane];
      mv = ladder_decide(ls, r == 0, r == 2 ? 0u : it);
      __syncwarp();
      if (tid == 0) L.ladder[lane] = ls;
      __syncwarp();
    }
    if (stage == 2) {
      rc = mv.result < 3 ? 0 : 1;
      it_total += mv.report;
      if (scaled) {
        fill_sources<32>(T, rec, sim, vsrc, tid);
        if (tid == 0) vsrc[P.src] = P.values[pt];
      }
      for (uint32_t i = tid; i < n; i += 32) sol[i] = m.x[i];
      __syncwarp();
    }
    const bool converged = rc == 0;
    for (uint32_t i = tid; i < n; i += 32) P.x_out[row * n + i] = sol[i];
    if (tid == 0) {
      P.iters[row] = it_total;
      P.conv[row] = converged ? 1 : 0;
    }
    if (converged) {
      if (pt == 0)
        for (uint32_t i = tid; i < n; i += 32) prev[i] = sol[i];
      cold = false;
    } else {
      cold = true;
    }
    __syncwarp();
  }
  if (tid == 0) {
    P.status[lane] = status;
    L.status[lane] = kConverged;  // this lane's sweep is done
  }
}

// Uneven batching: lanes of several topologies (circuits of different sizes)
// in one launch. CTA b serves topology cta_ctx[b], lanes cta_first[b] ..
// + ctx_lpb[that topology] (one warp each); it copies its topology's tables
// into shared memory and stages that topology's programs, then runs the same
// per-lane solve as dc_newton_kernel.
template <bool kHasB3>
__global__ void __launch_bounds__(256) dc_newton_group_kernel(const TopoDev* Ts, const LaneDev* Ls,
                                                              const uint32_t* cta_ctx, const uint32_t* cta_first,
                                                              const uint32_t* ctx_lpb, LaneOpts o) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ TopoDev T;
  __shared__ LaneDev L;
  const uint32_t c = cta_ctx[blockIdx.x];
  if (threadIdx.x == 0) {
    T = Ts[c];
    L = Ls[c];
  }
  __syncthreads();
  double* lanes_smem = stage_programs(T, smem_raw);
  const uint32_t prog = saddr(smem_raw);
  const int tid = threadIdx.x & 31;
  const uint32_t w = threadIdx.x >> 5;
  const uint32_t lane = cta_first[blockIdx.x] + w;
  if (w < ctx_lpb[c] && lane < L.n_lanes)
    dc_solve_lane<kHasB3>(T, L, o, prog, lanes_smem + size_t(w) * T.smem_doubles, lane, tid);
}

cudaError_t launch_dc_newton_group(const TopoDev* d_topos, const LaneDev* d_lanes, const uint32_t* d_cta_ctx,
                                   const uint32_t* d_cta_first, const uint32_t* d_ctx_lpb, uint32_t n_ctas,
                                   uint32_t max_lpb, size_t smem, const LaneOpts& o, bool has_b3, cudaStream_t s) {
  auto* k = has_b3 ? dc_newton_group_kernel<true> : dc_newton_group_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  k<<<n_ctas, 32 * max_lpb, smem, s>>>(d_topos, d_lanes, d_cta_ctx, d_cta_first, d_ctx_lpb, o);
  return cudaGetLastError();
}

// Transient lanes: a persistent grid, each CTA staging the programs once,
// each warp running one lane's transient to its end.
template <bool kHasB3>
__global__ void __launch_bounds__(256) tran_kernel(TopoDev T, LaneDev L, TranDev P, LaneOpts o) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* lanes_smem = stage_programs(T, smem_raw);
  const uint32_t prog = saddr(smem_raw);
  const int tid = threadIdx.x & 31;
  const uint32_t warps = blockDim.x >> 5, w = threadIdx.x >> 5;
  double* block = lanes_smem + size_t(w) * (T.tran_doubles + kMeasDoubles * P.n_meas);
  // Lane refill: a warp that finishes takes the next lane from a counter,
  // so lanes of unequal length (early stops, rejections) balance over the
  // GPU instead of following a fixed stride.
  for (;;) {
    uint32_t lane = 0;
    if (tid == 0) lane = atomicAdd(P.next_lane, 1u);
    lane = __shfl_sync(kFull, lane, 0);
    if (lane >= L.n_lanes) break;
    tran_lane<kHasB3>(T, L, P, o, prog, block, lane, tid);
    __syncwarp();
  }
}

template <bool kHasB3>
__global__ void __launch_bounds__(256) sweep_kernel(TopoDev T, LaneDev L, SweepDev P, LaneOpts o) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* lanes_smem = stage_programs(T, smem_raw);
  const uint32_t prog = saddr(smem_raw);
  const int tid = threadIdx.x & 31;
  const uint32_t warps = blockDim.x >> 5, w = threadIdx.x >> 5;
  double* block = lanes_smem + size_t(w) * sweep_doubles(T);
  for (;;) {  // lane refill, as tran_kernel
    uint32_t lane = 0;
    if (tid == 0) lane = atomicAdd(P.next_lane, 1u);
    lane = __shfl_sync(kFull, lane, 0);
    if (lane >= L.n_lanes) break;
    sweep_lane<kHasB3>(T, L, P, o, prog, block, lane, tid);
    __syncwarp();
  }
}

cudaError_t launch_sweep(const TopoDev& T, const LaneDev& L, const SweepDev& P, const LaneOpts& o,
                         uint32_t lanes_per_block, cudaStream_t s) {
  const size_t smem = T.prog_bytes + lanes_per_block * size_t(sweep_doubles(T)) * sizeof(double);
  auto* k = topo_has_b3(T) ? sweep_kernel<true> : sweep_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(P.next_lane, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  k<<<persistent_grid(k, L.n_lanes, lanes_per_block, smem), 32 * lanes_per_block, smem, s>>>(T, L, P, o);
  return cudaGetLastError();
}

cudaError_t launch_tran(const TopoDev& T, const LaneDev& L, const TranDev& P, const LaneOpts& o,
                        uint32_t lanes_per_block, cudaStream_t s) {
  const size_t smem =
      T.prog_bytes + lanes_per_block * size_t(T.tran_doubles + kMeasDoubles * P.n_meas) * sizeof(double);
  auto* k = topo_has_b3(T) ? tran_kernel<true> : tran_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(P.next_lane, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  k<<<persistent_grid(k, L.n_lanes, lanes_per_block, smem), 32 * lanes_per_block, smem, s>>>(T, L, P, o);
  return cudaGetLastError();
}

}  // namespace esl

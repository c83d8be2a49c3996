// Per-lane device evaluation shared by the warp lanes (newton.cu) and the
// block lanes (block.cu): the lane's working-set view, device evaluation
// into staging cells, the junction limiters, the residual gate and the
// pattern-order matrix of a paused lane. Each loop strides over the lane's
// kStride threads: 32 when a warp owns the lane, the CTA's width when a
// block does.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include "lanes.cuh"
#include "models.cuh"
#include "bsim3.cuh"

namespace esl {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr double kGrowth = 1e-12;    // direct.zig refactor_growth_limit
constexpr double kWide = 1e3;        // 1 / direct.zig pivot_tol
constexpr double kXPlausible = 1e9;  // converger.zig x_plausible

__device__ __forceinline__ uint64_t dbits(double x) { return static_cast<uint64_t>(__double_as_longlong(x)); }
__device__ __forceinline__ double from_bits(uint64_t u) { return __longlong_as_double(static_cast<long long>(u)); }

// One lane's shared block (the host's lane_layout).
struct LaneMem {
  double* base;
  double* x;     // n: current iterate
  double* xo;    // n: previous iterate
  double* rhs;   // n: residual F(x)
  double* diag;  // n: assembled diagonal (gates, runaway bound)
  double* v;     // tape values (U, diagonal, L, discard) | y | 0.0 | 1.0 | sink
  double* y;     // n: permuted solve vector, inside v
  double* st;    // n_stage: device contributions
  double* lim;   // nlim: limited junction images
};

__device__ __forceinline__ LaneMem carve(const TopoDev& T, double* base) {
  LaneMem m;
  m.base = base;
  m.x = base;
  m.xo = m.x + T.n;
  m.rhs = m.xo + T.n;
  m.diag = m.rhs + T.n;
  m.v = m.diag + T.n;
  m.y = m.v + T.ntv;
  m.st = m.v + T.nv;
  m.lim = m.st + T.n_stage;
  return m;
}

// Device evaluation: every instance of every batch, strided over the lane's
// kStride threads (a warp, or a block lane's CTA),
// each writing its own staging cells (no shared cell, no atomics).
template <bool kHasB3, uint32_t kStride = 32>
__device__ void eval_all(const TopoDev& T, const double* rec, const LaneMem& m, bool lim_active,
                         const SimDev& sim, int tid, bool charges_only = false, const double* vcache = nullptr,
                         bool dc_only = false) {
  for (uint32_t bi = 0; bi < T.n_batches; ++bi) {
    const BatchDev& B = T.b[bi];
    // a DC solve reads no charge cell: capacitors stamp nothing else
    if (dc_only && B.type == kC) continue;
    // the charge re-read (the reference's evalQ) needs only the batches
    // that carry charge: capacitors, diodes, MOSFETs with charge cells
    if (charges_only && !(B.type == kC || B.type == kD || (B.type == kM && B.stride >= kStageM))) continue;
    const int s = static_cast<int>(B.count);
    for (uint32_t i = tid; i < B.count; i += kStride) {
      const uint32_t* nd = B.nodes + size_t(i) * B.nt;
      double* st = m.st + B.stage_base + size_t(i) * B.stride;
      const double* r = rec + B.rec_off + i;
      switch (B.type) {
        case kR: {
          const double rv = r[0];
          const double g = 1.0 / rv;
          const double cur = div_rn(m.x[nd[0]] - m.x[nd[1]], rv);
          st[0] = cur;
          st[1] = -cur;
          st[2] = g;
          st[3] = -g;
          st[4] = -g;
          st[5] = g;
          break;
        }
        case kC: {
          const double c = r[0];
          const double q = c * (m.x[nd[0]] - m.x[nd[1]]);
          st[0] = q;
          st[1] = -q;
          st[2] = c;
          st[3] = -c;
          st[4] = -c;
          st[5] = c;
          break;
        }
        case kV: {
          const double v = vcache ? vcache[B.src_off + i] : source_value(r, s, sim);
          const double ib = m.x[nd[2]];
          st[0] = ib;
          st[1] = -ib;
          st[2] = m.x[nd[0]] - m.x[nd[1]] - v;
          st[3] = 1.0;
          st[4] = -1.0;
          st[5] = 1.0;
          st[6] = -1.0;
          break;
        }
        case kI: {
          const double v = vcache ? vcache[B.src_off + i] : source_value(r, s, sim);
          st[0] = v;
          st[1] = -v;
          break;
        }
        case kM:
          mos1_stamp(r, s, m.x[nd[0]], m.x[nd[1]], m.x[nd[2]], m.x[nd[3]], m.x[nd[4]], m.x[nd[5]],
                     lim_active ? m.lim + B.lim_off + 3 * i : nullptr, sim.kind == 1 && B.stride >= kStageM, st);
          break;
        case kD:
          diode_stamp(r, s, m.x[nd[0]], m.x[nd[1]], m.x[nd[2]], lim_active ? m.lim + B.lim_off + i : nullptr, st);
          break;
        case kB3:
          if constexpr (kHasB3)
            bsim3_stamp(r, s, m.x[nd[0]], m.x[nd[1]], m.x[nd[2]], m.x[nd[3]], m.x[nd[4]], m.x[nd[5]],
                        lim_active ? m.lim + B.lim_off + 3 * i : nullptr, st, sim.gmin);
          break;
        default:
          break;
      }
    }
  }
}

// The matrix in pattern order, for a lane the host factors (the CSR lists,
// staging indices or the two pin sources).
template <uint32_t kStride = 32>
__device__ void gather_pattern(const TopoDev& T, const LaneMem& m, double* out, int tid) {
  for (uint32_t p = tid; p < T.nnz; p += kStride) {
    double s = 0.0;
    for (uint32_t e = T.a_ptr[p]; e < T.a_ptr[p + 1]; ++e) {
      const uint32_t src = T.a_src[e];
      s = __dadd_rn(s, src == kSrcOne ? 1.0 : src == kSrcX0 ? m.x[0] : m.st[src]);
    }
    out[p] = s;
  }
}

__device__ __forceinline__ double residual_gate(const LaneOpts& o, double diag, double xi) {
  const double scale = fabs(diag);
  const double s = scale == 0.0 ? 1.0 : scale;
  return fmax(o.residual_tol, 10.0 * s * (o.reltol * fabs(xi) + o.vntol));
}

// pnjlim on every diode, and the MOS1 ladder on every MOSFET, against their
// images (or x_old before the first pass); true when any junction was
// limited (Circuit.applyLimits): across the warp when the lane is a warp,
// this thread's own flag when it is a CTA.
template <bool kHasB3, uint32_t kStride = 32>
__device__ bool apply_limits(const TopoDev& T, const double* rec, const LaneMem& m, bool lim_active, int tid) {
  bool limited = false;
  for (uint32_t bi = 0; bi < T.n_batches; ++bi) {
    const BatchDev& B = T.b[bi];
    const int s = static_cast<int>(B.count);
    if (B.type == kM || B.type == kB3) {
      for (uint32_t i = tid; i < B.count; i += kStride) {
        const uint32_t* nd = B.nodes + size_t(i) * B.nt;
        double* li = m.lim + B.lim_off + 3 * i;
        double old[3];
        if (lim_active) {
          old[0] = li[0];
          old[1] = li[1];
          old[2] = li[2];
        } else {
          const double type = rec[B.rec_off + (B.type == kM ? kMType : kB3Type) * s + i];
          old[0] = type * (m.xo[nd[1]] - m.xo[nd[5]]);
          old[1] = type * (m.xo[nd[4]] - m.xo[nd[5]]);
          old[2] = type * (m.xo[nd[3]] - m.xo[nd[5]]);
        }
        if (B.type == kM)
          limited |= mos1_limit(rec + B.rec_off + i, s, m.x[nd[1]], m.x[nd[3]], m.x[nd[4]], m.x[nd[5]], old, li);
        else if constexpr (kHasB3)
          limited |= bsim3_limit(rec + B.rec_off + i, s, m.x[nd[1]], m.x[nd[3]], m.x[nd[4]], m.x[nd[5]], old, li);
      }
      continue;
    }
    if (B.type != kD) continue;
    for (uint32_t i = tid; i < B.count; i += kStride) {
      const uint32_t* nd = B.nodes + size_t(i) * B.nt;
      const double* r = rec + B.rec_off + i;
      const double vnew = m.x[nd[2]] - m.x[nd[1]];
      const double vold = lim_active ? m.lim[B.lim_off + i] : m.xo[nd[2]] - m.xo[nd[1]];
      bool l = false;
      m.lim[B.lim_off + i] = pnjlim_dev(vnew, vold, r[kDVte * s], r[kDVcrit * s], l);
      limited |= l;
    }
  }
  if constexpr (kStride == 32) return __any_sync(kFull, limited);
  return limited;  // the block lane reduces it across its CTA
}

}  // namespace

}  // namespace esl

// The transient step control's per-lane pieces (tran.zig Sim.begin/Sim.end
// and the integrator.zig kernels), written for a lane of kW threads: a warp
// (kW 32: warp shuffles) or a block lane's CTA (kW > 32: shuffles, then one
// word per warp through `red` in shared memory). Each returns the same
// value on every thread of the lane.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include <cstdint>

#include "../common.h"
#include "lanes.cuh"
#include "models.cuh"

namespace esl {

constexpr double kLteBe = 0.5;              // integrator.lteCoeff, gearCoeff[0]
constexpr double kLteTrap = 0.08333333333;  // trapCoeff[1]

// fmin over the lane's threads (NaN ignored, as fmin does).
template <uint32_t kW>
__device__ __forceinline__ double lane_fmin(double v, uint64_t* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if constexpr (kW == 32) {
    return v;
  } else {
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = __double_as_longlong(v);
    __syncthreads();
    double r = __longlong_as_double(red[0]);
#pragma unroll
    for (uint32_t w = 1; w < kW / 32; ++w) r = fmin(r, __longlong_as_double(red[w]));
    __syncthreads();
    return r;
  }
}

// True on every thread when p holds on any thread of the lane.
template <uint32_t kW>
__device__ __forceinline__ bool lane_any(bool p) {
  if constexpr (kW == 32)
    return __any_sync(0xffffffffu, p);
  else
    return __syncthreads_or(p) != 0;
}

template <uint32_t kW>
__device__ __forceinline__ void lane_sync() {
  if constexpr (kW == 32)
    __syncwarp();
  else
    __syncthreads();
}

// a and b equal or at most `ulps` representable doubles apart, of one sign.
__device__ __forceinline__ bool almost_equal_ulps(double a, double b, long long ulps) {
  if (a == b) return true;
  if ((a < 0) != (b < 0)) return false;
  const long long d = __double_as_longlong(a) - __double_as_longlong(b);
  return (d < 0 ? -d : d) <= ulps;
}

// integrator.stepBound over the lane's m charge states: the LTE step for
// `method` (1 BE, 2 trapezoidal) with the current currents of order `cur`;
// NaN when any input or bound is not finite.
template <uint32_t kW>
__device__ __forceinline__ double step_bound(int method, int cur, uint32_t m, const double* q0, const double* q1,
                                             const double* q2, const double* q3, const double* ip, double ag0,
                                             double ag1, double dt, double dt1, double dt2, const TranDev& P, int tid,
                                             uint64_t* red) {
  const double sum01 = dt + dt1, sum12 = dt1 + dt2, sum012 = dt + (dt1 + dt2);
  const double coeff = method == 1 ? kLteBe : kLteTrap;
  double vmin = CUDART_INF, poison = 0.0;
  for (uint32_t j = tid; j < m; j += kW) {
    const double qc = q0[j], qp = q1[j], qp2 = q2[j], ipj = ip[j];
    const double i_new = cur == 2 ? ag0 * (qc - qp) - ag1 * ipj : ag0 * (qc - qp);
    const double volttol = P.abstol + P.reltol * fmax(fabs(i_new), fabs(ipj));
    const double chargetol = div_rn(P.reltol * fmax(fmax(fabs(qc), fabs(qp)), P.chgtol), dt);
    const double tol = fmax(volttol, chargetol);
    poison += (qc - qc) + (qp - qp) + (qp2 - qp2) + (ipj - ipj);
    const double f12 = div_rn(qp - qp2, dt1);
    double dd = div_rn(div_rn(qc - qp, dt) - f12, sum01);
    if (method != 1) {
      const double qp3 = q3[j];
      poison += qp3 - qp3;
      const double f123 = div_rn(f12 - div_rn(qp2 - qp3, dt2), sum12);
      dd = div_rn(dd - f123, sum012);
    }
    const double del = div_rn(P.trtol * tol, fmax(P.abstol, coeff * fabs(dd)));
    poison += del == del ? 0.0 : del;
    vmin = fmin(vmin, del);
  }
  vmin = lane_fmin<kW>(vmin, red);
  if (lane_any<kW>(poison != poison)) return CUDART_NAN;
  return method == 1 ? vmin : sqrt(vmin);
}

// PULSE corner timers: for each V and I source, its four corners' first
// times and the period (infinite for other waves), 8 doubles a source.
template <uint32_t kW>
__device__ void pulse_timers(const TopoDev& T, const double* rec, double* tm, int tid) {
  for (uint32_t bi = 0; bi < T.n_batches; ++bi) {
    const BatchDev& B = T.b[bi];
    if (B.type != kV && B.type != kI) continue;
    const int s = static_cast<int>(B.count);
    for (uint32_t i = tid; i < B.count; i += kW) {
      const double* p = rec + B.rec_off + i;
      double* t = tm + 8 * (B.src_off + i);
      if (p[1 * s] != 1.0) {
        for (int k = 0; k < 4; ++k) {
          t[2 * k] = CUDART_INF;
          t[2 * k + 1] = 1.0;
        }
        continue;
      }
      const double tr = p[5 * s] > 1.0e-12 ? p[5 * s] : 1.0e-12;
      const double tf = p[6 * s] > 1.0e-12 ? p[6 * s] : 1.0e-12;
      const double pwr = p[7 * s];
      const double pw = (pwr > 0.0 ? pwr : 0.0) + (-pwr > 0.0 ? -pwr : 0.0) * 1.0e30;
      double per = p[8 * s];
      const double per_min = tr + pw + tf + 1.0e-12;
      if (per < per_min) per = per_min;
      const double td = p[4 * s];
      const double st[4] = {td, td + tr, td + tr + pw, td + tr + pw + tf};
      for (int k = 0; k < 4; ++k) {
        t[2 * k] = st[k];
        t[2 * k + 1] = per;
      }
    }
  }
  lane_sync<kW>();
}

// The first source breakpoint at or after `after` (PULSE corners from the
// timers, PWL corners from the records); false when none.
template <uint32_t kW>
__device__ bool next_bp(const TopoDev& T, const double* rec, const double* tm, double after, double& bp, int tid,
                        uint64_t* red) {
  double best = CUDART_INF;
  for (uint32_t k = tid; k < 4 * T.n_src; k += kW) {
    const double start = tm[2 * k], per = tm[2 * k + 1];
    if (!(start < CUDART_INF)) continue;
    double t = start;
    if (t < after) {
      const double kk = ceil(div_rn(after - start, per));
      t = start + kk * per;
      if (t < after) t += per;
    }
    if (t < best) best = t;
  }
  for (uint32_t bi = 0; bi < T.n_batches; ++bi) {
    const BatchDev& B = T.b[bi];
    if (B.type != kV && B.type != kI) continue;
    const int s = static_cast<int>(B.count);
    for (uint32_t i = tid; i < B.count; i += kW) {
      const double* p = rec + B.rec_off + i;
      if (p[s] != 4.0) continue;
      const int len = static_cast<int>(p[2 * s]);
      const double td = p[4 * s];
      if (len < kPwlMax && td >= after && td < best) best = td;
      for (int j = 0; j < len; ++j) {
        const double c = p[(kSrcPwlT + j) * s] + td;
        if (c >= after) {
          if (c < best) best = c;
          break;  // the table is sorted: the first corner at or after `after`
        }
      }
    }
  }
  best = lane_fmin<kW>(best, red);
  if (best == CUDART_INF) return false;
  bp = best;
  return true;
}

// The LTE charge states of every instance at x (capacitor charge, diode
// depletion + diffusion charge, MOS1 overlap charges), into out at each
// batch's qt_off.
template <uint32_t kW>
__device__ __forceinline__ void state_charges(const TopoDev& T, const double* rec, const double* x, double* out,
                                              int tid) {
  for (uint32_t bi = 0; bi < T.n_batches; ++bi) {
    const BatchDev& B = T.b[bi];
    if (B.qt_sites == 0) continue;
    const int s = static_cast<int>(B.count);
    for (uint32_t i = tid; i < B.count; i += kW) {
      const uint32_t* nd = B.nodes + size_t(i) * B.nt;
      const double* r = rec + B.rec_off + i;
      double* o = out + B.qt_off + i * B.qt_sites;
      if (B.type == kC) {
        o[0] = r[0] * (x[nd[0]] - x[nd[1]]);
      } else if (B.type == kD) {
        double q = 0.0, c;
        if (r[kDHasQ * s] != 0.0) {
          const double vd = x[nd[2]] - x[nd[1]];
          double id, gd;
          diode_iv(r, s, vd, id, gd);
          diode_qc(r, s, vd, id, gd, q, c);
        }
        o[0] = q;
      } else if (B.type == kM) {
        const double xg = x[nd[1]];
        o[0] = r[kMCgs * s] * (xg - x[nd[5]]);
        o[1] = r[kMCgd * s] * (xg - x[nd[4]]);
        o[2] = r[kMCgb * s] * (xg - x[nd[3]]);
      }
    }
  }
}

// Every V and I source's value at sim (time, source factor) into vcache.
template <uint32_t kW>
__device__ void fill_sources(const TopoDev& T, const double* rec, const SimDev& sim, double* vcache, int tid) {
  for (uint32_t bi = 0; bi < T.n_batches; ++bi) {
    const BatchDev& B = T.b[bi];
    if (B.type != kV && B.type != kI) continue;
    for (uint32_t i = tid; i < B.count; i += kW)
      vcache[B.src_off + i] = source_value(rec + B.rec_off + i, static_cast<int>(B.count), sim);
  }
  lane_sync<kW>();
}

}  // namespace esl

// The operating-point ladder on the device (op.zig solveLadder and
// afterPlain, rungs 1-3): between a lane's Newton runs, the warp or CTA that
// owns the lane decides the next run the way the reference's continuation
// does, and sets up its start (the cold start, the last converged stepping
// point, or the run's own end point). Rungs 4 (JFNK) and 5 (OPtran) are
// not built: a lane that the full-source Newton after source stepping does
// not converge reads not converged.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../common.h"
#include "lanes.cuh"
#include "models.cuh"

namespace esl {

constexpr double kLadderGminStart = 1e-2;    // Tolerances.gmin_start (numerics.zig:389)
constexpr double kLadderGminTarget = 1e-12;  // Tolerances.gmin
constexpr uint32_t kLadderItl2 = 50;         // Tolerances.itl2

// The settings of one Newton run under the ladder: the stamps' gmin (0:
// none), the source factor, the junction gmin the BSIM3 cards read
// (negative: the card's) and the iteration cap. Every run's cap is at least
// 100 (optionsFromTolerances); the stepping rungs pass itl2, so theirs is
// 100 too. `ld` null: a plain DC solve.
struct LadderRun {
  double gs, src, gmin_dev;
  uint32_t max_iter;
};

__device__ __forceinline__ LadderRun ladder_run(const LaneOpts& o, const LadderDev* ld) {
  LadderRun r{0.0, 1.0, -1.0, o.max_iter < 100 ? 100u : o.max_iter};
  if (ld) {
    const uint32_t rung = ld->rung;
    if (rung == kRungGmin) {
      r.gs = ld->gmin_val;
      r.gmin_dev = ld->gmin_val;
      r.max_iter = kLadderItl2 < 100 ? 100u : kLadderItl2;
    } else if (rung == kRungSource) {
      r.src = ld->lambda;
      r.max_iter = kLadderItl2 < 100 ? 100u : kLadderItl2;
    }
  }
  if (o.iter_cap && o.iter_cap < r.max_iter) r.max_iter = o.iter_cap;
  return r;
}

// op.zig coldStart's junction seeds into a lane's limited images (diode
// vcrit; MOS1 vgs at its seed, vds 0, vbs -1; BSIM3 vgs at its seed, vds
// 0.1, vbs 0), threads t0, t0 + stride, ... over the instances.
__device__ __forceinline__ void cold_images(const TopoDev& T, const double* rec, double* lim, uint32_t t0,
                                            uint32_t stride) {
  for (uint32_t b = 0; b < T.n_batches; ++b) {
    const BatchDev& B = T.b[b];
    if (B.type == kD)
      for (uint32_t i = t0; i < B.count; i += stride) lim[B.lim_off + i] = rec[B.rec_off + kDVcrit * B.count + i];
    if (B.type == kM)
      for (uint32_t i = t0; i < B.count; i += stride) {
        lim[B.lim_off + 3 * i] = rec[B.rec_off + kMSeedVgs * B.count + i];
        lim[B.lim_off + 3 * i + 1] = 0.0;
        lim[B.lim_off + 3 * i + 2] = -1.0;
      }
    if (B.type == kB3)
      for (uint32_t i = t0; i < B.count; i += stride) {
        lim[B.lim_off + 3 * i] = rec[B.rec_off + kB3SeedVgs * B.count + i];
        lim[B.lim_off + 3 * i + 1] = 0.1;
        lim[B.lim_off + 3 * i + 2] = 0.0;
      }
  }
}

__device__ __forceinline__ uint32_t ladder_sat(uint32_t a, uint32_t b) {
  const uint32_t s = a + b;
  return s > 65535u ? 65535u : s;
}

__device__ __forceinline__ void ladder_sync(uint32_t width) {
  if (width == 32)
    __syncwarp();
  else
    __syncthreads();
}

// Where the ladder's next run starts: the run's own end point, the cold
// start (zero, junction seeds), or the last converged stepping point.
enum LadderStart : uint32_t { kStartKeep = 0, kStartCold = 1, kStartGood = 2 };

// The ladder's step after a run (converged or not, `it` its iterations, 0
// for a singular Jacobian), on the lane's state `s`: the next run's start
// and INITFIX, whether the run's end point becomes the last good point, or
// that the lane is done (result: 0 plain, 1 gmin, 2 source, 3 none; report:
// the plain run's iterations, or the sum over every run once the ladder
// was entered). Pure: every thread of the lane computes the same move.
struct LadderMove {
  uint32_t start;
  bool save, done, init_fix;
  uint32_t result, report;
};

__device__ __forceinline__ LadderMove ladder_decide(LadderDev& s, bool conv, uint32_t it) {
  LadderMove mv{kStartKeep, false, false, false, 3u, 0u};
  bool to_source = false, to_final = false;
  switch (s.rung) {
    case kRungPlain:
      if (conv) {
        mv.done = true;
        mv.result = 0;
        mv.report = it;
        break;
      }
      // rung 2 from the cold start: gmin_start / 10 first
      s.total = it;
      s.rung = kRungGmin;
      s.factor = 10.0;
      s.good_gmin = kLadderGminStart;
      s.gmin_val = div_rn(kLadderGminStart, 10.0);
      s.have_good = 0;
      s.solves = 0;
      mv.start = kStartCold;
      mv.init_fix = true;
      break;
    case kRungGmin:
      s.total = ladder_sat(s.total, it);
      if (conv) {
        if (s.gmin_val <= kLadderGminTarget) {
          // the target reached: one more run without the shunt
          s.rung = kRungClean;
          break;
        }
        mv.save = true;
        s.have_good = 1;
        s.good_gmin = s.gmin_val;
        // an easy step accelerates (capped at 10), a hard one slows down
        if (it <= kLadderItl2 / 4) {
          const double f = s.factor * sqrt(s.factor);
          s.factor = f < 10.0 ? f : 10.0;
        } else if (it > 3 * kLadderItl2 / 4) {
          const double f = sqrt(s.factor);
          s.factor = f > 1.00005 ? f : 1.00005;
        }
        if (s.gmin_val < s.factor * kLadderGminTarget) {
          s.factor = div_rn(s.gmin_val, kLadderGminTarget);
          s.gmin_val = kLadderGminTarget;
        } else {
          s.gmin_val = div_rn(s.gmin_val, s.factor);
        }
      } else {
        if (s.factor < 1.00005) {
          to_source = true;  // wedged against the last good step
          break;
        }
        s.factor = sqrt(sqrt(s.factor));
        s.gmin_val = div_rn(s.good_gmin, s.factor);
        mv.start = s.have_good ? kStartGood : kStartCold;
      }
      if (++s.solves >= 100) {
        to_source = true;  // rung 3 starts cold whatever x holds
        break;
      }
      mv.init_fix = !s.have_good;
      break;
    case kRungClean:
      s.total = ladder_sat(s.total, it);
      if (conv) {
        mv.done = true;
        mv.result = 1;
        mv.report = s.total;
        break;
      }
      to_source = true;
      break;
    case kRungSource:
      s.total = ladder_sat(s.total, it);
      if (conv) {
        if (s.lambda >= 1.0) {
          to_final = true;
          break;
        }
        s.lambda_good = s.lambda;
        mv.save = true;
        s.delta *= 1.5;
        s.lambda = s.lambda + s.delta < 1.0 ? s.lambda + s.delta : 1.0;
      } else {
        s.delta *= 0.5;
        if (s.delta < 1e-4 || s.lambda_good < 0.0) {
          to_final = true;
          break;
        }
        mv.start = kStartGood;
        s.lambda = s.lambda_good + s.delta < 1.0 ? s.lambda_good + s.delta : 1.0;
      }
      if (++s.solves >= 100) {
        to_final = true;  // from x as the last run left it, or the restored good point
        break;
      }
      mv.init_fix = s.lambda_good < 0.0;
      break;
    default:  // kRungFinal
      s.total = ladder_sat(s.total, it);
      mv.done = true;
      mv.result = conv ? 2 : 3;
      mv.report = s.total;
      break;
  }
  if (to_source) {
    // rung 3 from the cold start at lambda = 0
    s.rung = kRungSource;
    s.lambda = 0.0;
    s.lambda_good = -1.0;
    s.delta = 0.25;
    s.solves = 0;
    mv.start = kStartCold;
    mv.init_fix = true;
  }
  if (to_final) {
    // the full-source Newton from where the stepping left x
    s.rung = kRungFinal;
    mv.init_fix = false;
  }
  if (mv.done) s.rung = kRungDone;
  return mv;
}

// The lane's Newton run has ended (status kConverged, kMaxIter or kSingular,
// its end point in L.x): the ladder's next step, by every thread of the
// lane's warp (width 32) or CTA. Returns true when it set up another run
// (status kRunning, its start in L.x and L.lim), false when the lane is
// done (its iterations the move's report, rung_out its result).
static __device__ __noinline__ bool ladder_step(const TopoDev& T, const LaneDev& L, uint32_t lane, int tid,
                                                uint32_t width) {
  ladder_sync(width);
  LadderDev s = L.ladder[lane];
  const uint32_t st = *(volatile uint32_t*)(L.status + lane);
  // a singular Jacobian is a failed run of zero iterations (newtonRun)
  const uint32_t it = st == kSingular ? 0u : *(volatile uint32_t*)(L.iters + lane);
  const LadderMove mv = ladder_decide(s, st == kConverged, it);
  const uint32_t n = T.n;
  double* x = L.x + size_t(lane) * n;
  double* xg = L.x_good + size_t(lane) * n;
  if (mv.save)
    for (uint32_t i = tid; i < n; i += width) xg[i] = x[i];
  if (mv.start == kStartGood)
    for (uint32_t i = tid; i < n; i += width) x[i] = xg[i];
  if (mv.start == kStartCold) {
    for (uint32_t i = tid; i < n; i += width) x[i] = 0.0;
    cold_images(T, L.rec + size_t(lane) * T.rec_size, L.lim + size_t(lane) * T.nlim, tid, width);
  }
  ladder_sync(width);
  if (tid == 0) {
    L.ladder[lane] = s;
    if (mv.done) {
      L.iters[lane] = mv.report;
      if (L.rung_out) L.rung_out[lane] = mv.result;
    } else {
      L.status[lane] = kRunning;
      L.iters[lane] = 0;
      L.flags[lane] = (L.flags[lane] & 2u) | 4u | (mv.init_fix ? 1u : 0u);
      L.lim_active[lane] = mv.start == kStartCold && T.nlim ? 1u : 0u;
      L.limit[lane] = 1e9;
    }
  }
  ladder_sync(width);
  return !mv.done;
}

}  // namespace esl

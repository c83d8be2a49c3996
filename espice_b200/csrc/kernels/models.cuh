// Device-model evaluation on the GPU, one instance per thread, written into
// the instance's staging cells (layout in common.h). Physics restated from
// the reference's Verilog-A sources:
//   models/resistor.va:42-54, capacitor.va:64, vsource.va:131-333,
//   isource.va, diode.va:243-371
// The limiting correction follows src/device/eval.zig:820-877: a limited
// junction is evaluated at its limited voltage and its residual (and charge)
// linearised back to x, f += g * (v - v_lim).
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include "../common.h"

namespace esl {

// a / b correctly rounded (IEEE round-to-nearest), bitwise __ddiv_rn. A zero
// dividend over a finite nonzero divisor (frequent: zero fill-in, zero
// steps, a node at zero volts) returns its signed zero directly, keeping the
// division sequence on its fast path for the operands it is built for.
__device__ __forceinline__ double div_rn(double a, double b) {
  if (a == 0.0 && b != 0.0 && fabs(b) < CUDART_INF)
    return __longlong_as_double((__double_as_longlong(a) ^ __double_as_longlong(b)) & (1ll << 63));
  return __ddiv_rn(a, b);
}

struct SimDev {
  double t;          // time (transient)
  double src_scale;  // source-stepping factor
  int kind;          // 0 static (.op / .dc), 1 transient
};

// PULSE (vsource.va:211-222); p = the 10 V-source fields.
__device__ __forceinline__ double pulse_value(const double* p, int stride, double t) {
  const double v1 = p[2 * stride], v2 = p[3 * stride], td = p[4 * stride];
  const double tr = fmax(p[5 * stride], 1.0e-12);
  const double tf = fmax(p[6 * stride], 1.0e-12);
  const double pwr = p[7 * stride];
  const double pw = fmax(pwr, 0.0) + fmax(-pwr, 0.0) * 1.0e30;
  const double per = fmax(p[8 * stride], tr + pw + tf + 1.0e-12);
  const double t_rel = t - td;
  double t_mod = t_rel + (p[9 * stride] / 360.0) * per;
  t_mod = t_mod - floor(t_mod / per) * per;
  t_mod = fmax(t_mod, 0.0);
  if (t_rel < 0.0) return v1;
  if (t_mod < tr) return v1 + (v2 - v1) * (t_mod / tr);
  if (t_mod < tr + pw) return v2;
  if (t_mod < tr + pw + tf) return v2 - (v2 - v1) * ((t_mod - (tr + pw)) / tf);
  return v1;
}

// V source value: static analyses bias at `dc`; the transient at its wave.
__device__ __forceinline__ double vsource_value(const double* p, int stride, const SimDev& sim) {
  double out = p[0];
  if (sim.kind != 0 && p[stride] == 1.0) out = pulse_value(p, stride, sim.t);
  return out * sim.src_scale;
}

// Junction current and conductance (diode.va:261-318 without ISR/IKF).
__device__ __forceinline__ void diode_iv(const double* r, int s, double vd, double& i, double& g) {
  const double vte = r[kDVte * s], is = r[kDIs * s];
  double id, gd;
  if (vd >= -3.0 * vte) {
    const double u = div_rn(vd, vte);
    const double ulim = fmin(u, 80.0);
    const double e = exp(ulim);
    id = is * ((e * (1.0 + (u - ulim))) - 1.0);
    gd = div_rn(is * e, vte);
  } else {
    const double a = div_rn(3.0 * vte, vd * 2.718281828459045);
    const double a3 = pow(a, 3.0);
    id = -is * (1.0 + a3);
    gd = div_rn(3.0 * is * a3, vd);
  }
  const double xbv = r[kDXbv * s];
  if (r[kDBv * s] > 0.0 && vd < -3.0 * vte && vd < -xbv) {
    const double vtb = r[kDVtebrk * s];
    const double wb = div_rn(-(xbv + vd), vtb);
    const double wlim = fmin(wb, 80.0);
    const double e = exp(wlim);
    id = -is * e * (1.0 + (wb - wlim));
    gd = div_rn(is * e, vtb);
  }
  const double gmin = r[kDGmin * s];
  i = id + gmin * vd;
  g = gd + gmin;
}

// Depletion + diffusion charge and capacitance (diode.va:338-363).
__device__ __forceinline__ void diode_qc(const double* r, int s, double vd, double itot, double gtot,
                                         double& q, double& c) {
  double qj = 0.0, cj = 0.0;
  const double cjo = r[kDCjo * s];
  if (cjo > 0.0) {
    const double vj = r[kDVj * s], mt = r[kDMt * s], fc = r[kDFc * s];
    const double vfc = fc * vj;
    if (vd < vfc) {
      const double b = 1.0 - div_rn(vd, vj);
      qj = div_rn(cjo * vj * (1.0 - pow(b, 1.0 - mt)), 1.0 - mt);
      cj = cjo * pow(b, -mt);
    } else {
      const double f1 = vj * (1.0 - pow(1.0 - fc, 1.0 - mt)) / (1.0 - mt);
      const double f2 = pow(1.0 - fc, 1.0 + mt);
      const double f3 = 1.0 - fc * (1.0 + mt);
      qj = cjo * (f1 + (1.0 / f2) * (f3 * (vd - vfc) + (mt / (2.0 * vj)) * (vd * vd - vfc * vfc)));
      cj = cjo * ((1.0 / f2) * (f3 + (mt / vj) * vd));
    }
  }
  const double tt = r[kDTt * s];
  if (tt > 0.0) {
    qj = qj + tt * itot;
    cj = cj + tt * gtot;
  }
  q = qj;
  c = cj;
}

// pnjlim (ngspice DEVpnjlim as the reference documents it).
__device__ __forceinline__ double pnjlim_dev(double vnew, double vold, double vt, double vcrit, bool& lim) {
  if (vnew > vcrit && fabs(vnew - vold) > vt + vt) {
    if (vold > 0) {
      const double arg = div_rn(vnew - vold, vt);
      if (arg > 0) vnew = vold + vt * (2 + log(arg - 2));
      else vnew = vold - vt * (2 + log(2 - arg));
    } else {
      vnew = vt * log(div_rn(vnew, vt));
    }
    lim = true;
  } else if (vnew < 0) {
    const double arg = vold > 0 ? -1 * vold - 1 : 2 * vold - 1;
    if (vnew < arg) {
      vnew = arg;
      lim = true;
    } else {
      lim = false;
    }
  } else {
    lim = false;
  }
  return vnew;
}

// Diode stamp into its 16 staging cells (a = 0, c = 1, ai = 2).
// `lim` is the instance's limited junction voltage when limiting is live.
__device__ __forceinline__ void diode_stamp(const double* r, int s, double xa, double xc, double xai,
                                            const double* lim, double* st) {
  const double vraw = xai - xc;
  const double ve = lim ? *lim : vraw;
  double i, g;
  diode_iv(r, s, ve, i, g);
  double ires = i;
  double corr = 0.0;
  if (lim) {
    corr = vraw - ve;
    if (corr != 0.0) ires = ires + g * corr;
  }
  const double rs_t = r[kDRs * s];
  const bool has_rs = r[kDHasRs * s] != 0.0;
  const double grs = 1.0 / rs_t;
  const double irs = div_rn(xa - xai, rs_t);
  st[0] = irs;
  st[1] = -ires;
  st[2] = has_rs ? ires - irs : ires;
  st[3] = grs;
  st[4] = -grs;
  st[5] = g;
  st[6] = -g;
  st[7] = -grs;
  st[8] = -g;
  st[9] = has_rs ? g + grs : g;
  if (r[kDHasQ * s] != 0.0) {
    double qj, cj;
    diode_qc(r, s, ve, i, g, qj, cj);
    if (lim && corr != 0.0) qj = qj + cj * corr;
    st[10] = -qj;
    st[11] = qj;
    st[12] = cj;
    st[13] = -cj;
    st[14] = -cj;
    st[15] = cj;
  }
}

}  // namespace esl

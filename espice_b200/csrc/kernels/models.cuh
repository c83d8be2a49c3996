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
#include "../esl_math.h"

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
  int kind;          // 0 static (.op / .dc), 1 transient, 2 transient op
  // $simparam("gmin") read inside an analog block (BSIM3's junction gminx):
  // the gmin-stepping rung's value while it runs, negative for the card's
  double gmin = -1.0;
};

// PULSE (vsource.va:211-222); p = the source's record fields.
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

constexpr double kPiD = 3.141592653589793;
constexpr double kTwoPiD = 6.283185307179586;

// SIN (vsource.va:224-236): before TD the wave's own t = 0 value; the
// damping applies after TD, its exponent clamped at 80. The operations and
// their order are the oracle's (esl_sin / esl_exp are shared with it).
__device__ __forceinline__ double sin_value(const double* p, int s, double t) {
  const double vo = p[2 * s], va = p[3 * s], freq = p[4 * s], td = p[5 * s], theta = p[6 * s], phase = p[7 * s];
  const double t_sin = t - td;
  const double ph = div_rn(phase * kPiD, 180.0);
  if (t_sin < 0.0) return vo + va * esl_sin(ph);
  return vo + va * esl_sin(kTwoPiD * freq * t_sin + ph) * esl_exp(fmin(-theta * t_sin, 80.0));
}

// EXP (vsource.va:238-246): two one-sided exponentials on V1.
__device__ __forceinline__ double exp_value(const double* p, int s, double t) {
  const double v1 = p[2 * s], v2 = p[3 * s], td1 = p[4 * s], tau1 = p[5 * s], td2 = p[6 * s], tau2 = p[7 * s];
  const double t_e1 = t - td1, t_e2 = t - td2;
  double out = v1;
  if (t_e1 > 0.0) out = out + (v2 - v1) * (1.0 - esl_exp(fmin(div_rn(-t_e1, fmax(tau1, 1.0e-15)), 80.0)));
  if (t_e2 > 0.0) out = out + (v1 - v2) * (1.0 - esl_exp(fmin(div_rn(-t_e2, fmax(tau2, 1.0e-15)), 80.0)));
  return out;
}

// PWL (vsource.va:248-290): the repeat wraps [r, t_last]; bisection over the
// sorted times for the segment holding t.
__device__ __forceinline__ double pwl_value(const double* p, int s, double t) {
  const int len = static_cast<int>(p[2 * s]);
  if (len <= 0) return p[0];
  const double repeat = p[3 * s], td = p[4 * s];
  const double* tt = p + kSrcPwlT * s;
  const double* vv = p + kSrcPwlV * s;
  double t_e = t - td;
  const double t_first = tt[0], v_first = vv[0], t_last = tt[(len - 1) * s], v_last = vv[(len - 1) * s];
  if (repeat >= 0.0 && len > 1 && t_e > t_last && t_last > repeat) {
    const double span = t_last - repeat;
    if (span > 0.0) {
      const double excess = t_e - repeat;
      t_e = repeat + (excess - floor(div_rn(excess, span)) * span);
    }
  }
  if (t_e < 0.0 || t_e <= t_first) return v_first;
  if (t_e >= t_last) return v_last;
  int klo = 0, khi = len - 1;
  while (khi - klo > 1) {
    const int k = (klo + khi) / 2;
    if (tt[k * s] > t_e) khi = k;
    else klo = k;
  }
  const double tp = tt[klo * s], vp = vv[klo * s], tk = tt[khi * s], vk = vv[khi * s];
  return vp + div_rn((vk - vp) * (t_e - tp), fmax(tk - tp, 1.0e-15));
}

// A V or I source's value (vsource.va:198-290): static analyses (kind 0)
// bias at `dc`; the transient and its own operating point (kinds 1, 2) at
// the wave; times the source-stepping factor.
__device__ __forceinline__ double source_value(const double* p, int stride, const SimDev& sim) {
  double out = p[0];
  if (sim.kind != 0) {
    const double w = p[stride];
    if (w == 1.0) out = pulse_value(p, stride, sim.t);
    else if (w == 2.0) out = sin_value(p, stride, sim.t);
    else if (w == 3.0) out = exp_value(p, stride, sim.t);
    else if (w == 4.0) out = pwl_value(p, stride, sim.t);
  }
  return out * sim.src_scale;
}

// Junction current and conductance (diode.va:261-318 without ISR/IKF).
__device__ __forceinline__ void diode_iv(const double* r, int s, double vd, double& i, double& g) {
  const double vte = r[kDVte * s], is = r[kDIs * s];
  double id, gd;
  if (vd >= -3.0 * vte) {
    const double u = div_rn(vd, vte);
    const double ulim = fmin(u, 80.0);
    const double e = esl_exp(ulim);
    id = is * ((e * (1.0 + (u - ulim))) - 1.0);
    gd = div_rn(is * e, vte);
  } else {
    const double a = div_rn(3.0 * vte, vd * 2.718281828459045);
    const double a3 = esl_pow(a, 3.0);
    id = -is * (1.0 + a3);
    gd = div_rn(3.0 * is * a3, vd);
  }
  const double xbv = r[kDXbv * s];
  if (r[kDBv * s] > 0.0 && vd < -3.0 * vte && vd < -xbv) {
    const double vtb = r[kDVtebrk * s];
    const double wb = div_rn(-(xbv + vd), vtb);
    const double wlim = fmin(wb, 80.0);
    const double e = esl_exp(wlim);
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
      qj = div_rn(cjo * vj * (1.0 - esl_pow(b, 1.0 - mt)), 1.0 - mt);
      cj = cjo * esl_pow(b, -mt);
    } else {
      const double f1 = vj * (1.0 - esl_pow(1.0 - fc, 1.0 - mt)) / (1.0 - mt);
      const double f2 = esl_pow(1.0 - fc, 1.0 + mt);
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
      if (arg > 0) vnew = vold + vt * (2 + esl_log(arg - 2));
      else vnew = vold - vt * (2 + esl_log(2 - arg));
    } else {
      vnew = vt * esl_log(div_rn(vnew, vt));
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

// ---------------------------------------------------------------------------
// MOS1 (models/mos1.va), type frame: v = type * V. Derivatives hand-written
// in the reference's forward-AD sense; gmbs as ngspice takes it,
// gm * gamma / (2 sarg) on both branches of the body root (mos1.va:316-323).

// DEVfetlim / DEVlimvds (ngspice devsup.c as the reference documents them,
// dev/solvers/newton-raphson-convergence.md:58-69).
__device__ __forceinline__ double fetlim_dev(double vnew, double vold, double vto) {
  const double vtsthi = fabs(2 * (vold - vto)) + 2;
  const double vtstlo = fabs(vold - vto) + 1;
  const double vtox = vto + 3.5;
  const double delv = vnew - vold;
  if (vold >= vto) {
    if (vold >= vtox) {
      if (delv <= 0) {
        if (vnew >= vtox) {
          if (-delv > vtstlo) vnew = vold - vtstlo;
        } else {
          vnew = fmax(vnew, vto + 2);
        }
      } else if (delv >= vtsthi) {
        vnew = vold + vtsthi;
      }
    } else if (delv <= 0) {
      vnew = fmax(vnew, vto - 0.5);
    } else {
      vnew = fmin(vnew, vto + 4);
    }
  } else if (delv <= 0) {
    if (-delv > vtsthi) vnew = vold - vtsthi;
  } else {
    const double vtemp = vto + 0.5;
    if (vnew <= vtemp) {
      if (delv > vtstlo) vnew = vold + vtstlo;
    } else {
      vnew = vtemp;
    }
  }
  return vnew;
}

__device__ __forceinline__ double limvds_dev(double vnew, double vold) {
  if (vold >= 3.5) {
    if (vnew > vold) vnew = fmin(vnew, 3 * vold + 2);
    else if (vnew < 3.5) vnew = fmax(vnew, 2.0);
  } else if (vnew > vold) {
    vnew = fmin(vnew, 4.0);
  } else {
    vnew = fmax(vnew, -0.5);
  }
  return vnew;
}

// jcur (mos1.va:118-129) and its slope.
__device__ __forceinline__ void mos_jcur(double v, double isat, double vtx, double gm, double& i, double& g) {
  if (v > -3.0 * vtx) {
    const double u = fmin(div_rn(v, vtx), 80.0);
    const double e = esl_exp(u);
    i = isat * (e * (1.0 + (div_rn(v, vtx) - u)) - 1.0) + gm * v;
    g = div_rn(isat * e, vtx) + gm;
  } else {
    i = gm * v - isat;
    g = gm;
  }
}

// sbody (mos1.va:131-141); ds = -1 / (2 sarg) where sarg > 0.
__device__ __forceinline__ double mos_sbody(double vbx, double phit, double& ds) {
  double sv;
  if (vbx <= 0.0) sv = sqrt(phit - vbx);
  else sv = fmax(sqrt(phit) - div_rn(vbx, 2.0 * sqrt(phit)), 0.0);
  ds = sv > 0.0 ? div_rn(-1.0, 2.0 * sv) : 0.0;
  return sv;
}

// jchg (mos1.va:143-163) and its capacitance.
__device__ __forceinline__ void mos_jchg(double v, double cz, double czsw, double pbx, double mjx, double mjswx,
                                         double fcx, double f2, double f3, double f4, double& q, double& c) {
  if (cz == 0.0 && czsw == 0.0) {
    q = 0.0;
    c = 0.0;
  } else if (v < fcx * pbx) {
    const double a = 1.0 - div_rn(v, pbx);
    q = pbx * (div_rn(cz * (1.0 - esl_pow(a, 1.0 - mjx)), 1.0 - mjx) + div_rn(czsw * (1.0 - esl_pow(a, 1.0 - mjswx)), 1.0 - mjswx));
    c = cz * esl_pow(a, -mjx) + czsw * esl_pow(a, -mjswx);
  } else {
    q = f4 + v * (f2 + 0.5 * f3 * v);
    c = f2 + f3 * v;
  }
}

// MOS1 stamp into its 40 staging cells (layout in common.h). `lim` is the
// instance's three images (vgs, vds, vbs) when limiting is live; the
// charges are written for a transient (`dyn`) when the instance has any.
__device__ __forceinline__ void mos1_stamp(const double* r, int s, double xd, double xg, double xs, double xb,
                                           double xdi, double xsi, const double* lim, bool dyn, double* st) {
  const double type = r[kMType * s], vt = r[kMVt * s];
  const double vgs_r = type * (xg - xsi), vds_r = type * (xdi - xsi), vbs_r = type * (xb - xsi);
  const double vgs = lim ? lim[0] : vgs_r, vds = lim ? lim[1] : vds_r, vbs = lim ? lim[2] : vbs_r;
  const double vbd = vbs - vds, vgd = vgs - vds;
  double ibs, gbs, ibd, gbd;
  mos_jcur(vbs, r[kMIsats * s], vt, r[kMGmin * s], ibs, gbs);
  mos_jcur(vbd, r[kMIsatd * s], vt, r[kMGmin * s], ibd, gbd);
  const double mode = vds >= 0.0 ? 1.0 : -1.0;
  const double vbx = mode > 0 ? vbs : vbd;
  const double vgsx = mode > 0 ? vgs : vgd;
  const double vdsx = mode * vds;
  double ds;
  const double gamma = r[kMGamma * s];
  const double sarg = mos_sbody(vbx, r[kMPhit * s], ds);
  const double von = r[kMVbit * s] * type + gamma * sarg;
  const double vgst = vgsx - von;
  const double beta = r[kMBeta * s], lambda = r[kMLambda * s];
  const double bp = beta * (1.0 + lambda * vdsx);
  double id = 0.0, gm = 0.0, gds = 0.0;
  if (vgst <= 0.0) {
    id = 0.0;
  } else if (vgst <= vdsx) {
    id = 0.5 * bp * vgst * vgst;
    gm = bp * vgst;
    gds = 0.5 * beta * lambda * vgst * vgst;
  } else {
    id = bp * vdsx * (vgst - 0.5 * vdsx);
    gm = bp * vdsx;
    gds = beta * lambda * vdsx * (vgst - 0.5 * vdsx) + bp * (vgst - vdsx);
  }
  const double gmbs = gm * (-gamma * ds);
  double ich, gmg, gdd, gbb;
  if (mode > 0) {
    ich = id;
    gmg = gm;
    gdd = gds;
    gbb = gmbs;
  } else {
    ich = -id;
    gmg = -gm;
    gbb = -gmbs;
    gdd = gm + gds + gmbs;
  }
  const double cgs_ = vgs_r - vgs, cds = vds_r - vds, cbs = vbs_r - vbs;
  const double cbd = (vbs_r - vds_r) - vbd;
  if (lim) {
    if (cgs_ != 0.0 || cds != 0.0 || cbs != 0.0) ich = ich + (gmg * cgs_ + gdd * cds + gbb * cbs);
    if (cbs != 0.0) ibs = ibs + gbs * cbs;
    if (cbd != 0.0) ibd = ibd + gbd * cbd;
  }
  const double ids = type * ich, tbs = type * ibs, tbd = type * ibd;
  const double gdr = r[kMGdrain * s], gsr = r[kMGsource * s];
  const double idr = gdr * (xd - xdi), isr = gsr * (xs - xsi);
  const double gsum = gmg + gdd + gbb;
  st[0] = idr;
  st[1] = isr;
  st[2] = tbd + tbs;
  st[3] = (ids - tbd) - idr;
  st[4] = ((-ids) - tbs) - isr;
  st[5] = gdr;
  st[6] = -gdr;
  st[7] = gsr;
  st[8] = -gsr;
  st[9] = gbd + gbs;
  st[10] = -gbd;
  st[11] = -gbs;
  st[12] = -gdr;
  st[13] = gmg;
  st[14] = gbb - gbd;
  st[15] = (gdd + gbd) + gdr;
  st[16] = -gsum;
  st[17] = -gmg;
  st[18] = -gsr;
  st[19] = (-gbb) - gbs;
  st[20] = -gdd;
  st[21] = (gsum + gbs) + gsr;
  if (dyn && r[kMHasQ * s] != 0.0) {
    double qbd, cbdc, qbs, cbsc;
    const double pbt = r[kMPbt * s], mj = r[kMMj * s], mjsw = r[kMMjsw * s], fc = r[kMFc * s];
    mos_jchg(vbd, r[kMCzbd * s], r[kMCzbdsw * s], pbt, mj, mjsw, fc, r[kMF2d * s], r[kMF3d * s], r[kMF4d * s], qbd, cbdc);
    mos_jchg(vbs, r[kMCzbs * s], r[kMCzbssw * s], pbt, mj, mjsw, fc, r[kMF2s * s], r[kMF3s * s], r[kMF4s * s], qbs, cbsc);
    if (lim) {
      if (cbd != 0.0) qbd = qbd + cbdc * cbd;
      if (cbs != 0.0) qbs = qbs + cbsc * cbs;
    }
    const double cgs = r[kMCgs * s], cgd = r[kMCgd * s], cgb = r[kMCgb * s];
    const double qgs = cgs * (xg - xsi), qgd = cgd * (xg - xdi), qgb = cgb * (xg - xb);
    const double tqbd = type * qbd, tqbs = type * qbs;
    st[22] = (qgs + qgd) + qgb;
    st[23] = (tqbd + tqbs) - qgb;
    st[24] = (-tqbd) - qgd;
    st[25] = (-tqbs) - qgs;
    st[26] = (cgs + cgd) + cgb;
    st[27] = -cgb;
    st[28] = -cgd;
    st[29] = -cgs;
    st[30] = -cgb;
    st[31] = (cbdc + cbsc) + cgb;
    st[32] = -cbdc;
    st[33] = -cbsc;
    st[34] = -cgd;
    st[35] = -cbdc;
    st[36] = cbdc + cgd;
    st[37] = -cgs;
    st[38] = -cbsc;
    st[39] = cbsc + cgs;
  }
}

// The MOS1 limiting ladder (mos1load.c:361-384) against `old` (images, or
// x_old's voltages before the first pass), writing the three images; true
// when pnjlim limited. Images within 16 ulps of the raw value snap to it.
__device__ __forceinline__ bool mos1_limit(const double* r, int s, double xg, double xb, double xdi, double xsi,
                                           const double* old, double* img) {
  const double type = r[kMType * s], vt = r[kMVt * s];
  const double vgs_n = type * (xg - xsi), vds_n = type * (xdi - xsi), vbs_n = type * (xb - xsi);
  const double vgd_n = type * (xg - xdi), vbd_n = type * (xb - xdi);
  const double vgs_o = old[0], vds_o = old[1], vbs_o = old[2];
  const double vgd_o = vgs_o - vds_o, vbd_o = vbs_o - vds_o;
  const double vbx = vds_o >= 0.0 ? vbs_o : vbd_o;
  double ds;
  const double von = r[kMVbit * s] * type + r[kMGamma * s] * mos_sbody(vbx, r[kMPhit * s], ds);
  double vgs, vds, vbs;
  if (vds_o >= 0.0) {
    vgs = fetlim_dev(vgs_n, vgs_o, von);
    vds = vgs - vgd_n;
    vds = limvds_dev(vds, vds_o);
  } else {
    const double vgd = fetlim_dev(vgd_n, vgd_o, von);
    vds = vgs_n - vgd;
    vds = -limvds_dev(-vds, -vds_o);
    vgs = vgd + vds;
  }
  bool l = false;
  if (vds >= 0.0) {
    vbs = pnjlim_dev(vbs_n, vbs_o, vt, r[kMVcrits * s], l);
  } else {
    const double vbd = pnjlim_dev(vbd_n, vbd_o, vt, r[kMVcritd * s], l);
    vbs = vbd + vds;
  }
  const double scale = fmax(fmax(fabs(xg), fabs(xb)), fmax(fabs(xdi), fabs(xsi)));
  const double tol = 16.0 * 2.220446049250313e-16 * scale;
  if (fabs(vgs - vgs_n) <= tol) vgs = vgs_n;
  if (fabs(vds - vds_n) <= tol) vds = vds_n;
  if (fabs(vbs - vbs_n) <= tol) vbs = vbs_n;
  img[0] = vgs;
  img[1] = vds;
  img[2] = vbs;
  return l;
}

}  // namespace esl

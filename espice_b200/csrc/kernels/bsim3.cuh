// BSIM3v3.3 DC core on the GPU, restated from models/bsim3.va: the
// bias-dependent chain of b3ld.c (:399-611) and the contributions
// (:613-624), on the bias-independent record the host derives (b3temp.c,
// :186-346). The model has no charges (capMod is not built), as in the
// reference.
//
// Derivatives: the reference differentiates the value chain by VerA's
// forward AD; here every bias-dependent quantity is a dual number carrying
// its partials in the type-frame (vgs, vds, vbs) images. Divisions are
// correctly rounded and the build keeps multiply-adds unfused, so the chain
// rounds as the host restatement does (exp, log and sqrt are CUDA's).
#pragma once

#include "models.cuh"

namespace esl {

struct Dual {
  double v, g, d, b;
};

__device__ __forceinline__ Dual dk(double c) { return {c, 0.0, 0.0, 0.0}; }
__device__ __forceinline__ Dual dadd(Dual a, Dual b) { return {a.v + b.v, a.g + b.g, a.d + b.d, a.b + b.b}; }
__device__ __forceinline__ Dual dsub(Dual a, Dual b) { return {a.v - b.v, a.g - b.g, a.d - b.d, a.b - b.b}; }
__device__ __forceinline__ Dual dneg(Dual a) { return {-a.v, -a.g, -a.d, -a.b}; }
__device__ __forceinline__ Dual dmul(Dual a, Dual b) {
  return {a.v * b.v, a.g * b.v + a.v * b.g, a.d * b.v + a.v * b.d, a.b * b.v + a.v * b.b};
}
// a * c, c a constant
__device__ __forceinline__ Dual dscl(Dual a, double c) { return {a.v * c, a.g * c, a.d * c, a.b * c}; }
__device__ __forceinline__ Dual ddiv(Dual a, Dual b) {
  const double q = div_rn(a.v, b.v);
  return {q, div_rn(a.g - q * b.g, b.v), div_rn(a.d - q * b.d, b.v), div_rn(a.b - q * b.b, b.v)};
}
// a / c, c a constant
__device__ __forceinline__ Dual ddivk(Dual a, double c) {
  return {div_rn(a.v, c), div_rn(a.g, c), div_rn(a.d, c), div_rn(a.b, c)};
}
// c / b, c a constant
__device__ __forceinline__ Dual dkdiv(double c, Dual b) {
  const double q = div_rn(c, b.v);
  const double s = div_rn(-q, b.v);
  return {q, s * b.g, s * b.d, s * b.b};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const double s = sqrt(a.v);
  const double h = div_rn(0.5, s);
  return {s, a.g * h, a.d * h, a.b * h};
}
__device__ __forceinline__ Dual dexp(Dual a) {
  const double e = esl_exp(a.v);
  return {e, a.g * e, a.d * e, a.b * e};
}
__device__ __forceinline__ Dual dlog(Dual a) {
  return {esl_log(a.v), div_rn(a.g, a.v), div_rn(a.d, a.v), div_rn(a.b, a.v)};
}
// a + c and c - a, c a constant
__device__ __forceinline__ Dual daddk(Dual a, double c) { return {a.v + c, a.g, a.d, a.b}; }
__device__ __forceinline__ Dual dksub(double c, Dual a) { return {c - a.v, -a.g, -a.d, -a.b}; }

__device__ __forceinline__ void b3_channel(const double* r, int s, Dual vgsx, Dual vdsx, Dual vbsx, Dual& id_out,
                                           Dual& isub_out) {
  auto F = [&](int f) { return r[f * s]; };
  const double vt = F(kB3Vt), phi = F(kB3Phi), sqrtphi = F(kB3Sqrtphi), vbsc = F(kB3Vbsc);
  const double leff = F(kB3Leff), weff = F(kB3Weff), tox = F(kB3Tox), cox = F(kB3Cox);
  const double type = F(kB3Type);
  Dual t0, t1, t2, t3, t4, t5, t6, t7, t8, t9, t10, t11, tmp1, tmp2, tmp3, tmp4;

  // Vbseff, Phis, Xdep
  t0 = daddk(daddk(vbsx, -vbsc), -0.001);
  t1 = dsqrt(dsub(dmul(t0, t0), dk(0.004 * vbsc)));
  Dual vbseff = daddk(dscl(dadd(t0, t1), 0.5), vbsc);
  if (vbseff.v < vbsx.v) vbseff = vbsx;
  Dual phis, sqrtphis;
  if (vbseff.v > 0.0) {
    t0 = dkdiv(phi, daddk(vbseff, phi));
    phis = dscl(t0, phi);
    sqrtphis = dkdiv(F(kB3Phis3), daddk(dscl(vbseff, 0.5), phi));
  } else {
    phis = dksub(phi, vbseff);
    sqrtphis = dsqrt(phis);
  }
  Dual xdep = ddivk(dscl(sqrtphis, F(kB3Xdep0)), sqrtphi);

  // Vth
  t3 = dsqrt(xdep);
  t0 = dscl(vbseff, F(kB3Dvt2));
  if (t0.v >= -0.5) t1 = daddk(t0, 1.0);
  else t1 = ddiv(daddk(dscl(t0, 3.0), 1.0), daddk(dscl(t0, 8.0), 3.0));
  Dual lt1 = dmul(dscl(t3, F(kB3Factor1)), t1);
  t0 = dscl(vbseff, F(kB3Dvt2w));
  if (t0.v >= -0.5) t1 = daddk(t0, 1.0);
  else t1 = ddiv(daddk(dscl(t0, 3.0), 1.0), daddk(dscl(t0, 8.0), 3.0));
  Dual ltw = dmul(dscl(t3, F(kB3Factor1)), t1);

  t0 = dkdiv(-0.5 * F(kB3Dvt1) * leff, lt1);
  if (t0.v > -34.0) t1 = dexp(t0);
  else t1 = dk(1.713908431e-15);
  Dual theta0 = dmul(t1, daddk(dscl(t1, 2.0), 1.0));
  Dual deltvth = dscl(dscl(theta0, F(kB3Dvt0)), F(kB3Vbi) - phi);

  t0 = dkdiv(-0.5 * F(kB3Dvt1w) * weff * leff, ltw);
  if (t0.v > -34.0) t1 = dexp(t0);
  else t1 = dk(1.713908431e-15);
  Dual dvthw = dscl(dmul(dscl(t1, F(kB3Dvt0w)), daddk(dscl(t1, 2.0), 1.0)), F(kB3Vbi) - phi);

  const double tempratio = F(kB3Tratio1);
  const double nlxt = sqrt(1.0 + F(kB3Nlx) / leff);
  t5 = daddk(dscl(daddk(dscl(vbseff, F(kB3Kt2)), F(kB3Kt1) + F(kB3Kt1l) / leff), tempratio),
       F(kB3K1ox) * (nlxt - 1.0) * sqrtphi);
  const double tmp2k = tox * phi / (weff + F(kB3W0));

  t3 = daddk(dscl(vbseff, F(kB3Etab)), F(kB3Eta0));
  if (t3.v < 1.0e-4) t3 = ddiv(dksub(2.0e-4, t3), dksub(3.0, dscl(t3, 2.0e4)));
  Dual diblsft = dmul(dscl(t3, F(kB3Theta0vb0)), vdsx);

  Dual vth = dk(type * F(kB3Vth0i) - F(kB3K1x) * sqrtphi);
  vth = dadd(vth, dscl(sqrtphis, F(kB3K1ox)));
  vth = dsub(vth, dscl(vbseff, F(kB3K2ox)));
  vth = dsub(vth, deltvth);
  vth = dsub(vth, dvthw);
  vth = dadd(vth, dscl(daddk(dscl(vbseff, F(kB3K3b)), F(kB3K3)), tmp2k));
  vth = dadd(vth, t5);
  vth = dsub(vth, diblsft);

  // n, the subthreshold swing
  tmp2 = dkdiv(F(kB3Nfactor) * 1.03594e-10, xdep);
  tmp3 = dadd(daddk(dscl(vbseff, F(kB3Cdscb)), F(kB3Cdsc)), dscl(vdsx, F(kB3Cdscd)));
  tmp4 = ddivk(daddk(dadd(tmp2, dmul(tmp3, theta0)), F(kB3Cit)), cox);
  Dual n;
  if (tmp4.v >= -0.5) n = daddk(tmp4, 1.0);
  else n = ddiv(daddk(dscl(tmp4, 3.0), 1.0), daddk(dscl(tmp4, 8.0), 3.0));

  // poly gate depletion, Vgsteff
  const double vfbphi = F(kB3Vfbi) + phi;
  const double ngatex = F(kB3Ngate);
  Dual vgs_eff;
  if (ngatex > 1.0e18 && ngatex < 1.0e25 && vgsx.v > vfbphi) {
    const double k = 1.0e6 * 1.60219e-19 * 1.03594e-10 * ngatex / (cox * cox);
    t4 = dsqrt(daddk(ddivk(dscl(daddk(vgsx, -vfbphi), 2.0), k), 1.0));
    t2 = dscl(daddk(t4, -1.0), k);
    t3 = ddivk(dscl(dmul(t2, t2), 0.5), k);
    t7 = daddk(dksub(1.12, t3), -0.05);
    t6 = dsqrt(daddk(dmul(t7, t7), 0.224));
    vgs_eff = dsub(vgsx, dksub(1.12, dscl(dadd(t7, t6), 0.5)));
  } else {
    vgs_eff = vgsx;
  }
  Dual vgst = dsub(vgs_eff, vth);

  t10 = dscl(n, 2.0 * vt);
  t11 = ddiv(vgst, t10);
  t9 = ddiv(dksub(2.0 * F(kB3Voff), vgst), t10);
  Dual vgsteff;
  if (t11.v > 34.0) {
    vgsteff = vgst;
  } else if (t9.v > 34.0) {
    t0 = ddiv(daddk(vgst, -F(kB3Voff)), dscl(n, vt));
    vgsteff = dscl(dexp(t0), vt * F(kB3Cdep0) / cox);
  } else {
    Dual expvgst = dexp(t11);
    t1 = dmul(t10, dlog(daddk(expvgst, 1.0)));
    t2 = daddk(dmul(ddivk(dscl(t10, cox), vt * F(kB3Cdep0)), dexp(t9)), 1.0);
    vgsteff = ddiv(t1, t2);
  }

  // Weff', Rds, Abulk
  t9 = daddk(sqrtphis, -sqrtphi);
  Dual weffp = dksub(weff, dscl(dadd(dscl(vgsteff, F(kB3Dwg)), dscl(t9, F(kB3Dwb))), 2.0));
  if (weffp.v < 2.0e-8) weffp = ddiv(dscl(dksub(4.0e-8, weffp), 2.0e-8), dksub(6.0e-8, dscl(weffp, 2.0)));
  t0 = dadd(dscl(vgsteff, F(kB3Prwg)), dscl(t9, F(kB3Prwb)));
  Dual rds;
  if (t0.v >= -0.9) rds = dscl(daddk(t0, 1.0), F(kB3Rds0));
  else rds = ddiv(dscl(daddk(t0, 0.8), F(kB3Rds0)), daddk(dscl(t0, 20.0), 17.0));

  t1 = dkdiv(0.5 * F(kB3K1ox), sqrtphis);
  t9 = dsqrt(dscl(xdep, F(kB3Xj)));
  tmp1 = daddk(dscl(t9, 2.0), leff);
  t5 = dkdiv(leff, tmp1);
  tmp2 = dscl(t5, F(kB3A0));
  const double tmp4k = F(kB3B0) / (weff + F(kB3B1));
  t2 = daddk(tmp2, tmp4k);
  t6 = dmul(t5, t5);
  t7 = dmul(t5, t6);
  Dual abulk0 = daddk(dmul(t1, t2), 1.0);
  t8 = dscl(t7, F(kB3Ags) * F(kB3A0));
  Dual abulk = dsub(abulk0, dmul(dmul(t1, t8), vgsteff));
  if (abulk0.v < 0.1) abulk0 = ddiv(dksub(0.2, abulk0), dksub(3.0, dscl(abulk0, 20.0)));
  if (abulk.v < 0.1) abulk = ddiv(dksub(0.2, abulk), dksub(3.0, dscl(abulk, 20.0)));
  t2 = dscl(vbseff, F(kB3Keta));
  if (t2.v >= -0.9) t0 = dkdiv(1.0, daddk(t2, 1.0));
  else t0 = ddiv(daddk(dscl(t2, 20.0), 17.0), daddk(t2, 0.8));
  abulk = dmul(abulk, t0);
  abulk0 = dmul(abulk0, t0);

  // mobility
  const int mobmod = static_cast<int>(F(kB3Mobmod));
  if (mobmod == 1) {
    t0 = dadd(dadd(vgsteff, vth), vth);
    t2 = daddk(dscl(vbseff, F(kB3Uc)), F(kB3Ua));
    t3 = ddivk(t0, tox);
    t5 = dmul(t3, dadd(t2, dscl(t3, F(kB3Ub))));
  } else if (mobmod == 2) {
    t5 = dmul(ddivk(vgsteff, tox),
         dadd(daddk(dscl(vbseff, F(kB3Uc)), F(kB3Ua)), ddivk(dscl(vgsteff, F(kB3Ub)), tox)));
  } else {
    t0 = dadd(dadd(vgsteff, vth), vth);
    t2 = daddk(dscl(vbseff, F(kB3Uc)), 1.0);
    t3 = ddivk(t0, tox);
    t4 = dmul(t3, daddk(dscl(t3, F(kB3Ub)), F(kB3Ua)));
    t5 = dmul(t4, t2);
  }
  Dual denomi;
  if (t5.v >= -0.8) denomi = daddk(t5, 1.0);
  else denomi = ddiv(daddk(t5, 0.6), daddk(dscl(t5, 10.0), 7.0));
  Dual ueff = dkdiv(F(kB3U0temp), denomi);

  // Esat, Lambda, Vdsat
  const double vsattemp = F(kB3Vsattemp);
  Dual wvcox = dscl(dscl(weffp, vsattemp), cox);
  Dual wvcoxrds = dmul(wvcox, rds);
  Dual esat = dkdiv(2.0 * vsattemp, ueff);
  Dual esatl = dscl(esat, leff);
  const double a1 = F(kB3A1), a2 = F(kB3A2);
  Dual lambda;
  if (a1 == 0.0) {
    lambda = dk(a2);
  } else if (a1 > 0.0) {
    const double c0 = 1.0 - a2;
    t1 = daddk(dksub(c0, dscl(vgsteff, a1)), -0.0001);
    t2 = dsqrt(daddk(dmul(t1, t1), 0.0004 * c0));
    lambda = dksub(a2 + c0, dscl(dadd(t1, t2), 0.5));
  } else {
    t1 = daddk(daddk(dscl(vgsteff, a1), a2), -0.0001);
    t2 = dsqrt(daddk(dmul(t1, t1), 0.0004 * a2));
    lambda = dscl(dadd(t1, t2), 0.5);
  }
  Dual vgst2vtm = daddk(vgsteff, 2.0 * vt);
  Dual vdsat;
  if (rds.v == 0.0 && lambda.v == 1.0) {
    vdsat = ddiv(dmul(esatl, vgst2vtm), dadd(dmul(abulk, esatl), vgst2vtm));
  } else {
    t9 = dmul(abulk, wvcoxrds);
    t7 = dmul(vgst2vtm, t9);
    t6 = dmul(vgst2vtm, wvcoxrds);
    t0 = dscl(dmul(abulk, dadd(daddk(t9, -1.0), dkdiv(1.0, lambda))), 2.0);
    t1 = dadd(dadd(dmul(vgst2vtm, daddk(dkdiv(2.0, lambda), -1.0)), dmul(abulk, esatl)), dscl(t7, 3.0));
    t2 = dmul(vgst2vtm, dadd(esatl, dscl(t6, 2.0)));
    t3 = dsqrt(dsub(dmul(t1, t1), dmul(dscl(t0, 2.0), t2)));
    vdsat = ddiv(dsub(t1, t3), t0);
  }

  // Vdseff
  const double delta = F(kB3Delta);
  t1 = daddk(dsub(vdsat, vdsx), -delta);
  t2 = dsqrt(dadd(dmul(t1, t1), dscl(vdsat, 4.0 * delta)));
  Dual vdseff = dsub(vdsat, dscl(dadd(t1, t2), 0.5));
  if (vdsx.v == 0.0) vdseff = dk(0.0);

  // VAsat (from Vdsat and the unclamped Vdseff)
  tmp4 = dksub(1.0, ddiv(dscl(dmul(abulk, vdsat), 0.5), vgst2vtm));
  t9 = dmul(wvcoxrds, vgsteff);
  t0 = dadd(dadd(esatl, vdsat), dmul(dscl(t9, 2.0), tmp4));
  t9 = dmul(wvcoxrds, abulk);
  t1 = dadd(daddk(dkdiv(2.0, lambda), -1.0), t9);
  Dual vasat = ddiv(t0, t1);
  if (vdseff.v > vdsx.v) vdseff = vdsx;
  Dual diffvds = dsub(vdsx, vdseff);

  // VACLM, VADIBL, VA, VASCBE
  const double pclm = F(kB3Pclm), litl = F(kB3Litl);
  Dual vaclm;
  if (pclm > 0.0 && diffvds.v > 1.0e-10) {
    t0 = dkdiv(1.0, dscl(dscl(abulk, pclm), litl));
    t2 = ddiv(vgsteff, esatl);
    t1 = dscl(dadd(abulk, t2), leff);
    vaclm = dmul(dmul(t0, t1), diffvds);
  } else {
    vaclm = dk(5.834617425e14);
  }
  const double thetarout = F(kB3Thetarout);
  Dual vadibl;
  if (thetarout > 0.0) {
    t8 = dmul(abulk, vdsat);
    t0 = dmul(vgst2vtm, t8);
    t1 = dadd(vgst2vtm, t8);
    vadibl = ddivk(dsub(vgst2vtm, ddiv(t0, t1)), thetarout);
    t7 = dscl(vbseff, F(kB3Pdiblcb));
    if (t7.v >= -0.9) vadibl = ddiv(vadibl, daddk(t7, 1.0));
    else vadibl = ddiv(dmul(vadibl, daddk(dscl(t7, 20.0), 17.0)), daddk(t7, 0.8));
  } else {
    vadibl = dk(5.834617425e14);
  }
  t8 = dkdiv(F(kB3Pvag), esatl);
  t9 = dmul(t8, vgsteff);
  if (t9.v > -0.9) t0 = daddk(t9, 1.0);
  else t0 = ddiv(daddk(t9, 0.8), daddk(dscl(t9, 20.0), 17.0));
  t1 = ddiv(dmul(vaclm, vadibl), dadd(vaclm, vadibl));
  Dual va = dadd(vasat, dmul(t0, t1));
  const double pscbe1 = F(kB3Pscbe1), pscbe2 = F(kB3Pscbe2);
  Dual vascbe;
  if (pscbe2 > 0.0) {
    if (diffvds.v > pscbe1 * litl / 34.0)
      vascbe = ddivk(dscl(dexp(dkdiv(pscbe1 * litl, diffvds)), leff), pscbe2);
    else
      vascbe = dk(5.834617425e14 * leff / pscbe2);
  } else {
    vascbe = dk(5.834617425e14);
  }

  // Ids chain
  Dual betax = ddivk(dmul(dscl(ueff, cox), weffp), leff);
  Dual fgche1 = dmul(vgsteff, dksub(1.0, ddiv(dscl(dmul(abulk, vdseff), 0.5), vgst2vtm)));
  Dual fgche2 = daddk(ddiv(vdseff, esatl), 1.0);
  Dual gche = ddiv(dmul(betax, fgche1), fgche2);
  Dual idl = ddiv(dmul(gche, vdseff), daddk(dmul(gche, rds), 1.0));
  Dual idsa = dmul(idl, daddk(ddiv(diffvds, va), 1.0));
  id_out = dmul(idsa, daddk(ddiv(diffvds, vascbe), 1.0));

  // substrate (impact ionisation) current
  const double tmp1k = F(kB3Alpha0) + F(kB3Alpha1) * leff;
  const double beta0 = F(kB3Beta0);
  if (tmp1k <= 0.0 || beta0 <= 0.0) {
    isub_out = dk(0.0);
  } else {
    const double t2k = tmp1k / leff;
    if (diffvds.v > beta0 / 34.0)
      t1 = dmul(dscl(diffvds, t2k), dexp(dkdiv(-beta0, diffvds)));
    else
      t1 = dscl(diffvds, t2k * 1.713908431e-15);
    isub_out = dmul(t1, idsa);
  }
}

// jcur (bsim3.va:166-184), linearised above vjm when IJTH > 0, with its slope.
__device__ __forceinline__ void b3_jcur(double v, double isat, double nvt, double vjm, double isevjm, double ijth,
                                        double gmin, double& i, double& g) {
  if (isat <= 0.0) {
    i = gmin * v;
    g = gmin;
  } else if (ijth > 0.0 && v >= vjm) {
    i = isevjm - isat + div_rn(isevjm, nvt) * (v - vjm) + gmin * v;
    g = div_rn(isevjm, nvt) + gmin;
  } else {
    const double u = fmin(div_rn(v, nvt), 80.0);
    const double e = esl_exp(u);
    i = isat * (e * (1.0 + (div_rn(v, nvt) - u)) - 1.0) + gmin * v;
    g = div_rn(isat * e, nvt) + gmin;
  }
}

// BSIM3 stamp into its 23 staging cells (layout in common.h). `lim` is the
// instance's three images (vgs, vds, vbs) when limiting is live; a limited
// instance is linearised back to x. `gmin` >= 0 replaces the card's junction
// gmin (the gmin-stepping rung).
static __device__ __noinline__ void bsim3_stamp(const double* r, int s, double xd, double xg, double xs, double xb,
                                         double xdi, double xsi, const double* lim, double* st, double gmin) {
  auto F = [&](int f) { return r[f * s]; };
  const double type = F(kB3Type), m = F(kB3M);
  const double vgs_r = type * (xg - xsi), vds_r = type * (xdi - xsi), vbs_r = type * (xb - xsi);
  const Dual vgs = {lim ? lim[0] : vgs_r, 1.0, 0.0, 0.0};
  const Dual vds = {lim ? lim[1] : vds_r, 0.0, 1.0, 0.0};
  const Dual vbs = {lim ? lim[2] : vbs_r, 0.0, 0.0, 1.0};
  const Dual vgd = dsub(vgs, vds), vbd = dsub(vbs, vds);
  // gminx = $simparam("gmin", 1e-12) (bsim3.va:353): the stepping rung's
  // gmin while it runs, else the card's
  if (!(gmin >= 0.0)) gmin = F(kB3Gmin);
  double ibs, gbs, ibd, gbd;
  b3_jcur(vbs.v, F(kB3Isats), F(kB3Nvtmj), F(kB3Vjsm), F(kB3Isevjsm), F(kB3Ijth), gmin, ibs, gbs);
  b3_jcur(vbd.v, F(kB3Isatd), F(kB3Nvtmj), F(kB3Vjdm), F(kB3Isevjdm), F(kB3Ijth), gmin, ibd, gbd);
  const bool fwd = vds.v >= 0.0;
  Dual id, isub;
  b3_channel(r, s, fwd ? vgs : vgd, fwd ? vds : dneg(vds), fwd ? vbs : vbd, id, isub);
  // channel current di -> si and substrate current, times m
  const Dual ich = dscl(fwd ? id : dneg(id), m);
  const Dual isb = dscl(isub, m);
  ibs = m * ibs;
  gbs = m * gbs;
  ibd = m * ibd;
  gbd = m * gbd;
  double ichv = ich.v, isbv = isb.v;
  if (lim) {
    const double cgs = vgs_r - vgs.v, cds = vds_r - vds.v, cbs = vbs_r - vbs.v;
    const double cbd = (vbs_r - vds_r) - vbd.v;
    if (cgs != 0.0 || cds != 0.0 || cbs != 0.0) {
      ichv = ichv + (ich.g * cgs + ich.d * cds + ich.b * cbs);
      isbv = isbv + (isb.g * cgs + isb.d * cds + isb.b * cbs);
    }
    if (cbs != 0.0) ibs = ibs + gbs * cbs;
    if (cbd != 0.0) ibd = ibd + gbd * cbd;
  }
  const double ids = type * ichv, tsub = type * isbv, tbs = type * ibs, tbd = type * ibd;
  const double gdr = F(kB3Gdrain), gsr = F(kB3Gsource);
  const double idr = gdr * (xd - xdi), isr = gsr * (xs - xsi);
  const double csum = (ich.g + ich.d) + ich.b, ssum = (isb.g + isb.d) + isb.b;
  // the substrate current leaves the channel end that is the drain in the
  // swapped frame: di forward, si reversed
  double f4 = (ids - tbd) - idr, f5 = ((-ids) - tbs) - isr;
  double j41 = ich.g, j43 = ich.b - gbd, j44 = (ich.d + gbd) + gdr, j45 = -csum;
  double j51 = -ich.g, j53 = (-ich.b) - gbs, j54 = -ich.d, j55 = (csum + gbs) + gsr;
  if (fwd) {
    f4 = f4 + tsub;
    j41 = j41 + isb.g;
    j43 = j43 + isb.b;
    j44 = j44 + isb.d;
    j45 = j45 - ssum;
  } else {
    f5 = f5 + tsub;
    j51 = j51 + isb.g;
    j53 = j53 + isb.b;
    j54 = j54 + isb.d;
    j55 = j55 - ssum;
  }
  st[0] = idr;
  st[1] = isr;
  st[2] = (tbd + tbs) - tsub;
  st[3] = f4;
  st[4] = f5;
  st[5] = gdr;
  st[6] = -gdr;
  st[7] = gsr;
  st[8] = -gsr;
  st[9] = -isb.g;
  st[10] = (gbd + gbs) - isb.b;
  st[11] = (-gbd) - isb.d;
  st[12] = ssum - gbs;
  st[13] = -gdr;
  st[14] = j41;
  st[15] = j43;
  st[16] = j44;
  st[17] = j45;
  st[18] = j51;
  st[19] = -gsr;
  st[20] = j53;
  st[21] = j54;
  st[22] = j55;
}

// The limiting ladder (bsim3.va:378-397): the MOS1 ladder with fetlim's
// threshold the zero-bias type*vth0i and pnjlim at the 300.15 K vt0 and its
// vcrit, against `old` (images, or x_old's voltages before the first
// pass); true when pnjlim limited. Images within 16 ulps of the raw value
// snap to it.
static __device__ __noinline__ bool bsim3_limit(const double* r, int s, double xg, double xb, double xdi, double xsi,
                                         const double* old, double* img) {
  const double type = r[kB3Type * s];
  const double vgs_n = type * (xg - xsi), vds_n = type * (xdi - xsi), vbs_n = type * (xb - xsi);
  const double vgd_n = type * (xg - xdi), vbd_n = type * (xb - xdi);
  const double vgs_o = old[0], vds_o = old[1], vbs_o = old[2];
  const double vgd_o = vgs_o - vds_o, vbd_o = vbs_o - vds_o;
  const double von = type * r[kB3Vth0i * s];
  const double vt0 = r[kB3Vt0 * s], vcrit = r[kB3Vcrit * s];
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
    vbs = pnjlim_dev(vbs_n, vbs_o, vt0, vcrit, l);
  } else {
    const double vbd = pnjlim_dev(vbd_n, vbd_o, vt0, vcrit, l);
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

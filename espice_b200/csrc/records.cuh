// Per-instance device records: the bias-independent part of each model (the
// reference's Circuit.recompute, which runs each model's parameter and
// temperature preamble). One source for the host (the template's nominal
// records) and the device (every lane's records, derived in parallel from
// its parameter values): the same IEEE operations and the shared exp, log
// and pow of esl_math.h, so both give the same bits. Layout: per batch,
// `fields` x `count` doubles, field-major, so the warp evaluating
// consecutive instances reads consecutive addresses; `stride` is the count.
#pragma once

#include <math.h>
#include <stdint.h>

#include "common.h"
#include "esl_math.h"

#if defined(__CUDACC__)
#define ESL_HD static __host__ __device__ inline
#else
#define ESL_HD static inline
#endif

namespace esl {

constexpr double kBoltz = 1.38064852e-23;   // ngspice const.h CONSTboltz
constexpr double kCharge = 1.6021766208e-19; // CONSTQ

// models/diode.va:115-241 at TLEV = TLEVC = 0, no sidewall, ISR, IKF/IKR or
// tempcos of BV/RS/M: temperature map, breakdown knee, RS floor, vcrit.
ESL_HD void diode_record(const double* p, double* rec, uint32_t stride) {
  const double tk = p[15];
  const double tnomk = p[14] + 273.15;
  const double ratio = tk / tnomk;
  const double vt = kBoltz / kCharge * tk;
  const double vtnom = kBoltz / kCharge * tnomk;
  const double n = p[1];
  const double vte = n * vt;
  const double ae = p[10];
  const double egp = p[13];
  const double vtebrk = n * vt;
  const double egfet = 1.16 - (7.02e-4 * tk * tk) / (tk + 1108.0);
  const double egfet1 = 1.16 - (7.02e-4 * tnomk * tnomk) / (tnomk + 1108.0);
  const double mt = p[7];
  const double fact1 = tnomk / 300.15, fact2 = tk / 300.15;
  const double arg1 = -egfet1 / (2.0 * kBoltz * tnomk) + 1.1150877 / (2.0 * kBoltz * 300.15);
  const double argt = -egfet / (2.0 * kBoltz * tk) + 1.1150877 / (2.0 * kBoltz * 300.15);
  const double pbfact1 = -2.0 * vtnom * (1.5 * esl_log(fact1) + kCharge * arg1);
  const double pbfact = -2.0 * vt * (1.5 * esl_log(fact2) + kCharge * argt);
  const double vj = p[6];
  const double pbo = (vj - pbfact1) / fact1;
  const double gmaold = (vj - pbo) / pbo;
  const double vj_t = pbfact + fact2 * pbo;
  const double gmanew = (vj_t - pbo) / pbo;
  double cjo_t = p[5] * (1.0 + mt * (400e-6 * (tk - 300.15) - gmanew)) /
                 (1.0 + mt * (400e-6 * (tnomk - 300.15) - gmaold));
  cjo_t = cjo_t * ae;
  const double is_t = p[0] * ae * esl_exp((ratio - 1.0) * egp / vte + (p[12] / n) * esl_log(ratio));
  const double bv_t = p[3];
  const double ibvx = p[4];
  double xbv = bv_t;
  if (p[3] > 0.0 && ibvx >= is_t * bv_t / vt) {
    xbv = bv_t - vtebrk * esl_log(1.0 + ibvx / is_t);
    xbv = bv_t - vtebrk * esl_log(ibvx / is_t + 1.0 - xbv / vt);
  }
  double rs_t = p[2] / ae;
  if (rs_t < 1.0e-9) rs_t = 1.0e-9;
  rec[kDVte * stride] = vte;
  rec[kDIs * stride] = is_t;
  rec[kDVcrit * stride] = vte * esl_log(vte / (1.4142135623730951 * is_t));
  rec[kDRs * stride] = rs_t;
  rec[kDGmin * stride] = p[11];
  rec[kDBv * stride] = p[3];
  rec[kDXbv * stride] = xbv;
  rec[kDVtebrk * stride] = vtebrk;
  rec[kDCjo * stride] = cjo_t;
  rec[kDVj * stride] = vj_t;
  rec[kDMt * stride] = mt;
  rec[kDFc * stride] = p[8];
  rec[kDTt * stride] = p[9];
  rec[kDHasRs * stride] = p[2] > 0.0 ? 1.0 : 0.0;
  rec[kDHasQ * stride] = (p[5] > 0.0 || p[9] > 0.0) ? 1.0 : 0.0;
}

// models/mos1.va:150-271 (no Meyer halves: a circuit with TOX runs DC
// only), NSUB/NSS/JS/RSH left out: KP's default, temperature, geometry, junction sizing,
// the forward-region charge constants, vcrit and the MODEINITJCT vgs seed.
ESL_HD void mos1_record(const double* p, double* rec, uint32_t stride) {
  const double type = p[0];
  const double tnomk = p[32] + 273.15;
  const double vtnom = tnomk * (kBoltz / kCharge);
  const double egfet1 = 1.16 - (7.02e-4 * tnomk * tnomk) / (tnomk + 1108.0);
  const double phix = p[4];
  const double gammax = p[3];
  const double vtox = p[1] + p[29];
  // KP: the card's, else u0 * Cox' with TOX given, else 2e-5 (mos1.va:159-192)
  const double coxp = p[kMParamTox] > 0.0 ? 3.9 * 8.854214871e-12 / p[kMParamTox] : 0.0;
  const double kpx = p[2] == p[2] ? p[2] : coxp > 0.0 ? p[21] * coxp * 1.0e-4 : 2.0e-5;
  const double tk = p[33];
  const double vt = tk * (kBoltz / kCharge);
  const double fact1 = tnomk / 300.15;
  const double fact2 = tk / 300.15;
  const double egfet = 1.16 - (7.02e-4 * tk * tk) / (tk + 1108.0);
  const double arg1 = -egfet1 / (2.0 * kBoltz * tnomk) + 1.1150877 / (2.0 * kBoltz * 300.15);
  const double argt = -egfet / (2.0 * kBoltz * tk) + 1.1150877 / (2.0 * kBoltz * 300.15);
  const double pbfact1 = -2.0 * vtnom * (1.5 * esl_log(fact1) + kCharge * arg1);
  const double pbfact = -2.0 * vt * (1.5 * esl_log(fact2) + kCharge * argt);
  const double ratio4 = (tk / tnomk) * sqrt(tk / tnomk);
  const double kpt = kpx / ratio4;
  const double phio = (phix - pbfact1) / fact1;
  const double phit = fact2 * phio + pbfact;
  const double vbit = vtox - type * (gammax * sqrt(phix)) + 0.5 * (egfet1 - egfet) + type * 0.5 * (phit - phix);
  const double ist = p[10] * esl_exp(-egfet / vt + egfet1 / vtnom);
  const double pb = p[11], mj = p[16], mjsw = p[18];
  const double pbo = (pb - pbfact1) / fact1;
  const double pbt = fact2 * pbo + pbfact;
  const double gmaold = (pb - pbo) / pbo;
  const double gmanew = (pbt - pbo) / pbo;
  const double cfb = (1.0 + mj * (4.0e-4 * (tk - 300.15) - gmanew)) / (1.0 + mj * (4.0e-4 * (tnomk - 300.15) - gmaold));
  const double cfsw = (1.0 + mjsw * (4.0e-4 * (tk - 300.15) - gmanew)) / (1.0 + mjsw * (4.0e-4 * (tnomk - 300.15) - gmaold));
  const double m = p[30], w = p[23];
  double leff = p[24] - 2.0 * p[20];
  if (leff < 1.0e-10) leff = 1.0e-10;
  const double beta = kpt * m * w / leff;
  const double isatd = ist * m, isats = ist * m;
  const double cj = p[15], cjsw = p[17];
  const double czbd = p[8] > 0.0 ? p[8] * cfb * m : cj * cfb * p[25] * m;
  const double czbs = p[9] > 0.0 ? p[9] * cfb * m : cj * cfb * p[26] * m;
  const double czbdsw = cjsw * cfsw * p[27] * m;
  const double czbssw = cjsw * cfsw * p[28] * m;
  const double fc = p[22];
  const double depcap = fc * pbt;
  const double argf = 1.0 - fc;
  const double sargb = esl_pow(argf, -mj);
  const double sargs = esl_pow(argf, -mjsw);
  const double f2d = czbd * (1.0 - fc * (1.0 + mj)) * sargb / argf + czbdsw * (1.0 - fc * (1.0 + mjsw)) * sargs / argf;
  const double f3d = czbd * mj * sargb / (argf * pbt) + czbdsw * mjsw * sargs / (argf * pbt);
  const double f4d = czbd * pbt * (1.0 - argf * sargb) / (1.0 - mj) + czbdsw * pbt * (1.0 - argf * sargs) / (1.0 - mjsw) -
                     0.5 * f3d * depcap * depcap - depcap * f2d;
  const double f2s = czbs * (1.0 - fc * (1.0 + mj)) * sargb / argf + czbssw * (1.0 - fc * (1.0 + mjsw)) * sargs / argf;
  const double f3s = czbs * mj * sargb / (argf * pbt) + czbssw * mjsw * sargs / (argf * pbt);
  const double f4s = czbs * pbt * (1.0 - argf * sargb) / (1.0 - mj) + czbssw * pbt * (1.0 - argf * sargs) / (1.0 - mjsw) -
                     0.5 * f3s * depcap * depcap - depcap * f2s;
  const double cgs = p[12] * w * m, cgd = p[13] * w * m, cgb = p[14] * leff * m;
  auto put = [&](int f, double v) { rec[f * stride] = v; };
  put(kMType, type);
  put(kMVt, vt);
  put(kMVbit, vbit);
  put(kMGamma, gammax);
  put(kMPhit, phit);
  put(kMBeta, beta);
  put(kMLambda, p[5]);
  put(kMIsats, isats);
  put(kMIsatd, isatd);
  put(kMVcrits, vt * esl_log(vt / (1.4142135623730951 * isats)));
  put(kMVcritd, vt * esl_log(vt / (1.4142135623730951 * isatd)));
  put(kMGdrain, p[6] > 0.0 ? m / p[6] : 0.0);
  put(kMGsource, p[7] > 0.0 ? m / p[7] : 0.0);
  put(kMCzbd, czbd);
  put(kMCzbs, czbs);
  put(kMCzbdsw, czbdsw);
  put(kMCzbssw, czbssw);
  put(kMPbt, pbt);
  put(kMMj, mj);
  put(kMMjsw, mjsw);
  put(kMFc, fc);
  put(kMF2d, f2d);
  put(kMF3d, f3d);
  put(kMF4d, f4d);
  put(kMF2s, f2s);
  put(kMF3s, f3s);
  put(kMF4s, f4s);
  put(kMCgs, cgs);
  put(kMCgd, cgd);
  put(kMCgb, cgb);
  put(kMGmin, p[31]);
  put(kMHasQ, (czbd != 0.0 || czbs != 0.0 || czbdsw != 0.0 || czbssw != 0.0 || cgs != 0.0 || cgd != 0.0 ||
               cgb != 0.0) ? 1.0 : 0.0);
  put(kMSeedVgs, type * vbit + gammax * sqrt(phit));
}

// BSIM3v3 card slots, in the order of include/espice_lanes.h (ESL_B3).
enum B3Slot {
  sType, sMobmod, sTnom, sTox, sToxm, sXj, sNch, sNsub, sNgate, sGamma1, sGamma2, sXt, sVbx, sVbm, sK1,
  sK2, sK3, sK3b, sW0, sNlx, sVth0, sVfb, sDvt0, sDvt1, sDvt2, sDvt0w, sDvt1w, sDvt2w, sDrout, sDsub,
  sNfactor, sCdsc, sCdscb, sCdscd, sCit, sVsat, sAt, sA0, sAgs, sA1, sA2, sKeta, sUa, sUa1, sUb, sUb1,
  sUc, sUc1, sU0, sUte, sVoff, sDelta, sRdsw, sPrwg, sPrwb, sPrt, sWr, sEta0, sEtab, sPclm, sPdiblc1,
  sPdiblc2, sPdiblcb, sPscbe1, sPscbe2, sPvag, sDwg, sDwb, sB0, sB1, sAlpha0, sAlpha1, sBeta0, sKt1,
  sKt1l, sKt2, sLint, sLl, sLln, sLw, sLwn, sLwl, sWint, sWl, sWln, sWw, sWwn, sWwl, sXl, sXw, sJs,
  sJsw, sNj, sXti, sIjth, sRsh, sL, sW, sAd, sAs, sPd, sPs, sNrd, sNrs, sMult, sDelvto, sMulu0, sGmin,
  sTemp, sB3Slots
};
static_assert(sB3Slots == kB3Params && sRsh == kB3ParamRsh && sNrd == kB3ParamNrd && sNrs == kB3ParamNrs,
              "BSIM3 card slots");

// models/bsim3.va:186-346 (b3temp.c): temperature scaling, geometry,
// parameter defaulting ($param_given = a non-NaN slot), the doping-derived
// quantities, the k1/k2 ladder, vfb/vth0, junction sizing and the series
// resistance; then the fields the bias-dependent chain reads.
ESL_HD void bsim3_record(const double* p, double* rec, uint32_t stride) {
  auto given = [p](int k) { return p[k] == p[k]; };  // $param_given: not NaN
  const double type = p[sType], tox = p[sTox];
  const double tnomk = p[sTnom] + 273.15, tk = p[sTemp];
  const double tratio = tk / tnomk;
  const double vtnom = 8.617087e-5 * tnomk;
  const double vt = 8.617087e-5 * tk;
  const double eg0 = 1.16 - 7.02e-4 * tnomk * tnomk / (tnomk + 1108.0);
  const double eg = 1.16 - 7.02e-4 * tk * tk / (tk + 1108.0);
  const double ni = 1.45e10 * (tnomk / 300.15) * sqrt(tnomk / 300.15) * esl_exp(21.5565981 - eg0 / (2.0 * vtnom));
  const double cox = 3.453133e-11 / tox;
  const double factor1 = sqrt(1.03594e-10 / 3.453133e-11 * tox);
  // pnjlim's constants at the device-support frame's 300.15 K
  const double vt0 = kBoltz * 300.15 / kCharge;
  const double vcrit = vt0 * esl_log(vt0 / (1.4142135623730951 * 1.0e-14));
  double jst = p[sJs], jswt = p[sJsw];
  if (tk != tnomk) {
    const double jtmp = esl_exp((eg0 / vtnom - eg / vt + p[sXti] * esl_log(tratio)) / p[sNj]);
    jst = p[sJs] * jtmp;
    jswt = p[sJsw] * jtmp;
  }
  if (jst < 0.0) jst = 0.0;
  if (jswt < 0.0) jswt = 0.0;

  const double l = p[sL], w = p[sW];
  const double pl = esl_pow(l, p[sLln]), pw = esl_pow(w, p[sLwn]);
  const double dl = p[sLint] + p[sLl] / pl + p[sLw] / pw + p[sLwl] / (pl * pw);
  const double ql = esl_pow(l, p[sWln]), qw = esl_pow(w, p[sWwn]);
  const double dw = p[sWint] + p[sWl] / ql + p[sWw] / qw + p[sWwl] / (ql * qw);
  double leff = l + p[sXl] - 2.0 * dl;
  double weff = w + p[sXw] - 2.0 * dw;
  if (leff < 1.0e-9) leff = 1.0e-9;
  if (weff < 1.0e-9) weff = 1.0e-9;

  const int mobmod = static_cast<int>(p[sMobmod]);
  const double uax = p[sUa] + p[sUa1] * (tratio - 1.0);
  const double ubx = p[sUb] + p[sUb1] * (tratio - 1.0);
  double ucx = given(sUc) ? p[sUc] : (mobmod == 3 ? -0.0465 : -0.0465e-9);
  const double uc1x = given(sUc1) ? p[sUc1] : (mobmod == 3 ? -0.056 : -0.056e-9);
  ucx = ucx + uc1x * (tratio - 1.0);
  double u0x = given(sU0) ? p[sU0] : (type > 0.0 ? 0.067 : 0.025);
  if (u0x > 1.0) u0x = u0x / 1.0e4;  // a cm^2/Vs card value
  const double u0temp = u0x * esl_pow(tratio, p[sUte]) * p[sMulu0];
  const double vsattemp = p[sVsat] - p[sAt] * (tratio - 1.0);
  const double rds0 = (p[sRdsw] + p[sPrt] * (tratio - 1.0)) / esl_pow(weff * 1.0e6, p[sWr]);

  double npeak;
  if (given(sNch)) {
    npeak = p[sNch];
    if (npeak > 1.0e20) npeak = npeak * 1.0e-6;  // an m^-3 card value
  } else if (given(sGamma1)) {
    const double g = p[sGamma1] * cox;
    npeak = 3.021e22 * g * g;
  } else {
    npeak = 1.7e17;
  }
  double ngate = p[sNgate];
  if (ngate > 1.000001e24) ngate = ngate * 1.0e-6;
  const double phi = 2.0 * vtnom * esl_log(npeak / ni);
  const double sqrtphi = sqrt(phi);
  const double xdep0 = sqrt(2.0 * 1.03594e-10 / (1.60219e-19 * npeak * 1.0e6)) * sqrtphi;
  const double vbi = vtnom * esl_log(1.0e20 * npeak / (ni * ni));
  const double cdep0 = sqrt(1.60219e-19 * 1.03594e-10 * npeak * 1.0e6 / 2.0 / phi);

  double vbm = p[sVbm], k1, k2;
  if (given(sK1) || given(sK2)) {
    k1 = given(sK1) ? p[sK1] : 0.53;
    k2 = given(sK2) ? p[sK2] : -0.0186;
  } else {
    double vbx = given(sVbx) ? p[sVbx] : phi - 7.7348e-4 * npeak * p[sXt] * p[sXt];
    if (vbx > 0.0) vbx = -vbx;
    if (vbm > 0.0) vbm = -vbm;
    const double g1 = given(sGamma1) ? p[sGamma1] : 5.753e-12 * sqrt(npeak) / cox;
    const double g2 = given(sGamma2) ? p[sGamma2] : 5.753e-12 * sqrt(p[sNsub]) / cox;
    const double a = g1 - g2;
    const double b = sqrt(phi - vbx) - sqrtphi;
    const double c = sqrt(phi * (phi - vbm)) - phi;
    k2 = a * b / (2.0 * c + vbm);
    k1 = g2 - 2.0 * k2 * sqrt(phi - vbm);
  }
  double vbsc = -30.0;
  if (k2 < 0.0) {
    const double h = 0.5 * k1 / k2;
    vbsc = 0.9 * (phi - h * h);
    if (vbsc > -3.0) vbsc = -3.0;
    else if (vbsc < -30.0) vbsc = -30.0;
  }
  if (vbsc > vbm) vbsc = vbm;

  double vfb;
  if (given(sVfb)) vfb = p[sVfb];
  else if (given(sVth0)) vfb = type * p[sVth0] - phi - k1 * sqrtphi;
  else vfb = -1.0;
  const double vth0 = given(sVth0) ? p[sVth0] : type * (vfb + phi + k1 * sqrtphi);
  const double vth0i = vth0 + p[sDelvto];
  const double vfbi = vfb + type * p[sDelvto];
  const double toxm = given(sToxm) ? p[sToxm] : tox;
  const double dsub = given(sDsub) ? p[sDsub] : p[sDrout];
  const double lt0 = factor1 * sqrt(xdep0);
  const double e1 = esl_exp(-0.5 * dsub * leff / lt0);
  const double e2 = esl_exp(-0.5 * p[sDrout] * leff / lt0);

  const double nvtmj = vt * p[sNj];
  const double isats = (p[sAs] <= 0.0 && p[sPs] <= 0.0) ? 1.0e-14 : p[sAs] * jst + p[sPs] * jswt;
  const double isatd = (p[sAd] <= 0.0 && p[sPd] <= 0.0) ? 1.0e-14 : p[sAd] * jst + p[sPd] * jswt;
  const double ijth = p[sIjth];
  double vjsm = 0.0, isevjsm = 0.0, vjdm = 0.0, isevjdm = 0.0;
  if (isats > 0.0 && ijth > 0.0) {
    vjsm = nvtmj * esl_log(ijth / isats + 1.0);
    isevjsm = isats * esl_exp(vjsm / nvtmj);
  }
  if (isatd > 0.0 && ijth > 0.0) {
    vjdm = nvtmj * esl_log(ijth / isatd + 1.0);
    isevjdm = isatd * esl_exp(vjdm / nvtmj);
  }
  const double m = p[sMult], rsh = p[sRsh];

  auto put = [&](int f, double v) { rec[f * stride] = v; };
  put(kB3Type, type);
  put(kB3Mobmod, static_cast<double>(mobmod));
  put(kB3Vt, vt);
  put(kB3Tratio1, tk / tnomk - 1.0);
  put(kB3Vth0i, vth0i);
  put(kB3Isats, isats);
  put(kB3Isatd, isatd);
  put(kB3Nvtmj, nvtmj);
  put(kB3Vjsm, vjsm);
  put(kB3Isevjsm, isevjsm);
  put(kB3Vjdm, vjdm);
  put(kB3Isevjdm, isevjdm);
  put(kB3Ijth, ijth);
  put(kB3Gmin, p[sGmin]);
  put(kB3Vbsc, vbsc);
  put(kB3Phi, phi);
  put(kB3Sqrtphi, sqrtphi);
  put(kB3Phis3, sqrtphi * phi);
  put(kB3Xdep0, xdep0);
  put(kB3Factor1, factor1);
  put(kB3Dvt2, p[sDvt2]);
  put(kB3Dvt2w, p[sDvt2w]);
  put(kB3Dvt1, p[sDvt1]);
  put(kB3Dvt1w, p[sDvt1w]);
  put(kB3Dvt0, p[sDvt0]);
  put(kB3Dvt0w, p[sDvt0w]);
  put(kB3Leff, leff);
  put(kB3Weff, weff);
  put(kB3Vbi, vbi);
  put(kB3Nlx, p[sNlx]);
  put(kB3K1x, k1);
  put(kB3K1ox, k1 * tox / toxm);
  put(kB3K2ox, k2 * tox / toxm);
  put(kB3Kt1, p[sKt1]);
  put(kB3Kt1l, p[sKt1l]);
  put(kB3Kt2, p[sKt2]);
  put(kB3Tox, tox);
  put(kB3W0, p[sW0]);
  put(kB3K3, p[sK3]);
  put(kB3K3b, p[sK3b]);
  put(kB3Eta0, p[sEta0]);
  put(kB3Etab, p[sEtab]);
  put(kB3Theta0vb0, e1 + 2.0 * e1 * e1);
  put(kB3Nfactor, p[sNfactor]);
  put(kB3Cdsc, p[sCdsc]);
  put(kB3Cdscb, p[sCdscb]);
  put(kB3Cdscd, p[sCdscd]);
  put(kB3Cit, p[sCit]);
  put(kB3Cox, cox);
  put(kB3Vfbi, vfbi);
  put(kB3Ngate, ngate);
  put(kB3Voff, p[sVoff]);
  put(kB3Cdep0, cdep0);
  put(kB3Dwg, p[sDwg]);
  put(kB3Dwb, p[sDwb]);
  put(kB3Rds0, rds0);
  put(kB3Prwg, p[sPrwg]);
  put(kB3Prwb, p[sPrwb]);
  put(kB3Xj, p[sXj]);
  put(kB3A0, p[sA0]);
  put(kB3B0, p[sB0]);
  put(kB3B1, p[sB1]);
  put(kB3Ags, p[sAgs]);
  put(kB3Keta, p[sKeta]);
  put(kB3Ua, uax);
  put(kB3Ub, ubx);
  put(kB3Uc, ucx);
  put(kB3U0temp, u0temp);
  put(kB3Vsattemp, vsattemp);
  put(kB3A1, p[sA1]);
  put(kB3A2, p[sA2]);
  put(kB3Delta, p[sDelta]);
  put(kB3Pclm, p[sPclm]);
  put(kB3Litl, sqrt(3.0 * p[sXj] * tox));
  put(kB3Thetarout, p[sPdiblc1] * (e2 + 2.0 * e2 * e2) + p[sPdiblc2]);
  put(kB3Pdiblcb, p[sPdiblcb]);
  put(kB3Pvag, p[sPvag]);
  put(kB3Pscbe1, p[sPscbe1]);
  put(kB3Pscbe2, p[sPscbe2]);
  put(kB3Alpha0, p[sAlpha0]);
  put(kB3Alpha1, p[sAlpha1]);
  put(kB3Beta0, p[sBeta0]);
  put(kB3M, m);
  put(kB3Gdrain, (rsh > 0.0 && p[sNrd] > 0.0) ? m / (rsh * p[sNrd]) : 0.0);
  put(kB3Gsource, (rsh > 0.0 && p[sNrs] > 0.0) ? m / (rsh * p[sNrs]) : 0.0);
  put(kB3Vt0, vt0);
  put(kB3Vcrit, vcrit);
  // MODEINITJCT (b3ld.c:202-214): vgs = type*vth0 + 0.1, vds = 0.1, vbs = 0
  put(kB3SeedVgs, type * vth0i + 0.1);
}

ESL_HD void derive_record(uint32_t type, const double* params, double* rec, uint32_t stride) {
  switch (type) {
    case kR:
    case kC:
      rec[0] = params[0];
      break;
    case kV:
    case kI:
      for (int f = 0; f < kSrcParams; ++f) rec[f * stride] = params[f];
      break;
    case kD:
      diode_record(params, rec, stride);
      break;
    case kM:
      mos1_record(params, rec, stride);
      break;
    case kB3:
      bsim3_record(params, rec, stride);
      break;
    default:
      break;
  }
}

}  // namespace esl

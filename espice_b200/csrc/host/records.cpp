// Per-instance device records: the bias-independent part of each model,
// derived on the host once per lane install (the reference's
// Circuit.recompute, which runs each model's parameter and temperature
// preamble). Layout: per batch, `fields` x `count` doubles, field-major, so
// the warp evaluating consecutive instances reads consecutive addresses.
#include "records.hpp"

#include <cmath>
#include <cstring>

namespace esl {

namespace {
constexpr double kBoltz = 1.38064852e-23;   // ngspice const.h CONSTboltz
constexpr double kCharge = 1.6021766208e-19; // CONSTQ
}

uint32_t record_fields(uint32_t type) {
  switch (type) {
    case kR: return kRFields;
    case kC: return kCFields;
    case kV: return kVFields;
    case kI: return kIFields;
    case kD: return kDiodeFields;
    case kM: return kMosFields;
    default: return 0;
  }
}

uint32_t param_count(uint32_t type) {
  static const uint32_t n[kNumTypes] = {1, 1, 10, 1, kDiodeParams, kMosParams};
  return type < kNumTypes ? n[type] : 0;
}

uint32_t node_count(uint32_t type) {
  static const uint32_t n[kNumTypes] = {2, 2, 3, 2, 3, 6};
  return type < kNumTypes ? n[type] : 0;
}

// models/diode.va:115-241 at TLEV = TLEVC = 0, no sidewall, ISR, IKF/IKR or
// tempcos of BV/RS/M: temperature map, breakdown knee, RS floor, vcrit.
static void diode_record(const double* p, double* rec, uint32_t stride) {
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
  const double pbfact1 = -2.0 * vtnom * (1.5 * std::log(fact1) + kCharge * arg1);
  const double pbfact = -2.0 * vt * (1.5 * std::log(fact2) + kCharge * argt);
  const double vj = p[6];
  const double pbo = (vj - pbfact1) / fact1;
  const double gmaold = (vj - pbo) / pbo;
  const double vj_t = pbfact + fact2 * pbo;
  const double gmanew = (vj_t - pbo) / pbo;
  double cjo_t = p[5] * (1.0 + mt * (400e-6 * (tk - 300.15) - gmanew)) /
                 (1.0 + mt * (400e-6 * (tnomk - 300.15) - gmaold));
  cjo_t = cjo_t * ae;
  const double is_t = p[0] * ae * std::exp((ratio - 1.0) * egp / vte + (p[12] / n) * std::log(ratio));
  const double bv_t = p[3];
  const double ibvx = p[4];
  double xbv = bv_t;
  if (p[3] > 0.0 && ibvx >= is_t * bv_t / vt) {
    xbv = bv_t - vtebrk * std::log(1.0 + ibvx / is_t);
    xbv = bv_t - vtebrk * std::log(ibvx / is_t + 1.0 - xbv / vt);
  }
  double rs_t = p[2] / ae;
  if (rs_t < 1.0e-9) rs_t = 1.0e-9;
  rec[kDVte * stride] = vte;
  rec[kDIs * stride] = is_t;
  rec[kDVcrit * stride] = vte * std::log(vte / (1.4142135623730951 * is_t));
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

// models/mos1.va:150-271 with KP given (no TOX: no derived KP, no Meyer
// halves), NSUB/NSS/JS/RSH left out: temperature, geometry, junction sizing,
// the forward-region charge constants, vcrit and the MODEINITJCT vgs seed.
static void mos1_record(const double* p, double* rec, uint32_t stride) {
  const double type = p[0];
  const double tnomk = p[32] + 273.15;
  const double vtnom = tnomk * (kBoltz / kCharge);
  const double egfet1 = 1.16 - (7.02e-4 * tnomk * tnomk) / (tnomk + 1108.0);
  const double phix = p[4];
  const double gammax = p[3];
  const double vtox = p[1] + p[29];
  const double kpx = p[2];
  const double tk = p[33];
  const double vt = tk * (kBoltz / kCharge);
  const double fact1 = tnomk / 300.15;
  const double fact2 = tk / 300.15;
  const double egfet = 1.16 - (7.02e-4 * tk * tk) / (tk + 1108.0);
  const double arg1 = -egfet1 / (2.0 * kBoltz * tnomk) + 1.1150877 / (2.0 * kBoltz * 300.15);
  const double argt = -egfet / (2.0 * kBoltz * tk) + 1.1150877 / (2.0 * kBoltz * 300.15);
  const double pbfact1 = -2.0 * vtnom * (1.5 * std::log(fact1) + kCharge * arg1);
  const double pbfact = -2.0 * vt * (1.5 * std::log(fact2) + kCharge * argt);
  const double ratio4 = (tk / tnomk) * std::sqrt(tk / tnomk);
  const double kpt = kpx / ratio4;
  const double phio = (phix - pbfact1) / fact1;
  const double phit = fact2 * phio + pbfact;
  const double vbit = vtox - type * (gammax * std::sqrt(phix)) + 0.5 * (egfet1 - egfet) + type * 0.5 * (phit - phix);
  const double ist = p[10] * std::exp(-egfet / vt + egfet1 / vtnom);
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
  const double sargb = std::pow(argf, -mj);
  const double sargs = std::pow(argf, -mjsw);
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
  put(kMVcrits, vt * std::log(vt / (1.4142135623730951 * isats)));
  put(kMVcritd, vt * std::log(vt / (1.4142135623730951 * isatd)));
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
  put(kMSeedVgs, type * vbit + gammax * std::sqrt(phit));
}

void derive_instance(uint32_t type, const double* params, double* rec, uint32_t stride) {
  switch (type) {
    case kR:
    case kC:
    case kI:
      rec[0] = params[0];
      break;
    case kV:
      for (int f = 0; f < kVFields; ++f) rec[f * stride] = params[f];
      break;
    case kD:
      diode_record(params, rec, stride);
      break;
    case kM:
      mos1_record(params, rec, stride);
      break;
    default:
      break;
  }
}

}  // namespace esl

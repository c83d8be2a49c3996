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
    default: return 0;
  }
}

uint32_t param_count(uint32_t type) {
  static const uint32_t n[kNumTypes] = {1, 1, 10, 1, kDiodeParams, 34};
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
    default:
      break;
  }
}

}  // namespace esl

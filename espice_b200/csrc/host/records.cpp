// Per-instance device records on the host: the field and parameter counts
// of each device type, and the template's nominal records (the derivation
// itself is csrc/records.cuh, shared with the device).
#include "records.hpp"

#include "../records.cuh"

namespace esl {

uint32_t record_fields(uint32_t type) {
  switch (type) {
    case kR: return kRFields;
    case kC: return kCFields;
    case kV: return kVFields;
    case kI: return kIFields;
    case kD: return kDiodeFields;
    case kM: return kMosFields;
    case kB3: return kB3Fields;
    default: return 0;
  }
}

uint32_t param_count(uint32_t type) {
  static const uint32_t n[kNumTypes] = {1, 1, kSrcParams, kSrcParams, kDiodeParams, kMosParams, kB3Params};
  return type < kNumTypes ? n[type] : 0;
}

uint32_t node_count(uint32_t type) {
  static const uint32_t n[kNumTypes] = {2, 2, 3, 2, 3, 6, 6};
  return type < kNumTypes ? n[type] : 0;
}

void derive_instance(uint32_t type, const double* params, double* rec, uint32_t stride) {
  derive_record(type, params, rec, stride);
}

}  // namespace esl

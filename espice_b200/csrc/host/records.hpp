// Per-instance device records (see records.cpp).
#pragma once

#include <cstdint>

#include "../common.h"

namespace esl {

constexpr uint32_t kDiodeParams = 16;  // is n rs bv ibv cjo vj m fc tt area gmin xti eg tnom temp

uint32_t record_fields(uint32_t type);
uint32_t param_count(uint32_t type);
uint32_t node_count(uint32_t type);
// Writes instance records with field stride `stride` (the batch count).
void derive_instance(uint32_t type, const double* params, double* rec, uint32_t stride);

}  // namespace esl

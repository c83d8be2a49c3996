// Device derivation of every lane's records (derive.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace esl {

// An instance a lane's swept parameters touch: its device type, its
// parameter count and nominal row (d_params + prm_at), where its record
// starts in a lane's records (rec_at, fields `stride` apart) and its
// overrides slots[slot0, slot1).
struct DeriveItem {
  uint32_t type, np, rec_at, stride, prm_at, slot0, slot1, pad;
};
// One override: parameter `param` of the instance takes column `col` of the
// lane's value row.
struct DeriveSlot {
  uint32_t param, col;
};

// d_rec [n_lanes][R]: the nominal records, then each item derived again
// with lane l's values d_values [n_lanes][n_cols].
cudaError_t launch_derive_lanes(const double* d_rec_nominal, uint32_t R, const DeriveItem* d_items, uint32_t n_items,
                                const DeriveSlot* d_slots, const double* d_params, const double* d_values,
                                uint32_t n_cols, uint32_t n_lanes, double* d_rec, cudaStream_t s);

}  // namespace esl

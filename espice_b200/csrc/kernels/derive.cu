// Every lane's device records derived on the device (the reference's
// Circuit.recompute per sweep point, src/device/Circuit.zig): each lane
// starts from the template's nominal records, then every instance a swept
// parameter touches is derived again from its nominal parameter row with
// the lane's values in place, by the same code the host uses for the
// nominal records (csrc/records.cuh).
#include "derive.h"

#include "../records.cuh"

namespace esl {

namespace {

constexpr uint32_t kMaxParams = kSrcParams;  // the widest parameter row (V and I sources)
static_assert(kB3Params <= kMaxParams && kMosParams <= kMaxParams, "parameter rows");

// rec[lane][f] = nominal[f]: lanes along y, fields along x (coalesced).
__global__ void rec_broadcast_kernel(const double* __restrict__ nominal, uint32_t R, uint32_t n_lanes,
                                     double* __restrict__ rec) {
  for (uint32_t lane = blockIdx.y; lane < n_lanes; lane += gridDim.y) {
    double* out = rec + size_t(lane) * R;
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < R; f += gridDim.x * blockDim.x) out[f] = nominal[f];
  }
}

// One thread per (lane, touched instance); the instances of a lane are
// consecutive threads, so a field's stores from a batch's instances are
// consecutive addresses.
__global__ void derive_lanes_kernel(const DeriveItem* __restrict__ items, uint32_t n_items,
                                    const DeriveSlot* __restrict__ slots, const double* __restrict__ nominal,
                                    const double* __restrict__ values, uint32_t n_cols, uint32_t n_lanes, uint32_t R,
                                    double* __restrict__ rec) {
  const size_t idx = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= size_t(n_items) * n_lanes) return;
  const uint32_t lane = uint32_t(idx / n_items), it = uint32_t(idx % n_items);
  const DeriveItem I = items[it];
  double prm[kMaxParams];
  for (uint32_t k = 0; k < I.np; ++k) prm[k] = nominal[I.prm_at + k];
  for (uint32_t s = I.slot0; s < I.slot1; ++s) prm[slots[s].param] = values[size_t(lane) * n_cols + slots[s].col];
  derive_record(I.type, prm, rec + size_t(lane) * R + I.rec_at, I.stride);
}

}  // namespace

cudaError_t launch_derive_lanes(const double* d_rec_nominal, uint32_t R, const DeriveItem* d_items, uint32_t n_items,
                                const DeriveSlot* d_slots, const double* d_params, const double* d_values,
                                uint32_t n_cols, uint32_t n_lanes, double* d_rec, cudaStream_t s) {
  if (n_lanes == 0 || R == 0) return cudaSuccess;
  const uint32_t bx = (R + 255) / 256;
  const dim3 grid(bx < 64 ? bx : 64, n_lanes < 8192 ? n_lanes : 8192);
  rec_broadcast_kernel<<<grid, 256, 0, s>>>(d_rec_nominal, R, n_lanes, d_rec);
  if (cudaError_t e = cudaGetLastError()) return e;
  if (n_items == 0) return cudaSuccess;
  const size_t threads = size_t(n_items) * n_lanes;
  const uint32_t block = 128;
  derive_lanes_kernel<<<uint32_t((threads + block - 1) / block), block, 0, s>>>(d_items, n_items, d_slots, d_params,
                                                                               d_values, n_cols, n_lanes, R, d_rec);
  return cudaGetLastError();
}

}  // namespace esl

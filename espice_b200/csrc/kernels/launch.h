// Host-callable launchers of the sweep-lane kernels (newton.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "lanes.cuh"

namespace esl {

size_t lane_smem_bytes(const TopoDev& T);
cudaError_t launch_dc_newton(const TopoDev& T, const LaneDev& L, const LaneOpts& o,
                             uint32_t lanes_per_block, cudaStream_t s);
cudaError_t launch_assemble(const TopoDev& T, const LaneDev& L, uint32_t lane, double* out,
                            cudaStream_t s);
cudaError_t launch_lu_replay(const TopoDev& T, uint32_t n_lanes, const double* a, const double* rhs,
                             double* tv, double* dx, uint8_t* bad, uint32_t lanes_per_block,
                             cudaStream_t s);

cudaError_t launch_sweep(const TopoDev& T, const LaneDev& L, const SweepDev& P, const LaneOpts& o,
                         uint32_t lanes_per_block, cudaStream_t s);
cudaError_t launch_tran(const TopoDev& T, const LaneDev& L, const TranDev& P, const LaneOpts& o,
                        uint32_t lanes_per_block, cudaStream_t s);

// Lane-interleaved refactor + solve: seq = the programs' real ops in row
// order (program A's first n_seq_a), planes [entry][lane].
uint32_t lu_lanes_smem(const TopoDev& T, uint32_t n_seq, uint32_t warps);
cudaError_t launch_lu_lanes(const TopoDev& T, const uint2* seq, uint32_t n_seq_a, uint32_t n_seq, uint32_t n_lanes,
                            const double* a, const double* rhs, double* tv, double* dx, uint8_t* bad,
                            uint32_t warps, cudaStream_t s);

// The same in FP32 with FP64 iterative refinement; seq = A ops, B ops, then
// the forward-only ops (n_seq_f).
uint32_t lu_lanes_mixed_smem(const TopoDev& T, uint32_t n_ops, uint32_t warps);
cudaError_t launch_lu_lanes_mixed(const TopoDev& T, const uint2* seq, uint32_t n_seq_a, uint32_t n_seq,
                                  uint32_t n_seq_f, uint32_t n_lanes, const double* a, const double* rhs, double* dx,
                                  uint8_t* bad, uint8_t* refine, uint32_t warps, cudaStream_t s);

// Uneven batching: one launch over the lanes of several topologies.
cudaError_t launch_dc_newton_group(const TopoDev* d_topos, const LaneDev* d_lanes, const uint32_t* d_cta_ctx,
                                   const uint32_t* d_cta_first, const uint32_t* d_ctx_lpb, uint32_t n_ctas,
                                   uint32_t max_lpb, size_t smem, const LaneOpts& o, bool has_b3, cudaStream_t s);
// True when a topology has a BSIM3 batch (its lanes run the kernels'
// BSIM3 instantiation).
bool topo_has_b3(const TopoDev& T);

// Fixed lane scratch of the allocation-free DC entry point: its size, the
// device address of the array on the current device (looked up once per
// device; the first call per device must precede any stream capture), and
// the device-side lane start-state kernel.
constexpr size_t kStaticScratchBytes = size_t(16) << 20;
cudaError_t static_scratch(void** ptr);
cudaError_t launch_lane_init(const TopoDev& T, const LaneDev& L, bool cold, bool init_fix, cudaStream_t s);

}  // namespace esl

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

}  // namespace esl

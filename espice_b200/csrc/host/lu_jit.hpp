// Tape-compiled lane LU: the lead lane's pivot tape turned into one
// straight-line CUDA kernel (refactor, the forward solve merged in, the peel
// tests, the back solve), compiled for sm_100a at run time with NVRTC and
// loaded through the runtime's library API.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "schedule.hpp"

namespace esl {

struct LuJitInput {
  uint32_t n = 0, nnz = 0, nu = 0, nl = 0, ntv = 0, nv = 0;
  const std::vector<uint32_t>* amap = nullptr;    // pattern slot -> tape value
  const std::vector<uint32_t>* fill = nullptr;    // tape values no slot writes
  const std::vector<uint32_t>* pinv = nullptr;    // row -> pivot position (first n)
  const std::vector<uint32_t>* qcol = nullptr;    // pivot position -> column
  const std::vector<uint8_t>* l_scaled = nullptr; // per L entry: scaled pivot column
  const std::vector<Op>* seq = nullptr;           // real ops, program A then program B
  uint32_t n_seq_a = 0, n_seq = 0;
  // register budget, in values: beyond it the final tape values needed
  // farthest ahead are let go and re-read from their plane at next use
  uint32_t resident_values = 48;
  // the mixed form: FP32 factors and solves, then FP64 refinement on the
  // residual over the pattern (col_ptr, row_idx), kernel `lu_tape_mixed`
  bool mixed = false;
  const std::vector<uint32_t>* col_ptr = nullptr;
  const std::vector<uint32_t>* row_idx = nullptr;
};

// CUDA C++ source of the kernel `lu_tape`: one thread per lane over
// [entry][lane] planes, every tape value a local variable, each op one
// statement in the given order; the tape values go to their plane `tv`
// (the caller's, or scratch) as they become final and come back from it
// when their next use is far off.
std::string lu_jit_source(const LuJitInput& in);

struct LuJitKernels {
  cudaLibrary_t lib = nullptr;
  cudaKernel_t kernel = nullptr;
  std::string log;  // NVRTC's log (ptxas register and spill lines included)
};

// Compiles `src` for sm_100a (NVRTC, loaded with dlopen; --fmad=false, so
// each multiply and subtract rounds on its own) and loads the cubin on the
// current device. Returns false with `out.log` set when NVRTC is missing or
// the compile or load fails.
bool lu_jit_build(const std::string& src, LuJitKernels& out, const char* name = "lu_tape");
void lu_jit_release(LuJitKernels& k);

// tv: [ntv][n_lanes], never NULL (the kernel re-reads values from it).
cudaError_t lu_jit_launch(const LuJitKernels& k, uint32_t n_lanes, const double* a, const double* rhs, double* tv,
                          double* dx, uint8_t* bad, cudaStream_t s);

// The mixed form: tf [ntv][n_lanes] FP32 plane (never NULL), refine may be NULL.
cudaError_t lu_jit_launch_mixed(const LuJitKernels& k, uint32_t n_lanes, const double* a, const double* rhs,
                                float* tf, double* dx, uint8_t* bad, uint8_t* refine, cudaStream_t s);

}  // namespace esl

// Launchers of the learned warm start's tensor-core kernels (mlp.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace esl {

// C = A (M x K) . B (N x K)^T, BF16 in, FP32 accumulate; K, N multiples of
// 16; epilogue: + bias[n], FP32 store to c, tanh (act 1) or identity as BF16
// to h. err receives 1 when a tensor-core completion wait ran out (after
// wait_rounds try_wait rounds; 0: the kernel's default bound; ~0u: no
// round at all, the wait runs out at once), and then nothing is stored.
cudaError_t launch_gemm_bf16(const __nv_bfloat16* a, int lda, const __nv_bfloat16* b, int ldb, int M, int N, int K,
                             const float* bias, float* c, int ldc, __nv_bfloat16* h, int ldh, int act, int* err,
                             cudaStream_t s, uint32_t wait_rounds = 0);
cudaError_t launch_tanh_backward(const float* dh, const float* zpre, int rows, int cols, int ld, float* dz,
                                 __nv_bfloat16* dzb, cudaStream_t s);
cudaError_t launch_transpose_f32(const float* in, int rows, int cols, int ldi, __nv_bfloat16* out, int ldo,
                                 cudaStream_t s);
cudaError_t launch_transpose_bf16(const __nv_bfloat16* in, int rows, int cols, int ldi, __nv_bfloat16* out, int ldo,
                                  cudaStream_t s);
cudaError_t launch_bias_grad(const float* dz, int rows, int cols, int ld, float* db, cudaStream_t s);
cudaError_t launch_mse_grad(const float* y, const float* t, int rows, int outs, int ld, float* d, float* loss,
                            cudaStream_t s);
cudaError_t launch_adam(float* w, const float* g, float* m, float* v, int rows, int cols, float lr, int step,
                        __nv_bfloat16* wb, __nv_bfloat16* wt, int ldt, cudaStream_t s);
cudaError_t launch_to_bf16(const float* in, int n, __nv_bfloat16* out, cudaStream_t s);

}  // namespace esl

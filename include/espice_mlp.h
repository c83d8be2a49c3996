/*
 * espice_mlp.h: the learned warm start of the sweep-lane library
 * (libespice_lanes.so). A tanh MLP maps a lane's swept parameters to its
 * unknowns; it is trained on the GPU on operating points the plain solver
 * produced, by hand-written BF16 tensor-core kernels (tcgen05, FP32
 * accumulation), and evaluated there to seed the lanes' Newton solves.
 *
 * No reference counterpart: the reference's points API takes a caller's
 * warm start (include/espice.h:301, espice_points_options.warm_start) or
 * starts from its nominal operating point (src/analysis/sweep/lanes.zig:
 * 73-80). Device pointers are row-major FP32 arrays.
 */
#ifndef ESPICE_MLP_H
#define ESPICE_MLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ESL_MLP_OK = 0,
    ESL_MLP_INVALID_ARGUMENT = 1,
    ESL_MLP_OUT_OF_MEMORY = 3,
    ESL_MLP_NO_DEVICE = 5,
    ESL_MLP_DEVICE_FAULT = 6,
    ESL_MLP_TIMEOUT = 7 /* a tensor-core completion wait ran out */
};

typedef struct esl_mlp esl_mlp;

/* n_in -> n_hidden (tanh) -> ... -> n_out, n_layers weight layers (>= 2),
 * Glorot-uniform initialisation from `seed`, on CUDA device `device`. */
int32_t esl_mlp_create(int n_in, int n_hidden, int n_layers, int n_out, int device, uint64_t seed,
                       esl_mlp **out);
int32_t esl_mlp_destroy(esl_mlp *m);
const char *esl_mlp_last_error(const esl_mlp *m);

/* Standardisation (host arrays; NULL keeps the current one): the network
 * sees (x - in_mu) / in_sig and predicts (y - out_mu) / out_sig. */
int32_t esl_mlp_set_scaling(esl_mlp *m, const float *in_mu, const float *in_sig, const float *out_mu,
                            const float *out_sig);

/* Adam on the mean squared error of the standardised outputs: `epochs`
 * passes over d_x [n][n_in] -> d_y [n][n_out] in shuffled batches of
 * `batch` rows (a multiple of 16), the step size decaying geometrically from
 * lr to lr_end (lr_end <= 0: constant). loss_out [epochs] (host, may be
 * NULL). */
int32_t esl_mlp_train(esl_mlp *m, const float *d_x, const float *d_y, uint32_t n, uint32_t epochs,
                      uint32_t batch, float lr, float lr_end, uint64_t seed, float *loss_out);

/* d_y [n][n_out] = the network at d_x [n][n_in] (unstandardised). */
int32_t esl_mlp_predict(esl_mlp *m, const float *d_x, uint32_t n, float *d_y);

/* One forward and backward pass over d_x, d_y [n rows, a multiple of 16]
 * without an update: the loss and, per layer, dW (n_l x k_l) then db (n_l)
 * into `grads` (host). Layer widths via esl_mlp_shapes; current weights via
 * esl_mlp_weights (same order). For gradient checks. */
int32_t esl_mlp_gradients(esl_mlp *m, const float *d_x, const float *d_y, uint32_t n, float *loss,
                          float *grads);
int32_t esl_mlp_shapes(const esl_mlp *m, int *k, int *n, int cap, int *n_layers);
int32_t esl_mlp_weights(esl_mlp *m, float *out);

/* The tensor-core GEMM itself: C (M x N, FP32, ldc) = A (M x K, BF16, lda)
 * . B (N x K, BF16, ldb)^T (+ bias[N]); h (BF16, ldh) receives tanh (act 1)
 * or identity of the result when not NULL. K and N multiples of 16. */
int32_t esl_gemm_bf16(const void *d_a, int lda, const void *d_b, int ldb, int M, int N, int K,
                      const float *d_bias, float *d_c, int ldc, void *d_h, int ldh, int act);

/* esl_gemm_bf16 with its tensor-core completion wait bounded by wait_rounds
 * mbarrier try_wait rounds per K chunk (0: the library's bound, 2^20;
 * ESL_GEMM_NO_WAIT: no round, so every wait runs out at once). When a wait
 * runs out the kernel drains the chunk's MMAs (under the library's bound)
 * before it reuses their staging buffer or frees the accumulator's tensor
 * memory, stores nothing, and the call returns ESL_MLP_TIMEOUT. The tests
 * use ESL_GEMM_NO_WAIT to check that path. */
#define ESL_GEMM_NO_WAIT 0xffffffffu
int32_t esl_gemm_bf16_bounded(const void *d_a, int lda, const void *d_b, int ldb, int M, int N, int K,
                              const float *d_bias, float *d_c, int ldc, void *d_h, int ldh, int act,
                              uint32_t wait_rounds);

#ifdef __cplusplus
}
#endif
#endif

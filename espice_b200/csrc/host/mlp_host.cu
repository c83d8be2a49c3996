// The learned warm start's network (include/espice_mlp.h): a tanh MLP
// from the swept parameters of a lane to its unknowns, trained on the GPU by
// the tensor-core GEMM of kernels/mlp.cu (forward, backward and Adam), and
// evaluated there to seed the lanes' Newton solves.
//
// Layout: every matrix is row-major. Layer l maps k_l inputs to n_l outputs
// with W_l (n_l x k_l); widths are padded to multiples of 16 (the padding
// columns of the input and the weights stay zero). Master weights and Adam
// moments are FP32; the GEMM operands are BF16 copies (W_l and W_l^T).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../../include/espice_mlp.h"
#include "../kernels/mlp.h"

namespace {

int pad16(int v) { return (v + 15) / 16 * 16; }

template <class T>
struct Dev {
  T* p = nullptr;
  size_t n = 0;
  ~Dev() {
    if (p) cudaFree(p);
  }
  cudaError_t ensure(size_t count) {
    if (count <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e == cudaSuccess) {
      n = count;
      cudaMemset(p, 0, count * sizeof(T));
    }
    return e;
  }
};

struct Layer {
  int k = 0, n = 0;  // padded input and output widths
  Dev<float> w, b, gw, gb, mw, vw, mb, vb;
  Dev<__nv_bfloat16> wb, wt;  // BF16 W (n x k) and W^T (k x n)
};

}  // namespace

struct esl_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int n_in = 0, n_out = 0, k_in = 0, k_out = 0;
  std::vector<std::unique_ptr<Layer>> layers;
  int step = 0;
  // standardization: x' = (x - in_mu) / in_sig, y = y' * out_sig + out_mu
  std::vector<float> in_mu, in_sig, out_mu, out_sig;
  Dev<float> d_in_mu, d_in_sig, d_out_mu, d_out_sig;
  // batch work buffers (rows = batch)
  int rows = 0;
  std::vector<std::unique_ptr<Dev<__nv_bfloat16>>> hb;  // layer inputs as BF16: hb[0] = x, hb[l] = tanh(z_{l-1})
  std::vector<std::unique_ptr<Dev<__nv_bfloat16>>> ht;  // their transposes
  std::vector<std::unique_ptr<Dev<float>>> z;           // pre-activations (the last one is the output)
  Dev<float> dz, dh, t, loss, xf;
  Dev<__nv_bfloat16> dzb, dzt;
  Dev<int> gerr;
  Dev<uint32_t> idx;

  int32_t fail(int32_t code, const std::string& what) {
    err = what;
    return code;
  }
};

namespace {

#define MLP_CUDA(call)                                              \
  do {                                                              \
    cudaError_t e_ = (call);                                        \
    if (e_ != cudaSuccess) {                                        \
      m->err = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return ESL_MLP_DEVICE_FAULT;                                  \
    }                                                               \
  } while (0)

__global__ void scale_rows(const float* x, const uint32_t* idx, int rows, int cols, int ld, const float* mu,
                           const float* sig, __nv_bfloat16* out, float* outf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * ld) return;
  const int r = i / ld, c = i % ld;
  float v = 0.0f;
  if (c < cols) {
    const size_t src = idx ? idx[r] : uint32_t(r);
    v = (x[src * cols + c] - mu[c]) / sig[c];
  }
  if (out) out[i] = __float2bfloat16_rn(v);
  if (outf && c < cols) outf[size_t(r) * cols + c] = v;
}

__global__ void unscale_rows(const float* y, int rows, int cols, int ld, const float* mu, const float* sig,
                             float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const int r = i / cols, c = i % cols;
  out[i] = y[size_t(r) * ld + c] * sig[c] + mu[c];
}

int32_t ensure_batch(esl_mlp* m, int rows) {
  if (rows <= m->rows) return ESL_MLP_OK;
  const size_t L = m->layers.size();
  m->hb.clear();
  m->ht.clear();
  m->z.clear();
  for (size_t l = 0; l < L; ++l) {
    auto h = std::make_unique<Dev<__nv_bfloat16>>();
    auto ht = std::make_unique<Dev<__nv_bfloat16>>();
    MLP_CUDA(h->ensure(size_t(rows) * m->layers[l]->k));
    MLP_CUDA(ht->ensure(size_t(rows) * m->layers[l]->k));
    m->hb.push_back(std::move(h));
    m->ht.push_back(std::move(ht));
    auto zz = std::make_unique<Dev<float>>();
    MLP_CUDA(zz->ensure(size_t(rows) * m->layers[l]->n));
    m->z.push_back(std::move(zz));
  }
  int wmax = 0;
  for (auto& l : m->layers) wmax = std::max({wmax, l->k, l->n});
  MLP_CUDA(m->dz.ensure(size_t(rows) * wmax));
  MLP_CUDA(m->dh.ensure(size_t(rows) * wmax));
  MLP_CUDA(m->dzb.ensure(size_t(rows) * wmax));
  MLP_CUDA(m->dzt.ensure(size_t(rows) * wmax));
  MLP_CUDA(m->t.ensure(size_t(rows) * m->n_out));
  MLP_CUDA(m->idx.ensure(size_t(rows)));
  m->rows = rows;
  return ESL_MLP_OK;
}

// Forward over `rows` rows whose BF16 input is in hb[0]; output in z.back().
// keep_z: store every layer's FP32 pre-activation (the backward pass reads
// them); inference stores only the last layer's.
int32_t forward(esl_mlp* m, int rows, bool keep_z = true) {
  const size_t L = m->layers.size();
  for (size_t l = 0; l < L; ++l) {
    Layer& ly = *m->layers[l];
    const bool last = l + 1 == L;
    __nv_bfloat16* next = last ? nullptr : m->hb[l + 1]->p;
    float* z = (keep_z || last) ? m->z[l]->p : nullptr;
    MLP_CUDA(esl::launch_gemm_bf16(m->hb[l]->p, ly.k, ly.wb.p, ly.k, rows, ly.n, ly.k, ly.b.p, z, ly.n, next,
                                   ly.n, last ? 0 : 1, m->gerr.p, m->stream));
  }
  return ESL_MLP_OK;
}

// Backward from dz (rows x n_out, FP32) into every layer's gw, gb.
int32_t backward(esl_mlp* m, int rows) {
  const int L = int(m->layers.size());
  for (int l = L - 1; l >= 0; --l) {
    Layer& ly = *m->layers[l];
    if (l != L - 1) MLP_CUDA(esl::launch_tanh_backward(m->dh.p, m->z[l]->p, rows, ly.n, ly.n, m->dz.p, m->dzb.p, m->stream));
    else MLP_CUDA(esl::launch_to_bf16(m->dz.p, rows * ly.n, m->dzb.p, m->stream));
    // dW (n x k) = dZ^T (n x rows) . H (rows x k) = GEMM(dZ^T, H^T)
    MLP_CUDA(esl::launch_transpose_bf16(m->dzb.p, rows, ly.n, ly.n, m->dzt.p, rows, m->stream));
    MLP_CUDA(esl::launch_transpose_bf16(m->hb[l]->p, rows, ly.k, ly.k, m->ht[l]->p, rows, m->stream));
    MLP_CUDA(esl::launch_gemm_bf16(m->dzt.p, rows, m->ht[l]->p, rows, ly.n, ly.k, rows, nullptr, ly.gw.p, ly.k,
                                   nullptr, 0, 0, m->gerr.p, m->stream));
    MLP_CUDA(esl::launch_bias_grad(m->dz.p, rows, ly.n, ly.n, ly.gb.p, m->stream));
    if (l > 0) {
      // dH_{l-1} (rows x k) = dZ (rows x n) . W (n x k) = GEMM(dZ, W^T)
      MLP_CUDA(esl::launch_gemm_bf16(m->dzb.p, ly.n, ly.wt.p, ly.n, rows, ly.k, ly.n, nullptr, m->dh.p, ly.k, nullptr,
                                     0, 0, m->gerr.p, m->stream));
    }
  }
  return ESL_MLP_OK;
}

int32_t check_gemm_err(esl_mlp* m) {
  int e = 0;
  MLP_CUDA(cudaMemcpyAsync(&e, m->gerr.p, 4, cudaMemcpyDeviceToHost, m->stream));
  MLP_CUDA(cudaStreamSynchronize(m->stream));
  if (e) return m->fail(ESL_MLP_TIMEOUT, "a tensor-core completion wait ran out");
  return ESL_MLP_OK;
}

}  // namespace

extern "C" {

int32_t esl_mlp_create(int n_in, int n_hidden, int n_layers, int n_out, int device, uint64_t seed, esl_mlp** out) {
  if (!out || n_in <= 0 || n_hidden <= 0 || n_out <= 0 || n_layers < 2 || n_hidden > 256 * 8)
    return ESL_MLP_INVALID_ARGUMENT;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return ESL_MLP_NO_DEVICE;
  auto m = std::make_unique<esl_mlp>();
  m->device = device;
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) return ESL_MLP_DEVICE_FAULT;
  m->n_in = n_in;
  m->n_out = n_out;
  m->k_in = pad16(n_in);
  m->k_out = pad16(n_out);
  std::mt19937_64 rng(seed);
  std::vector<int> widths;
  widths.push_back(m->k_in);
  for (int l = 0; l + 1 < n_layers; ++l) widths.push_back(pad16(n_hidden));
  widths.push_back(m->k_out);
  for (size_t l = 0; l + 1 < widths.size(); ++l) {
    auto ly = std::make_unique<Layer>();
    ly->k = widths[l];
    ly->n = widths[l + 1];
    const int real_k = l == 0 ? n_in : n_hidden;
    const int real_n = l + 2 == widths.size() ? n_out : n_hidden;
    // Glorot-uniform on the real block, zero padding
    const float lim = std::sqrt(6.0f / float(real_k + real_n));
    std::uniform_real_distribution<float> u(-lim, lim);
    std::vector<float> w(size_t(ly->n) * ly->k, 0.0f);
    for (int r = 0; r < real_n; ++r)
      for (int c = 0; c < real_k; ++c) w[size_t(r) * ly->k + c] = u(rng);
    const size_t nw = w.size();
    for (Dev<float>* d : {&ly->w, &ly->gw, &ly->mw, &ly->vw})
      if (d->ensure(nw) != cudaSuccess) return ESL_MLP_OUT_OF_MEMORY;
    for (Dev<float>* d : {&ly->b, &ly->gb, &ly->mb, &ly->vb})
      if (d->ensure(size_t(ly->n)) != cudaSuccess) return ESL_MLP_OUT_OF_MEMORY;
    if (ly->wb.ensure(nw) != cudaSuccess || ly->wt.ensure(nw) != cudaSuccess) return ESL_MLP_OUT_OF_MEMORY;
    cudaMemcpy(ly->w.p, w.data(), nw * 4, cudaMemcpyHostToDevice);
    std::vector<__nv_bfloat16> wb(nw), wt(nw);
    for (int r = 0; r < ly->n; ++r)
      for (int c = 0; c < ly->k; ++c) {
        wb[size_t(r) * ly->k + c] = __float2bfloat16_rn(w[size_t(r) * ly->k + c]);
        wt[size_t(c) * ly->n + r] = wb[size_t(r) * ly->k + c];
      }
    cudaMemcpy(ly->wb.p, wb.data(), nw * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(ly->wt.p, wt.data(), nw * 2, cudaMemcpyHostToDevice);
    m->layers.push_back(std::move(ly));
  }
  m->in_mu.assign(n_in, 0.0f);
  m->in_sig.assign(n_in, 1.0f);
  m->out_mu.assign(n_out, 0.0f);
  m->out_sig.assign(n_out, 1.0f);
  if (m->gerr.ensure(1) != cudaSuccess) return ESL_MLP_OUT_OF_MEMORY;
  if (int32_t rc = esl_mlp_set_scaling(m.get(), nullptr, nullptr, nullptr, nullptr)) return rc;
  *out = m.release();
  return ESL_MLP_OK;
}

int32_t esl_mlp_destroy(esl_mlp* m) {
  if (!m) return ESL_MLP_OK;
  cudaSetDevice(m->device);
  cudaStream_t s = m->stream;
  if (s) cudaStreamSynchronize(s);
  delete m;
  if (s) cudaStreamDestroy(s);
  return ESL_MLP_OK;
}

const char* esl_mlp_last_error(const esl_mlp* m) { return m ? m->err.c_str() : "no network"; }

int32_t esl_mlp_set_scaling(esl_mlp* m, const float* in_mu, const float* in_sig, const float* out_mu,
                            const float* out_sig) {
  if (!m) return ESL_MLP_INVALID_ARGUMENT;
  if (in_mu) m->in_mu.assign(in_mu, in_mu + m->n_in);
  if (in_sig) m->in_sig.assign(in_sig, in_sig + m->n_in);
  if (out_mu) m->out_mu.assign(out_mu, out_mu + m->n_out);
  if (out_sig) m->out_sig.assign(out_sig, out_sig + m->n_out);
  for (float v : m->in_sig)
    if (!(v > 0)) return m->fail(ESL_MLP_INVALID_ARGUMENT, "input scales must be positive");
  for (float v : m->out_sig)
    if (!(v > 0)) return m->fail(ESL_MLP_INVALID_ARGUMENT, "output scales must be positive");
  MLP_CUDA(m->d_in_mu.ensure(m->n_in));
  MLP_CUDA(m->d_in_sig.ensure(m->n_in));
  MLP_CUDA(m->d_out_mu.ensure(m->n_out));
  MLP_CUDA(m->d_out_sig.ensure(m->n_out));
  MLP_CUDA(cudaMemcpy(m->d_in_mu.p, m->in_mu.data(), m->n_in * 4, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemcpy(m->d_in_sig.p, m->in_sig.data(), m->n_in * 4, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemcpy(m->d_out_mu.p, m->out_mu.data(), m->n_out * 4, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemcpy(m->d_out_sig.p, m->out_sig.data(), m->n_out * 4, cudaMemcpyHostToDevice));
  return ESL_MLP_OK;
}

int32_t esl_mlp_train(esl_mlp* m, const float* d_x, const float* d_y, uint32_t n, uint32_t epochs, uint32_t batch,
                      float lr, float lr_end, uint64_t seed, float* loss_out) {
  if (!m || !d_x || !d_y || n == 0 || batch == 0 || batch % 16) return ESL_MLP_INVALID_ARGUMENT;
  cudaSetDevice(m->device);
  const int B = int(batch);
  if (int32_t rc = ensure_batch(m, B)) return rc;
  MLP_CUDA(m->loss.ensure(1));
  cudaStream_t s = m->stream;
  MLP_CUDA(cudaMemsetAsync(m->gerr.p, 0, 4, s));
  std::mt19937_64 rng(seed);
  std::vector<uint32_t> perm(n);
  for (uint32_t i = 0; i < n; ++i) perm[i] = i;
  const uint32_t n_batches = n / batch;
  if (n_batches == 0) return m->fail(ESL_MLP_INVALID_ARGUMENT, "fewer samples than one batch");
  Layer& last = *m->layers.back();
  for (uint32_t ep = 0; ep < epochs; ++ep) {
    // geometric decay from lr to lr_end over the epochs
    const float lr_ep = (lr_end > 0 && epochs > 1)
                            ? lr * std::pow(lr_end / lr, float(ep) / float(epochs - 1))
                            : lr;
    std::shuffle(perm.begin(), perm.end(), rng);
    MLP_CUDA(cudaMemsetAsync(m->loss.p, 0, 4, s));
    for (uint32_t bi = 0; bi < n_batches; ++bi) {
      MLP_CUDA(cudaMemcpyAsync(m->idx.p, perm.data() + size_t(bi) * batch, batch * 4, cudaMemcpyHostToDevice, s));
      const int kin = m->layers[0]->k;
      scale_rows<<<(B * kin + 255) / 256, 256, 0, s>>>(d_x, m->idx.p, B, m->n_in, kin, m->d_in_mu.p, m->d_in_sig.p,
                                                        m->hb[0]->p, nullptr);
      // targets, standardized: t = (y - out_mu) / out_sig
      scale_rows<<<(B * m->n_out + 255) / 256, 256, 0, s>>>(d_y, m->idx.p, B, m->n_out, m->n_out, m->d_out_mu.p,
                                                             m->d_out_sig.p, nullptr, m->t.p);
      MLP_CUDA(cudaGetLastError());
      if (int32_t rc = forward(m, B)) return rc;
      MLP_CUDA(esl::launch_mse_grad(m->z.back()->p, m->t.p, B, m->n_out, last.n, m->dz.p, m->loss.p, s));
      if (int32_t rc = backward(m, B)) return rc;
      ++m->step;
      for (auto& ly : m->layers) {
        MLP_CUDA(esl::launch_adam(ly->w.p, ly->gw.p, ly->mw.p, ly->vw.p, ly->n, ly->k, lr_ep, m->step, ly->wb.p,
                                  ly->wt.p, ly->n, s));
        MLP_CUDA(esl::launch_adam(ly->b.p, ly->gb.p, ly->mb.p, ly->vb.p, 1, ly->n, lr_ep, m->step, nullptr, nullptr,
                                  0, s));
      }
    }
    if (loss_out) {
      float l = 0;
      MLP_CUDA(cudaMemcpyAsync(&l, m->loss.p, 4, cudaMemcpyDeviceToHost, s));
      MLP_CUDA(cudaStreamSynchronize(s));
      loss_out[ep] = l / float(n_batches);
    }
  }
  return check_gemm_err(m);
}

int32_t esl_mlp_predict(esl_mlp* m, const float* d_x, uint32_t n, float* d_y) {
  if (!m || !d_x || !d_y || n == 0) return ESL_MLP_INVALID_ARGUMENT;
  cudaSetDevice(m->device);
  cudaStream_t s = m->stream;
  const uint32_t chunk = 32768;
  if (int32_t rc = ensure_batch(m, int(chunk))) return rc;
  MLP_CUDA(cudaMemsetAsync(m->gerr.p, 0, 4, s));
  const int kin = m->layers[0]->k;
  const Layer& last = *m->layers.back();
  for (uint32_t r0 = 0; r0 < n; r0 += chunk) {
    const int rows = int(std::min(chunk, n - r0));
    scale_rows<<<(rows * kin + 255) / 256, 256, 0, s>>>(d_x + size_t(r0) * m->n_in, nullptr, rows, m->n_in, kin,
                                                         m->d_in_mu.p, m->d_in_sig.p, m->hb[0]->p, nullptr);
    MLP_CUDA(cudaGetLastError());
    if (int32_t rc = forward(m, rows, false)) return rc;
    unscale_rows<<<(rows * m->n_out + 255) / 256, 256, 0, s>>>(m->z.back()->p, rows, m->n_out, last.n,
                                                                m->d_out_mu.p, m->d_out_sig.p,
                                                                d_y + size_t(r0) * m->n_out);
    MLP_CUDA(cudaGetLastError());
  }
  return check_gemm_err(m);
}

int32_t esl_mlp_gradients(esl_mlp* m, const float* d_x, const float* d_y, uint32_t n, float* loss, float* grads) {
  if (!m || !d_x || !d_y || n == 0 || n % 16) return ESL_MLP_INVALID_ARGUMENT;
  cudaSetDevice(m->device);
  const int B = int(n);
  if (int32_t rc = ensure_batch(m, B)) return rc;
  MLP_CUDA(m->loss.ensure(1));
  cudaStream_t s = m->stream;
  MLP_CUDA(cudaMemsetAsync(m->gerr.p, 0, 4, s));
  MLP_CUDA(cudaMemsetAsync(m->loss.p, 0, 4, s));
  const int kin = m->layers[0]->k;
  scale_rows<<<(B * kin + 255) / 256, 256, 0, s>>>(d_x, nullptr, B, m->n_in, kin, m->d_in_mu.p, m->d_in_sig.p,
                                                    m->hb[0]->p, nullptr);
  scale_rows<<<(B * m->n_out + 255) / 256, 256, 0, s>>>(d_y, nullptr, B, m->n_out, m->n_out, m->d_out_mu.p,
                                                         m->d_out_sig.p, nullptr, m->t.p);
  MLP_CUDA(cudaGetLastError());
  if (int32_t rc = forward(m, B)) return rc;
  MLP_CUDA(esl::launch_mse_grad(m->z.back()->p, m->t.p, B, m->n_out, m->layers.back()->n, m->dz.p, m->loss.p, s));
  if (int32_t rc = backward(m, B)) return rc;
  if (int32_t rc = check_gemm_err(m)) return rc;
  if (loss) MLP_CUDA(cudaMemcpy(loss, m->loss.p, 4, cudaMemcpyDeviceToHost));
  if (grads) {
    size_t at = 0;
    for (auto& ly : m->layers) {
      MLP_CUDA(cudaMemcpy(grads + at, ly->gw.p, size_t(ly->n) * ly->k * 4, cudaMemcpyDeviceToHost));
      at += size_t(ly->n) * ly->k;
      MLP_CUDA(cudaMemcpy(grads + at, ly->gb.p, size_t(ly->n) * 4, cudaMemcpyDeviceToHost));
      at += size_t(ly->n);
    }
  }
  return ESL_MLP_OK;
}

int32_t esl_mlp_shapes(const esl_mlp* m, int* k, int* n, int cap, int* n_layers) {
  if (!m || !n_layers) return ESL_MLP_INVALID_ARGUMENT;
  *n_layers = int(m->layers.size());
  for (int l = 0; l < std::min(cap, *n_layers); ++l) {
    if (k) k[l] = m->layers[l]->k;
    if (n) n[l] = m->layers[l]->n;
  }
  return ESL_MLP_OK;
}

int32_t esl_mlp_weights(esl_mlp* m, float* out) {
  if (!m || !out) return ESL_MLP_INVALID_ARGUMENT;
  cudaSetDevice(m->device);
  MLP_CUDA(cudaStreamSynchronize(m->stream));
  size_t at = 0;
  for (auto& ly : m->layers) {
    MLP_CUDA(cudaMemcpy(out + at, ly->w.p, size_t(ly->n) * ly->k * 4, cudaMemcpyDeviceToHost));
    at += size_t(ly->n) * ly->k;
    MLP_CUDA(cudaMemcpy(out + at, ly->b.p, size_t(ly->n) * 4, cudaMemcpyDeviceToHost));
    at += size_t(ly->n);
  }
  return ESL_MLP_OK;
}

int32_t esl_gemm_bf16_bounded(const void* d_a, int lda, const void* d_b, int ldb, int M, int N, int K,
                              const float* d_bias, float* d_c, int ldc, void* d_h, int ldh, int act,
                              uint32_t wait_rounds) {
  int* err = nullptr;
  if (cudaMalloc(&err, 4) != cudaSuccess) return ESL_MLP_OUT_OF_MEMORY;
  cudaMemset(err, 0, 4);
  cudaError_t e = esl::launch_gemm_bf16(static_cast<const __nv_bfloat16*>(d_a), lda,
                                        static_cast<const __nv_bfloat16*>(d_b), ldb, M, N, K, d_bias, d_c, ldc,
                                        static_cast<__nv_bfloat16*>(d_h), ldh, act, err, nullptr, wait_rounds);
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, err, 4, cudaMemcpyDeviceToHost);
  cudaFree(err);
  if (e == cudaErrorInvalidValue) return ESL_MLP_INVALID_ARGUMENT;
  if (e != cudaSuccess) return ESL_MLP_DEVICE_FAULT;
  return h ? ESL_MLP_TIMEOUT : ESL_MLP_OK;
}

int32_t esl_gemm_bf16(const void* d_a, int lda, const void* d_b, int ldb, int M, int N, int K, const float* d_bias,
                      float* d_c, int ldc, void* d_h, int ldh, int act) {
  return esl_gemm_bf16_bounded(d_a, lda, d_b, ldb, M, N, K, d_bias, d_c, ldc, d_h, ldh, act, 0);
}

}  // extern "C"

// The learned warm start's network on the 5th-generation tensor cores:
// a BF16 GEMM with FP32 accumulation in tensor memory (operand tiles moved
// by the Tensor Memory Accelerator, cp.async.bulk.tensor with the 128-byte
// swizzle, into a ring of shared-memory stages tracked by mbarriers;
// tcgen05.mma issued by one thread, each stage released by tcgen05.commit;
// the accumulator read back with tcgen05.ld), its fused epilogues (bias,
// tanh, BF16 copies), and the small kernels of training (tanh backward,
// transposes, bias gradient, MSE gradient, Adam).
//
// Descriptor layouts (bit positions of the instruction descriptor and the
// shared-memory matrix descriptor) follow the sm100 UMMA definitions;
// encode_idesc and encode_sdesc pack them by hand.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>

#include "mlp.h"

namespace esl {

namespace {

constexpr int kTileM = 128;     // UMMA M (one CTA, cta_group::1)
constexpr int kTileK = 64;      // K per staged chunk (4 MMAs of K = 16)
constexpr int kThreads = 128;   // four warps: warp w owns TMEM lanes 32w..32w+31
constexpr uint32_t kWaitLimit = 1u << 20;  // try_wait rounds before the error flag

// Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and
// B BF16 (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0),
// N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t encode_idesc(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | (uint32_t(kTileM >> 4) << 24);
}

// Shared-memory matrix descriptor of a K-major tile written by TMA with the
// 128-byte swizzle (rows of 64 BF16 = 128 B, 8-row atoms of 1 KB): start
// address >> 4 at bits 0-13, leading byte offset (unused by the swizzled
// K-major form) 16 B at 16-29, stride byte offset 1024 B (one atom) at
// 32-45, version 1 at bits 46-47, base offset 0 (stages are 1 KB aligned),
// layout type 2 (128-byte swizzle) at bits 61-63. The k-th K = 16 slice of a
// stage starts 32 k bytes in.
__device__ __forceinline__ uint64_t encode_sdesc(uint32_t saddr) {
  return uint64_t((saddr >> 4) & 0x3fffu) | (uint64_t(16 >> 4) << 16) | (uint64_t(1024 >> 4) << 32) | (1ull << 46) |
         (2ull << 61);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// One 2-D TMA tile load global -> shared, completing bytes on `bar`.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

constexpr int kMaxStages = 4;

// C = A (M x K, row-major BF16) . B (N x K, row-major BF16)^T with FP32
// accumulation; grid (ceil(M / 128), N / bn), block 128 threads. The
// epilogue adds bias[n] when given, stores the FP32 result to c (ldc) when
// given, and tanh (act = 1) or identity of it as BF16 to h (ldh) when given.
// Rows >= M are read as zero (the TMA box's out-of-bounds fill) and not
// stored; so are K columns past K. K is a multiple of 16, bn a multiple of 16
// in [16, 256].
//
// The pipeline (thread 0): `stages` shared-memory stages of one 64-wide K
// chunk each (A 128 x 64, B bn x 64 BF16). Chunk q's two TMA loads land on
// full[q % stages]; its four MMAs are issued once they have, and their
// completion is committed to empty[q % stages], which frees the stage for
// chunk q + stages. The refill of a stage waits for the MMAs of the chunk
// before the one just issued, so one chunk's MMAs are always queued behind
// the running ones. Every wait is bounded; one that runs out raises err,
// stops the issue, and waits (bounded again) for the loads and MMAs in
// flight before the tensor memory is freed.
__global__ void __launch_bounds__(kThreads) gemm_bf16_tc(const __grid_constant__ CUtensorMap ta,
                                                         const __grid_constant__ CUtensorMap tb, int M, int K, int bn,
                                                         int stages, const float* __restrict__ bias, float* c,
                                                         int ldc, __nv_bfloat16* h, int ldh, int act, int* err,
                                                         uint32_t wait_limit) {
  extern __shared__ unsigned char smem_raw[];
  // stages at a 1 KB boundary (the swizzle atom)
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char* smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t a_bytes = kTileM * kTileK * 2, b_bytes = uint32_t(bn) * kTileK * 2;
  const uint32_t stage_bytes = a_bytes + b_bytes;
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int ok_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * bn;
  uint32_t ncols = 32;
  while (ncols < uint32_t(bn)) ncols <<= 1;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < stages; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[s])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&done)));
    asm volatile("fence.mbarrier_init.release.cluster;");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_slot;

  if (tid == 0) {
    const uint32_t idesc = encode_idesc(uint32_t(bn));
    const uint32_t base = smem_u32(smem);
    const int n_chunks = (K + kTileK - 1) / kTileK;
    int issued = 0, consumed = 0;
    bool ok = true;
    auto issue = [&](int q) {
      const int s = q % stages;
      const uint32_t sa = base + uint32_t(s) * stage_bytes, bar = smem_u32(&full[s]);
      mbar_expect_tx(bar, stage_bytes);
      tma_load_2d(sa, &ta, q * kTileK, m0, bar);
      tma_load_2d(sa + a_bytes, &tb, q * kTileK, n0, bar);
      ++issued;
    };
    for (int q = 0; q < n_chunks && q < stages; ++q) issue(q);
    for (int q = 0; q < n_chunks; ++q) {
      const int s = q % stages;
      if (!mbar_wait(smem_u32(&full[s]), uint32_t(q / stages) & 1u, wait_limit)) {
        ok = false;
        break;
      }
      ++consumed;
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t sa = base + uint32_t(s) * stage_bytes, sb = sa + a_bytes;
      const int kc = min(kTileK, K - q * kTileK);
      for (int j = 0; j < kc / 16; ++j) {
        const uint64_t da = encode_sdesc(sa + uint32_t(j) * 32u);
        const uint64_t db = encode_sdesc(sb + uint32_t(j) * 32u);
        const uint32_t acc = (q > 0 || j > 0) ? 1u : 0u;
        const uint32_t z = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
      }
      umma_commit(smem_u32(&empty[s]));
      // refill the stage of the chunk before this one once its MMAs are done
      const int p = q - 1;
      if (p >= 0 && p + stages < n_chunks) {
        if (!mbar_wait(smem_u32(&empty[p % stages]), uint32_t(p / stages) & 1u, wait_limit)) {
          ok = false;
          break;
        }
        issue(p + stages);
      }
    }
    if (!ok) {
      // loads still in flight land before the stages are reused or freed
      for (int q = consumed; q < issued; ++q) mbar_wait(smem_u32(&full[q % stages]), uint32_t(q / stages) & 1u, kWaitLimit);
    }
    // every MMA issued, complete before the accumulator is read or freed
    umma_commit(smem_u32(&done));
    if (!mbar_wait(smem_u32(&done), 0u, ok ? wait_limit : kWaitLimit)) {
      ok = false;
      mbar_wait(smem_u32(&done), 0u, kWaitLimit);
    }
    ok_flag = ok;
    if (!ok) atomicExch(err, 1);
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const bool ok = ok_flag != 0;

  // epilogue: warp w owns accumulator rows 32w .. 32w + 31 (thread = row in
  // TMEM). Each 32-column block goes through the warp's 32 x 33 float
  // patch of the (now idle) staging buffer, so the global stores run along
  // rows: lane j writes column c0 + j of each row, 128 B per row per store
  // instead of 32 rows of 4 B. The MMAs that read the staging buffer are
  // complete (the last mbarrier wait above). Columns c0 .. c0 + 31 stay
  // inside the allocation: ncols is a power of two >= max(bn, 32).
  float* patch = reinterpret_cast<float*>(smem) + warp * 32 * 33;
  for (int c0 = 0; c0 < bn; c0 += 32) {
    uint32_t r[32];
    const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0);
#pragma unroll
    for (int j = 0; j < 4; ++j)
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
          : "=r"(r[8 * j]), "=r"(r[8 * j + 1]), "=r"(r[8 * j + 2]), "=r"(r[8 * j + 3]), "=r"(r[8 * j + 4]),
            "=r"(r[8 * j + 5]), "=r"(r[8 * j + 6]), "=r"(r[8 * j + 7])
          : "r"(taddr + uint32_t(8 * j)));
    asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
    for (int t = 0; t < 32; ++t) patch[lane * 33 + t] = __uint_as_float(r[t]);
    __syncwarp();
    const int n = n0 + c0 + lane;
    const bool col = c0 + lane < bn;
    const float bv = (bias && col) ? bias[n] : 0.0f;
    for (int rr = 0; rr < 32; ++rr) {
      const int m = m0 + warp * 32 + rr;
      if (m < M && col && ok) {
        const float v = patch[rr * 33 + lane] + bv;
        if (c) c[size_t(m) * ldc + n] = v;
        if (h) h[size_t(m) * ldh + n] = __float2bfloat16_rn(act == 1 ? tanhf(v) : v);
      }
    }
    __syncwarp();
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// dZ = dH * (1 - H^2) for a tanh layer (H stored as BF16); FP32 out and a
// BF16 copy for the next GEMMs.
__global__ void tanh_backward(const float* dh, const __nv_bfloat16* hb, int ldh, const float* zpre, int rows, int cols,
                              int ld, float* dz, __nv_bfloat16* dzb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const int r = i / cols, c = i % cols;
  const float t = tanhf(zpre[size_t(r) * ld + c]);
  const float g = dh[size_t(r) * ld + c] * (1.0f - t * t);
  dz[size_t(r) * ld + c] = g;
  dzb[size_t(r) * ld + c] = __float2bfloat16_rn(g);
  (void)hb;
  (void)ldh;
}

// out (cols x rows, BF16) = in (rows x cols)^T, through a 32 x 32 tile.
template <class T>
__global__ void transpose_to_bf16(const T* in, int rows, int cols, int ldi, __nv_bfloat16* out, int ldo) {
  __shared__ float tile[32][33];
  const int c = blockIdx.x * 32 + threadIdx.x, r0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + j;
    tile[j][threadIdx.x] = (r < rows && c < cols) ? float(in[size_t(r) * ldi + c]) : 0.0f;
  }
  __syncthreads();
  const int oc = r0 + threadIdx.x, orow0 = blockIdx.x * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int orow = orow0 + j;
    if (orow < cols && oc < rows) out[size_t(orow) * ldo + oc] = __float2bfloat16_rn(tile[threadIdx.x][j]);
  }
}

// db[c] = sum over rows of dz[r][c] (one thread per column; rows is a batch).
__global__ void bias_grad(const float* dz, int rows, int cols, int ld, float* db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += dz[size_t(r) * ld + c];
  db[c] = s;
}

// MSE gradient over the real output columns: d = 2 (y - t) / (rows * outs).
__global__ void mse_grad(const float* y, const float* t, int rows, int outs, int ld, float* d, float* loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * ld) return;
  const int r = i / ld, c = i % ld;
  float g = 0.0f;
  if (c < outs) {
    const float e = y[size_t(r) * ld + c] - t[size_t(r) * outs + c];
    g = 2.0f * e / float(rows * outs);
    atomicAdd(loss, e * e / float(rows * outs));
  }
  d[size_t(r) * ld + c] = g;
}

// Adam on FP32 master weights; refreshes the BF16 copy (and its transpose
// when given, for the backward GEMMs).
__global__ void adam_step(float* w, const float* g, float* m, float* v, int rows, int cols, float lr, float b1,
                          float b2, float eps, float c1, float c2, __nv_bfloat16* wb, __nv_bfloat16* wt, int ldt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
  if (wt) {
    const int r = i / cols, c = i % cols;
    wt[size_t(c) * ldt + r] = __float2bfloat16_rn(wi);
  }
}

__global__ void to_bf16(const float* in, int n, __nv_bfloat16* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __float2bfloat16_rn(in[i]);
}

}  // namespace

namespace {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library), looked up once.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The tensor map of a row-major BF16 matrix of `rows` x `cols` (leading
// dimension ld elements, a multiple of 8: 16-byte row strides) read in
// boxes of box_rows x 64 with the 128-byte swizzle; out-of-bounds elements
// read as zero.
cudaError_t bf16_tile_map(CUtensorMap* map, const __nv_bfloat16* base, int rows, int cols, int ld, int box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return cudaErrorNotSupported;
  const cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(ld) * 2};
  const cuuint32_t box[2] = {cuuint32_t(kTileK), cuuint32_t(box_rows)};
  const cuuint32_t elem[2] = {1, 1};
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims, strides,
                            box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_gemm_bf16(const __nv_bfloat16* a, int lda, const __nv_bfloat16* b, int ldb, int M, int N, int K,
                             const float* bias, float* c, int ldc, __nv_bfloat16* h, int ldh, int act, int* err,
                             cudaStream_t s, uint32_t wait_rounds) {
  if (M <= 0 || N <= 0 || K <= 0 || K % 16 || N % 16 || lda % 8 || ldb % 8) return cudaErrorInvalidValue;
  // TMA: 16-byte aligned bases (the strides are, by lda, ldb)
  if ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15u) return cudaErrorInvalidValue;
  int bn = N <= 256 ? N : 128;
  while (N % bn) bn -= 16;
  CUtensorMap ta, tb;
  cudaError_t e = bf16_tile_map(&ta, a, M, K, lda, kTileM);
  if (e != cudaSuccess) return e;
  e = bf16_tile_map(&tb, b, N, K, ldb, bn);
  if (e != cudaSuccess) return e;
  // Stages of A (16 KB) and B (bn x 64 BF16, at most 32 KB): three when B is
  // at most 128 rows, else two, which keeps a CTA under 100 KB so two share
  // an SM (their tensor-memory allocations, at most 256 columns each, fit
  // in its 512); 1 KB more for the stages' alignment.
  const int stages = bn <= 128 ? 3 : 2;
  const size_t stage_bytes = size_t(kTileM) * kTileK * 2 + size_t(bn) * kTileK * 2;
  const size_t smem = std::max<size_t>(100 * 1024, size_t(stages) * stage_bytes + 1024);
  e = cudaFuncSetAttribute(gemm_bf16_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  dim3 grid((M + kTileM - 1) / kTileM, N / bn);
  gemm_bf16_tc<<<grid, kThreads, smem, s>>>(ta, tb, M, K, bn, stages, bias, c, ldc, h, ldh, act, err,
                                            wait_rounds == 0 ? kWaitLimit : wait_rounds == ~0u ? 0u : wait_rounds);
  return cudaGetLastError();
}

cudaError_t launch_tanh_backward(const float* dh, const float* zpre, int rows, int cols, int ld, float* dz,
                                 __nv_bfloat16* dzb, cudaStream_t s) {
  const int n = rows * cols;
  tanh_backward<<<(n + 255) / 256, 256, 0, s>>>(dh, nullptr, 0, zpre, rows, cols, ld, dz, dzb);
  return cudaGetLastError();
}

cudaError_t launch_transpose_f32(const float* in, int rows, int cols, int ldi, __nv_bfloat16* out, int ldo,
                                 cudaStream_t s) {
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_to_bf16<float><<<grid, block, 0, s>>>(in, rows, cols, ldi, out, ldo);
  return cudaGetLastError();
}

cudaError_t launch_transpose_bf16(const __nv_bfloat16* in, int rows, int cols, int ldi, __nv_bfloat16* out, int ldo,
                                  cudaStream_t s) {
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_to_bf16<__nv_bfloat16><<<grid, block, 0, s>>>(in, rows, cols, ldi, out, ldo);
  return cudaGetLastError();
}

cudaError_t launch_bias_grad(const float* dz, int rows, int cols, int ld, float* db, cudaStream_t s) {
  bias_grad<<<(cols + 127) / 128, 128, 0, s>>>(dz, rows, cols, ld, db);
  return cudaGetLastError();
}

cudaError_t launch_mse_grad(const float* y, const float* t, int rows, int outs, int ld, float* d, float* loss,
                            cudaStream_t s) {
  const int n = rows * ld;
  mse_grad<<<(n + 255) / 256, 256, 0, s>>>(y, t, rows, outs, ld, d, loss);
  return cudaGetLastError();
}

cudaError_t launch_adam(float* w, const float* g, float* m, float* v, int rows, int cols, float lr, int step,
                        __nv_bfloat16* wb, __nv_bfloat16* wt, int ldt, cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  float c1 = 1.0f, c2 = 1.0f;
  for (int i = 0; i < step; ++i) {
    c1 *= b1;
    c2 *= b2;
  }
  const int n = rows * cols;
  adam_step<<<(n + 255) / 256, 256, 0, s>>>(w, g, m, v, rows, cols, lr, b1, b2, 1e-8f, 1.0f - c1, 1.0f - c2, wb, wt,
                                            ldt);
  return cudaGetLastError();
}

cudaError_t launch_to_bf16(const float* in, int n, __nv_bfloat16* out, cudaStream_t s) {
  to_bf16<<<(n + 255) / 256, 256, 0, s>>>(in, n, out);
  return cudaGetLastError();
}

}  // namespace esl

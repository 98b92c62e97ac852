// mlp.cu -- the network of the learned ZF initialisers: a 3-layer MLP
// (n_in -> width -> width -> n_out, ReLU after the first two layers) with
// FP32 master weights; every product takes BF16 weights and BF16
// activations (or upstream gradients) with FP32 accumulation, the training
// products on the tensor cores (tcgen05.mma), trained by the project's own
// forward, backward and Adam kernels.  No counterpart in the reference.
//
// The training loss is the quadratic form the initialiser needs: each sample
// carries a symmetric O x O matrix A, a vector b and a scalar c, and for the
// network output y the loss is y^T A y - 2 b^T y + c (the squared Frobenius
// distance of the blended initial iterate to the exact inverse, normalised;
// see lzf.cu), averaged over the batch.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <random>
#include <vector>

#include "common.cuh"
#include "tc.cuh"

namespace mb {
namespace {

// the activations enter every product as BF16, like the weights
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float ldf(const float *p, size_t i) { return p[i]; }
__device__ __forceinline__ float ldf(const __nv_bfloat16 *p, size_t i) { return __bfloat162float(p[i]); }

// Every product of the network runs on the tensor cores (tcgen05.mma,
// kind::f16): BF16 operands, FP32 accumulation in tensor memory.
//   C(m, n) = sum_k A(m, k) B(k, n), A(m, k) = TRA ? A[k lda + m] : A[m lda + k],
//   B(k, n) = TRB ? B[n ldb + k] : B[k ldb + n]
// A CTA of 128 threads owns a 128 x NT tile of C (NT = 64, 128 or 256) over
// the k range of its split; the threads convert 64-wide k chunks of A and B
// to BF16 and store them in the K-major canonical layout (8-row groups 1024 B
// apart, 8-element k chunks 128 B apart), two stages deep, and thread 0
// issues the four K = 16 MMAs of each chunk.  Thread t then reads row t of
// the tile from TMEM lane t.  Epilogue as the network needs it: + bias[n],
// then times (mask(m, n) > 0) (the ReLU derivative), or ReLU with the
// pre-activation kept in zout; accumulate adds to C.  With split-K the
// splits write their partial sums to `partial` [split][M][N] and a second
// kernel adds them in a fixed order and applies the epilogue
// (deterministic).
constexpr int kGM = 128, kGK = 64, kGThreads = 128;

__device__ __forceinline__ uint32_t gkmaj(uint32_t row, uint32_t kk) {
  return (row / 8) * 1024 + (kk / 8) * 128 + (row % 8) * 16 + (kk % 8) * 2;
}

// rows x 64 k chunk of a BF16 operand into shared memory: element (row, k)
// of the source at trans ? src[k ld + row] : src[row ld + k], zero outside
// [0, nrow) x [0, nk).  Consecutive threads take consecutive rows of one
// 8-element k chunk: their 16-byte stores fill whole 128-byte core-matrix
// rows (no bank conflicts), and their loads are coalesced across threads
// (row-contiguous source) or a whole 32-byte sector each (k-contiguous).
template <typename T>
__device__ __forceinline__ void load_chunk(uint8_t *dst, const T *src, int ld, int trans, int row0, int nrow,
                                           int k0, int nk, int rows) {
  const int chunks = rows * (kGK / 8);
  for (int e = threadIdx.x; e < chunks; e += kGThreads) {
    const int r = e % rows, kc = e / rows;
    const int gr = row0 + r, gk = k0 + kc * 8;
    float v[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const bool in = gr < nrow && gk + j < nk;
      v[j] = in ? ldf(src, trans ? (size_t)(gk + j) * ld + gr : (size_t)gr * ld + gk + j) : 0.f;
    }
    uint32_t w[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
      w[j] = *reinterpret_cast<const uint32_t *>(&h);
    }
    *reinterpret_cast<uint4 *>(dst + gkmaj(r, kc * 8)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

__device__ __forceinline__ float epi(float v, int m, int n, int ldc, float *C, const float *bias, const float *mask,
                                     float *zout, int relu, int accumulate) {
  const size_t o = (size_t)m * ldc + n;
  v += bias ? bias[n] : 0.f;
  if (mask && !(mask[o] > 0.f)) v = 0.f;
  if (relu) {
    if (zout) zout[o] = v;
    v = fmaxf(v, 0.f);
  }
  return accumulate ? C[o] + v : v;
}

template <typename TA, typename TB>
__global__ void __launch_bounds__(kGThreads) gemm_tc_kernel(int M, int N, int K, const TA *A, int lda, int tra,
                                                            const TB *B, int ldb, int trb, float *C, int ldc,
                                                            const float *bias, const float *mask, float *zout,
                                                            int relu, int accumulate, int NT, int k_split,
                                                            float *partial, int *err) {
  extern __shared__ __align__(1024) uint8_t gsm[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid / 32;
  const int n0 = blockIdx.x * NT, m0 = blockIdx.y * kGM;
  const int kb = blockIdx.z * k_split, ke = min(K, kb + k_split);
  const uint32_t a_bytes = kGM * kGK * 2, b_bytes = (uint32_t)NT * kGK * 2;
  uint8_t *stage[2] = {gsm, gsm + a_bytes + b_bytes};
  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
    tc::fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(&tmem_slot, (uint32_t)NT);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = tc::idesc_bf16(kGM, (uint32_t)NT, false, false);
  const int nchunks = (ke - kb + kGK - 1) / kGK;
  bool ok = true;
  for (int c = 0; c < nchunks; c++) {
    const int s = c & 1;
    // the stage's previous chunk (c - 2) must have been multiplied
    if (c >= 2 && !tc::mbar_wait(&bar[s], ((c - 2) >> 1) & 1)) ok = false;
    if (__syncthreads_or(!ok)) break;
    // A's rows are m: A(m, k) sits at A[k lda + m] exactly when TRA; B's
    // rows are n: B(k, n) sits at B[k ldb + n] exactly when not TRB
    load_chunk(stage[s], A, lda, tra, m0, M, kb + c * kGK, ke, kGM);
    load_chunk(stage[s] + a_bytes, B, ldb, !trb, n0, N, kb + c * kGK, ke, NT);
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t a0 = tc::smem_u32(stage[s]), b0 = a0 + a_bytes;
#pragma unroll
      for (int ks = 0; ks < kGK / 16; ks++)
        tc::mma_f16(tmem, tc::smem_desc(a0 + ks * 256, 128, 1024), tc::smem_desc(b0 + ks * 256, 128, 1024), idesc,
                    (c | ks) != 0);
      tc::mma_commit(&bar[s]);
    }
  }
  // the last chunk's commit covers every MMA issued before it
  if (ok && nchunks > 0 && !tc::mbar_wait(&bar[(nchunks - 1) & 1], ((nchunks - 1) >> 1) & 1)) ok = false;
  if (__syncthreads_or(!ok)) {
    if (tid == 0 && err) atomicOr(err, tc::kErrTimeout);
  } else {
    tc::fence_after_sync();
    const int m = m0 + tid;
    for (int c16 = 0; c16 < NT / 16; c16++) {
      float v[16];
      if (nchunks > 0) {
        tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c16 * 16, v);
      } else {
#pragma unroll
        for (int j = 0; j < 16; j++) v[j] = 0.f;
      }
      if (m >= M) continue;
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const int n = n0 + c16 * 16 + j;
        if (n >= N) break;
        if (partial)
          partial[((size_t)blockIdx.z * M + m) * N + n] = v[j];
        else
          C[(size_t)m * ldc + n] = epi(v[j], m, n, ldc, C, bias, mask, zout, relu, accumulate);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, (uint32_t)NT);
}

// C = epilogue(sum over the splits of partial[s][M][N]), in split order
__global__ void splitk_reduce_kernel(int M, int N, int splits, const float *partial, float *C, int ldc,
                                     const float *bias, const float *mask, float *zout, int relu, int accumulate) {
  const size_t total = (size_t)M * N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    float v = 0.f;
    for (int s = 0; s < splits; s++) v += partial[(size_t)s * total + e];
    const int m = (int)(e / N), n = (int)(e % N);
    C[(size_t)m * ldc + n] = epi(v, m, n, ldc, C, bias, mask, zout, relu, accumulate);
  }
}

constexpr int kMaxSplits = 16;

// the host side of one product; partial: split-K scratch of kMaxSplits * M * N
// floats (nullable: no split-K)
template <typename TA, typename TB, bool TRA, bool TRB>
cudaError_t gemm(int M, int N, int K, const TA *A, int lda, const TB *B, int ldb, float *C, int ldc,
                 const float *bias, const float *mask, float *zout, int relu, int accumulate, cudaStream_t st,
                 float *partial = nullptr, int *err = nullptr) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  const int NT = N <= 64 ? 64 : N <= 128 ? 128 : 256;
  const size_t smem = 2 * ((size_t)kGM * kGK * 2 + (size_t)NT * kGK * 2);
  static std::atomic<uint64_t> configured{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(configured.load() & bit)) {
    e = cudaFuncSetAttribute(gemm_tc_kernel<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * ((size_t)kGM * kGK * 2 + 256 * kGK * 2)));
    if (e != cudaSuccess) return e;
    configured.fetch_or(bit);
  }
  const int gx = (N + NT - 1) / NT, gy = (M + kGM - 1) / kGM;
  // few output tiles over a long reduction (the weight gradients: K is the
  // batch): split K so that the launch fills the GPU
  int splits = 1;
  if (partial && gx * gy < 32 && K >= 4 * kGK)
    splits = std::min(kMaxSplits, std::max(1, K / (4 * kGK)));
  const int k_split = ((K + splits - 1) / splits + kGK - 1) / kGK * kGK;
  splits = std::max(1, (K + k_split - 1) / k_split);
  gemm_tc_kernel<TA, TB><<<dim3(gx, gy, splits), kGThreads, smem, st>>>(
      M, N, K, A, lda, TRA ? 1 : 0, B, ldb, TRB ? 1 : 0, C, ldc, bias, mask, zout, relu, accumulate, NT, k_split,
      splits > 1 ? partial : nullptr, err);
  e = cudaGetLastError();
  if (e != cudaSuccess || splits == 1) return e;
  const size_t total = (size_t)M * N;
  const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 8);
  splitk_reduce_kernel<<<blocks, 256, 0, st>>>(M, N, splits, partial, C, ldc, bias, mask, zout, relu, accumulate);
  return cudaGetLastError();
}

// out[n] = sum_m X[m][n] (bias gradients), X row-major [M][N]
__global__ void colsum_kernel(const float *X, int M, int N, float *out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; m++) s += X[(size_t)m * N + n];
  out[n] = s;
}

// per sample: L = y^T A y - 2 b^T y + c; dY = 2 (A y - b) / B; the batch
// mean of L is accumulated into *loss (zeroed by the caller)
__global__ void quad_loss_kernel(const float *Y, const float *A, const float *b, const float *c,
                                 int B, int O, float *dY, float *loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float li = 0.f;
  if (i < B) {
    const float *y = Y + (size_t)i * O;
    const float *Ai = A + (size_t)i * O * O;
    const float *bi = b + (size_t)i * O;
    float quad = 0.f, lin = 0.f;
    for (int r = 0; r < O; r++) {
      float ay = 0.f;
      for (int q = 0; q < O; q++) ay = fmaf(Ai[r * O + q], y[q], ay);
      quad = fmaf(y[r], ay, quad);
      lin = fmaf(bi[r], y[r], lin);
      dY[(size_t)i * O + r] = 2.f * (ay - bi[r]) / (float)B;
    }
    li = (quad - 2.f * lin + (c ? c[i] : 0.f)) / (float)B;
  }
  for (int o = 16; o > 0; o >>= 1) li += __shfl_xor_sync(0xffffffffu, li, o);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, li);
}

__global__ void adam_kernel(float *p, const float *g, float *m, float *v, uint64_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Inference: all three layers in one kernel, ROWS samples per CTA with the
// activations in shared memory; thread n of a layer owns output column n
// (coalesced BF16 weight loads, activations broadcast from shared memory).
template <int ROWS>
__global__ void __launch_bounds__(256) mlp_infer_kernel(const float *x, int B, int I, int W, int O,
                                                        const __nv_bfloat16 *W1, const float *b1,
                                                        const __nv_bfloat16 *W2, const float *b2,
                                                        const __nv_bfloat16 *W3, const float *b3,
                                                        float *y) {
  extern __shared__ __align__(16) float msm[];
  // a0 padded to a multiple of 4 floats so that a1 / a2 rows are 16-byte aligned
  float *a0 = msm, *a1 = a0 + ((ROWS * I + 3) & ~3), *a2 = a1 + ROWS * W;
  const int r0 = blockIdx.x * ROWS, nr = min(ROWS, B - r0);
  for (int e = threadIdx.x; e < ROWS * I; e += blockDim.x) {
    const int r = e / I;
    a0[e] = r < nr ? bf16r(x[(size_t)(r0 + r) * I + e % I]) : 0.f;
  }
  __syncthreads();
  // hidden layers: relu(a W + b)
  for (int layer = 0; layer < 2; layer++) {
    const float *ain = layer == 0 ? a0 : a1;
    float *aout = layer == 0 ? a1 : a2;
    const __nv_bfloat16 *Wl = layer == 0 ? W1 : W2;
    const float *bl = layer == 0 ? b1 : b2;
    const int K = layer == 0 ? I : W;
    for (int n = threadIdx.x; n < W; n += blockDim.x) {
      float acc[ROWS];
#pragma unroll
      for (int r = 0; r < ROWS; r++) acc[r] = bl[n];
      for (int k0 = 0; k0 < K; k0 += 16) {
        // sixteen weight loads in flight, then their products
        float w[16];
#pragma unroll
        for (int j = 0; j < 16; j++)
          w[j] = k0 + j < K ? __bfloat162float(Wl[(size_t)(k0 + j) * W + n]) : 0.f;
        if ((K & 15) == 0) {
          // activations four at a time (16-byte shared-memory loads)
#pragma unroll
          for (int j = 0; j < 16; j += 4) {
#pragma unroll
            for (int r = 0; r < ROWS; r++) {
              const float4 a4 = *reinterpret_cast<const float4 *>(ain + r * K + k0 + j);
              acc[r] = fmaf(a4.x, w[j], acc[r]);
              acc[r] = fmaf(a4.y, w[j + 1], acc[r]);
              acc[r] = fmaf(a4.z, w[j + 2], acc[r]);
              acc[r] = fmaf(a4.w, w[j + 3], acc[r]);
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; j++) {
            if (k0 + j >= K) break;
#pragma unroll
            for (int r = 0; r < ROWS; r++) acc[r] = fmaf(ain[r * K + k0 + j], w[j], acc[r]);
          }
        }
      }
#pragma unroll
      for (int r = 0; r < ROWS; r++) aout[r * W + n] = bf16r(fmaxf(acc[r], 0.f));
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nr * O; e += blockDim.x) {
    const int r = e / O, o = e % O;
    float acc = b3[o];
    for (int k0 = 0; k0 < W; k0 += 16) {
      float w[16];
#pragma unroll
      for (int j = 0; j < 16; j++) w[j] = k0 + j < W ? __bfloat162float(W3[(size_t)(k0 + j) * O + o]) : 0.f;
#pragma unroll
      for (int j = 0; j < 16; j++)
        if (k0 + j < W) acc = fmaf(a2[r * W + k0 + j], w[j], acc);
    }
    y[(size_t)(r0 + r) * O + o] = acc;
  }
}

// Inference with every weight staged once per CTA in shared memory (16-byte
// loads, all in flight together), then ROWS samples at a time through the
// three layers; CTAs walk the row blocks blockIdx.x, + gridDim.x, ...
// ws holds W1 [I][W], W2 [W][W], W3 [W][O] (BF16) back to back.
template <int ROWS>
__global__ void __launch_bounds__(256) mlp_infer_smem_kernel(const float *x, int B, int I, int W, int O,
                                                             const __nv_bfloat16 *W1, const __nv_bfloat16 *W2,
                                                             const __nv_bfloat16 *W3, const float *b1,
                                                             const float *b2, const float *b3, float *y,
                                                             int *err) {
  extern __shared__ __align__(16) unsigned char ism[];
  const size_t n1 = (size_t)I * W, n2 = (size_t)W * W, n3 = (size_t)W * O;
  const size_t nw = (n1 + n2 + n3 + 7) & ~(size_t)7;
  __nv_bfloat16 *ws = reinterpret_cast<__nv_bfloat16 *>(ism);
  float *a0 = reinterpret_cast<float *>(ism + nw * 2);
  float *a1 = a0 + ((ROWS * I + 3) & ~3), *a2 = a1 + ROWS * W;
  // stage the weights with three bulk copies (each block a multiple of 16
  // bytes and 16-byte aligned: W % 8 == 0, checked by the launcher)
  __shared__ __align__(8) uint64_t wbar;
  __shared__ int wok;
  if (threadIdx.x == 0) {
    tc::mbar_init(&wbar, 1);
    tc::fence_mbar_init();
    tc::mbar_arrive_expect_tx(&wbar, (uint32_t)((n1 + n2 + n3) * 2));
    tc::bulk_g2s(ws, W1, (uint32_t)(n1 * 2), &wbar);
    tc::bulk_g2s(ws + n1, W2, (uint32_t)(n2 * 2), &wbar);
    tc::bulk_g2s(ws + n1 + n2, W3, (uint32_t)(n3 * 2), &wbar);
    wok = tc::mbar_wait(&wbar, 0) ? 1 : 0;
  }
  __syncthreads();
  if (!wok) {
    if (threadIdx.x == 0 && err) atomicOr(err, tc::kErrTimeout);
    return;
  }
  const __nv_bfloat16 *s1 = ws, *s2 = ws + n1, *s3 = ws + n1 + n2;
  for (int r0 = blockIdx.x * ROWS; r0 < B; r0 += gridDim.x * ROWS) {
    const int nr = min(ROWS, B - r0);
    for (int e = threadIdx.x; e < ROWS * I; e += blockDim.x) {
      const int r = e / I;
      a0[e] = r < nr ? bf16r(x[(size_t)(r0 + r) * I + e % I]) : 0.f;
    }
    __syncthreads();
    for (int layer = 0; layer < 2; layer++) {
      const float *ain = layer == 0 ? a0 : a1;
      float *aout = layer == 0 ? a1 : a2;
      const __nv_bfloat16 *Wl = layer == 0 ? s1 : s2;
      const float *bl = layer == 0 ? b1 : b2;
      const int K = layer == 0 ? I : W;
      for (int n = threadIdx.x; n < W; n += blockDim.x) {
        float acc[ROWS];
#pragma unroll
        for (int r = 0; r < ROWS; r++) acc[r] = bl[n];
        int k = 0;
        if ((K & 3) == 0) {
          // four activations per 16-byte shared-memory load
          for (; k < K; k += 4) {
            const float w0 = __bfloat162float(Wl[(size_t)k * W + n]);
            const float w1 = __bfloat162float(Wl[(size_t)(k + 1) * W + n]);
            const float w2 = __bfloat162float(Wl[(size_t)(k + 2) * W + n]);
            const float w3 = __bfloat162float(Wl[(size_t)(k + 3) * W + n]);
#pragma unroll
            for (int r = 0; r < ROWS; r++) {
              const float4 a4 = *reinterpret_cast<const float4 *>(ain + r * K + k);
              acc[r] = fmaf(a4.x, w0, acc[r]);
              acc[r] = fmaf(a4.y, w1, acc[r]);
              acc[r] = fmaf(a4.z, w2, acc[r]);
              acc[r] = fmaf(a4.w, w3, acc[r]);
            }
          }
        }
        for (; k < K; k++) {
          const float w = __bfloat162float(Wl[(size_t)k * W + n]);
#pragma unroll
          for (int r = 0; r < ROWS; r++) acc[r] = fmaf(ain[r * K + k], w, acc[r]);
        }
#pragma unroll
        for (int r = 0; r < ROWS; r++) aout[r * W + n] = bf16r(fmaxf(acc[r], 0.f));
      }
      __syncthreads();
    }
    for (int e = threadIdx.x; e < nr * O; e += blockDim.x) {
      const int r = e / O, o = e % O;
      float acc = b3[o];
      for (int k = 0; k < W; k++) acc = fmaf(a2[r * W + k], __bfloat162float(s3[(size_t)k * O + o]), acc);
      y[(size_t)(r0 + r) * O + o] = acc;
    }
    __syncthreads();
  }
}

__global__ void to_bf16_kernel(const float *x, __nv_bfloat16 *y, uint64_t n) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

}  // namespace
}  // namespace mb

using namespace mb;

struct mb_mlp {
  uint32_t n_in, width, n_out, max_batch;
  uint64_t n_params;
  // flat FP32 layout: W1 [n_in][width], b1, W2 [width][width], b2, W3 [width][n_out], b3
  uint64_t off[6];
  float *p, *g, *m, *v;        // params, grads, Adam moments
  __nv_bfloat16 *wb;           // BF16 copies of p (all entries; only W* are read)
  float *z1, *h1, *z2, *h2, *y, *dy, *d2, *d1;  // activations and their gradients
  float *part;                 // split-K partial sums of the weight gradients
  uint32_t step;
};

static cudaError_t mlp_refresh_bf16(mb_mlp *n, cudaStream_t st) {
  const unsigned blocks = (unsigned)((n->n_params + 255) / 256);
  to_bf16_kernel<<<blocks, 256, 0, st>>>(n->p, n->wb, n->n_params);
  return cudaGetLastError();
}

extern "C" mb_status mb_mlp_destroy(mb_mlp *n) {
  if (!n) return MB_BAD_ARG;
  for (void *q : {(void *)n->p, (void *)n->g, (void *)n->m, (void *)n->v, (void *)n->wb,
                  (void *)n->z1, (void *)n->h1, (void *)n->z2, (void *)n->h2, (void *)n->y,
                  (void *)n->dy, (void *)n->d2, (void *)n->d1, (void *)n->part})
    cudaFree(q);
  delete n;
  return MB_OK;
}

extern "C" mb_status mb_mlp_create(uint32_t n_in, uint32_t width, uint32_t n_out,
                                   uint32_t max_batch, uint64_t seed, mb_mlp **out) {
  if (!out) return MB_BAD_ARG;
  *out = nullptr;
  if (n_in == 0 || width == 0 || n_out == 0 || max_batch == 0 || n_in > 4096 || width > 4096 ||
      n_out > 64)
    return MB_BAD_SHAPE;
  mb_mlp *n = new mb_mlp();
  n->n_in = n_in;
  n->width = width;
  n->n_out = n_out;
  n->max_batch = max_batch;
  const uint64_t sizes[6] = {(uint64_t)n_in * width, width, (uint64_t)width * width, width,
                             (uint64_t)width * n_out, n_out};
  uint64_t o = 0;
  for (int i = 0; i < 6; i++) {
    n->off[i] = o;
    o += sizes[i];
  }
  n->n_params = o;
  mb_status st = MB_OK;
  auto alloc = [&](void **q, size_t bytes) {
    if (st != MB_OK) return;
    cudaError_t e = cudaMalloc(q, bytes);
    if (e != cudaSuccess) st = record_error(e);
  };
  const size_t P = sizeof(float) * o;
  alloc((void **)&n->p, P);
  alloc((void **)&n->g, P);
  alloc((void **)&n->m, P);
  alloc((void **)&n->v, P);
  alloc((void **)&n->wb, sizeof(__nv_bfloat16) * o);
  const size_t BW = sizeof(float) * (size_t)max_batch * width;
  alloc((void **)&n->z1, BW);
  alloc((void **)&n->h1, BW);
  alloc((void **)&n->z2, BW);
  alloc((void **)&n->h2, BW);
  alloc((void **)&n->d2, BW);
  alloc((void **)&n->d1, BW);
  alloc((void **)&n->y, sizeof(float) * (size_t)max_batch * n_out);
  alloc((void **)&n->dy, sizeof(float) * (size_t)max_batch * n_out);
  alloc((void **)&n->part, sizeof(float) * kMaxSplits * (size_t)std::max(n_in, width) * std::max(width, n_out));
  if (st == MB_OK) {
    // He-normal hidden layers; the output layer starts at zero weights so the
    // untrained network returns its bias (set by the caller)
    std::vector<float> h(o, 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    const float s1 = std::sqrt(2.f / n_in), s2 = std::sqrt(2.f / width);
    for (uint64_t i = 0; i < sizes[0]; i++) h[n->off[0] + i] = s1 * nd(rng);
    for (uint64_t i = 0; i < sizes[2]; i++) h[n->off[2] + i] = s2 * nd(rng);
    cudaError_t e = cudaMemcpy(n->p, h.data(), P, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(n->m, 0, P);
    if (e == cudaSuccess) e = cudaMemset(n->v, 0, P);
    if (e == cudaSuccess) e = cudaMemset(n->g, 0, P);
    if (e == cudaSuccess) e = mlp_refresh_bf16(n, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) st = record_error(e);
  }
  if (st != MB_OK) {
    mb_mlp_destroy(n);
    return st;
  }
  *out = n;
  return MB_OK;
}

extern "C" mb_status mb_mlp_num_params(const mb_mlp *n, uint64_t *count) {
  if (!n || !count) return MB_BAD_ARG;
  *count = n->n_params;
  return MB_OK;
}

extern "C" mb_status mb_mlp_get_params(const mb_mlp *n, float *host) {
  if (!n || !host) return MB_BAD_ARG;
  MB_CUDA_TRY(cudaMemcpy(host, n->p, sizeof(float) * n->n_params, cudaMemcpyDeviceToHost));
  return MB_OK;
}

extern "C" mb_status mb_mlp_get_grads(const mb_mlp *n, float *host) {
  if (!n || !host) return MB_BAD_ARG;
  MB_CUDA_TRY(cudaMemcpy(host, n->g, sizeof(float) * n->n_params, cudaMemcpyDeviceToHost));
  return MB_OK;
}

extern "C" mb_status mb_mlp_set_params(mb_mlp *n, const float *host) {
  if (!n || !host) return MB_BAD_ARG;
  const size_t P = sizeof(float) * n->n_params;
  MB_CUDA_TRY(cudaMemcpy(n->p, host, P, cudaMemcpyHostToDevice));
  MB_CUDA_TRY(cudaMemset(n->m, 0, P));
  MB_CUDA_TRY(cudaMemset(n->v, 0, P));
  n->step = 0;
  MB_CUDA_TRY(mlp_refresh_bf16(n, nullptr));
  MB_CUDA_TRY(cudaDeviceSynchronize());
  return MB_OK;
}

// forward into n->y (and the activations), BF16 weights, FP32 accumulation
static cudaError_t mlp_fwd(mb_mlp *n, const float *x, uint32_t B, float *y, cudaStream_t st) {
  const int I = n->n_in, W = n->width, O = n->n_out;
  const __nv_bfloat16 *wb = n->wb;
  int *err = device_tables() ? device_tables()->err : nullptr;
  cudaError_t e = gemm<float, __nv_bfloat16, false, false>(B, W, I, x, I, wb + n->off[0], W, n->h1, W,
                                                          n->p + n->off[1], nullptr, n->z1, 1, 0, st, nullptr, err);
  if (e == cudaSuccess)
    e = gemm<float, __nv_bfloat16, false, false>(B, W, W, n->h1, W, wb + n->off[2], W, n->h2, W,
                                                n->p + n->off[3], nullptr, n->z2, 1, 0, st, nullptr, err);
  if (e == cudaSuccess)
    e = gemm<float, __nv_bfloat16, false, false>(B, O, W, n->h2, W, wb + n->off[4], O, y, O,
                                                n->p + n->off[5], nullptr, nullptr, 0, 0, st, nullptr, err);
  return e;
}

extern "C" mb_status mb_mlp_forward(mb_mlp *n, const float *x, uint32_t batch, float *y,
                                    void *stream) {
  if (!n || !x || !y) return MB_BAD_ARG;
  if (batch == 0) return MB_OK;
  constexpr int kRows = 8;
  const __nv_bfloat16 *wb = n->wb;
  {
    // weights resident in shared memory when they fit (one CTA per SM)
    const size_t nw = ((size_t)n->n_in * n->width + (size_t)n->width * n->width +
                       (size_t)n->width * n->n_out + 7) & ~(size_t)7;
    const size_t smem = nw * 2 + sizeof(float) * (((kRows * n->n_in + 3) & ~3u) + 2 * kRows * n->width);
    int dev = 0, maxs = 0, sms = 0;
    MB_CUDA_TRY(cudaGetDevice(&dev));
    MB_CUDA_TRY(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    MB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (smem + 1024 <= (size_t)maxs && n->width % 8 == 0) {
      static std::atomic<uint64_t> configured{0};
      const uint64_t bit = 1ull << (dev & 63);
      if (!(configured.load() & bit)) {
        MB_CUDA_TRY(cudaFuncSetAttribute(mlp_infer_smem_kernel<kRows>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, maxs - 1024));
        configured.fetch_or(bit);
      }
      const unsigned grid = (unsigned)std::min<uint64_t>((batch + kRows - 1) / kRows, (uint64_t)sms);
      mlp_infer_smem_kernel<kRows><<<grid, 256, smem, as_stream(stream)>>>(
          x, (int)batch, (int)n->n_in, (int)n->width, (int)n->n_out, wb + n->off[0], wb + n->off[2],
          wb + n->off[4], n->p + n->off[1], n->p + n->off[3], n->p + n->off[5], y,
          device_tables() ? device_tables()->err : nullptr);
      MB_CUDA_TRY(cudaGetLastError());
      return MB_OK;
    }
  }
  const size_t smem = sizeof(float) * (((kRows * n->n_in + 3) & ~3u) + 2 * kRows * n->width);
  if (smem > 48 * 1024) {
    // wide networks: the tiled products of the training path
    if (batch > n->max_batch) return MB_BAD_SHAPE;
    MB_CUDA_TRY(mlp_fwd(n, x, batch, y, as_stream(stream)));
    return MB_OK;
  }
  mlp_infer_kernel<kRows><<<(batch + kRows - 1) / kRows, 256, smem, as_stream(stream)>>>(
      x, (int)batch, (int)n->n_in, (int)n->width, (int)n->n_out, wb + n->off[0], n->p + n->off[1],
      wb + n->off[2], n->p + n->off[3], wb + n->off[4], n->p + n->off[5], y);
  MB_CUDA_TRY(cudaGetLastError());
  return MB_OK;
}

extern "C" mb_status mb_mlp_loss_grad(mb_mlp *n, const float *x, const float *A, const float *b,
                                      const float *c, uint32_t batch, float *loss, void *stream) {
  if (!n || !x || !A || !b) return MB_BAD_ARG;
  if (batch == 0 || batch > n->max_batch) return MB_BAD_SHAPE;
  cudaStream_t st = as_stream(stream);
  const int I = n->n_in, W = n->width, O = n->n_out, B = (int)batch;
  const __nv_bfloat16 *wb = n->wb;
  float *g = n->g;
  MB_CUDA_TRY(mlp_fwd(n, x, batch, n->y, st));
  if (loss) MB_CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(float), st));
  quad_loss_kernel<<<(B + 255) / 256, 256, 0, st>>>(n->y, A, b, c, B, O, n->dy, loss);
  MB_CUDA_TRY(cudaGetLastError());
  int *err = device_tables() ? device_tables()->err : nullptr;
  // layer 3: dW3 = H2^T dY, db3 = colsum dY, dH2 = (dY W3^T) * relu'(Z2)
  MB_CUDA_TRY((gemm<float, float, true, false>(W, O, B, n->h2, W, n->dy, O, g + n->off[4], O, nullptr,
                                               nullptr, nullptr, 0, 0, st, n->part, err)));
  colsum_kernel<<<(O + 255) / 256, 256, 0, st>>>(n->dy, B, O, g + n->off[5]);
  MB_CUDA_TRY((gemm<float, __nv_bfloat16, false, true>(B, W, O, n->dy, O, wb + n->off[4], O, n->d2, W,
                                                       nullptr, n->z2, nullptr, 0, 0, st, nullptr, err)));
  // layer 2
  MB_CUDA_TRY((gemm<float, float, true, false>(W, W, B, n->h1, W, n->d2, W, g + n->off[2], W, nullptr,
                                               nullptr, nullptr, 0, 0, st, n->part, err)));
  colsum_kernel<<<(W + 255) / 256, 256, 0, st>>>(n->d2, B, W, g + n->off[3]);
  MB_CUDA_TRY((gemm<float, __nv_bfloat16, false, true>(B, W, W, n->d2, W, wb + n->off[2], W, n->d1, W,
                                                       nullptr, n->z1, nullptr, 0, 0, st, nullptr, err)));
  // layer 1
  MB_CUDA_TRY((gemm<float, float, true, false>(I, W, B, x, I, n->d1, W, g + n->off[0], W, nullptr,
                                               nullptr, nullptr, 0, 0, st, n->part, err)));
  colsum_kernel<<<(W + 255) / 256, 256, 0, st>>>(n->d1, B, W, g + n->off[1]);
  MB_CUDA_TRY(cudaGetLastError());
  return MB_OK;
}

extern "C" mb_status mb_mlp_adam_step(mb_mlp *n, float lr, void *stream) {
  if (!n) return MB_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  n->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)n->step), c2 = 1.f - std::pow(b2, (float)n->step);
  const unsigned blocks = (unsigned)((n->n_params + 255) / 256);
  adam_kernel<<<blocks, 256, 0, st>>>(n->p, n->g, n->m, n->v, n->n_params, lr, b1, b2, 1e-8f, c1, c2);
  MB_CUDA_TRY(cudaGetLastError());
  MB_CUDA_TRY(mlp_refresh_bf16(n, st));
  return MB_OK;
}

#include "zf.cuh"

// The mixed ZF reads the network of its learned initial iterate from the
// handle's own device buffers (the BF16 copies are refreshed by every
// parameter update), so a captured slot replays with the current weights.
mb_status mb::mlp_zf_init_view(const mb_mlp *n, ZfNetView *v) {
  if (!n || !v) return MB_BAD_ARG;
  if (n->n_in != kZfInitFeatures || n->n_out != kZfInitCoeffs || n->width == 0 ||
      n->width > kZfInitMaxWidth)
    return MB_BAD_SHAPE;
  v->w1 = n->wb + n->off[0];
  v->w2 = n->wb + n->off[2];
  v->w3 = n->wb + n->off[4];
  v->b1 = n->p + n->off[1];
  v->b2 = n->p + n->off[3];
  v->b3 = n->p + n->off[5];
  v->width = n->width;
  return MB_OK;
}

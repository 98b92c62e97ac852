// zf.cu -- per-subcarrier-group zero-forcing detector and precoder.
//
// Replaces Beamform::beamformer_uplink (beamform/beamform.cu:74-122: cuBLAS
// CgemmStridedBatched for the Gram C C^H, cusolverDnCpotrfBatched and
// cusolverDnCpotrsBatched with G*M single right-hand sides) with ONE CTA per
// subcarrier group that keeps C in shared memory for the whole solve: Gram,
// Cholesky, the M triangular solves and the write-back of W = (C C^H)^{-1} C
// in the CSI layout.  The downlink precoder P = W^T / max|W|
// (beam_utils.cuh:40-80) can be emitted from the same CTA.
//
// FP32 (MB_ZF_FP32) follows the reference's arithmetic; FP64 (MB_ZF_FP64)
// runs the same schedule in double.  Unlike the reference, which ignores
// cuSOLVER's info array, a non positive definite Gram is reported per group
// (status 1) and its W is zeroed.
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "zf.cuh"

namespace mb {

template <typename T>
struct Cplx {
  T x, y;
};

template <typename T>
__device__ __forceinline__ Cplx<T> mk(T a, T b) {
  Cplx<T> c;
  c.x = a;
  c.y = b;
  return c;
}

// Fills the missing users of a short last group from group G-2 (see
// mb_zf_uplink); runs before the solve so the in-place update of group G-2
// cannot race with the read.
__global__ void zf_fill_tail_kernel(float2 *csi, uint32_t G, uint32_t M,
                                    uint32_t K, uint32_t rem, uint32_t sg) {
  const uint64_t total = (uint64_t)M * K;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u = (uint32_t)(e % K);
    if ((u % sg) >= rem) {
      csi[(uint64_t)(G - 1) * total + e] = csi[(uint64_t)(G - 2) * total + e];
    }
  }
}

// One CTA per group.  Shared memory: C as [K][M+1] complex of T, the Gram /
// Cholesky factor as [K][K+1], and a reduction buffer.
template <typename T>
__global__ void __launch_bounds__(256)
    zf_chol_kernel(float2 *csi, float2 *precoder, uint32_t M, uint32_t K,
                   int32_t *status, float *cond_out) {
  extern __shared__ __align__(16) unsigned char zf_smem_raw[];
  using C = Cplx<T>;
  const uint32_t g = blockIdx.x;
  const uint32_t ldc = M + 1, lda = K + 1;
  C *Cs = reinterpret_cast<C *>(zf_smem_raw);
  C *A = Cs + (size_t)K * ldc;
  float *red = reinterpret_cast<float *>(A + (size_t)K * lda);
  __shared__ int not_pd;
  const int tid = threadIdx.x, nt = blockDim.x;
  float2 *cg = csi + (uint64_t)g * M * K;

  if (tid == 0) not_pd = 0;
  // load C[u][b] = csi[g][b][u] (coalesced in b*K + u)
  for (uint32_t e = tid; e < M * K; e += nt) {
    float2 v = cg[e];
    uint32_t b = e / K, u = e % K;
    Cs[u * ldc + b] = mk<T>((T)v.x, (T)v.y);
  }
  __syncthreads();

  // Gram A = C C^H, lower triangle
  const uint32_t ntri = K * (K + 1) / 2;
  for (uint32_t q = tid; q < ntri; q += nt) {
    // q -> (i, j), j <= i
    uint32_t i = (uint32_t)((sqrtf(8.f * q + 1.f) - 1.f) * 0.5f);
    while (i * (i + 1) / 2 > q) i--;
    while ((i + 1) * (i + 2) / 2 <= q) i++;
    uint32_t j = q - i * (i + 1) / 2;
    const C *ci = Cs + i * ldc, *cj = Cs + j * ldc;
    T sr = 0, si = 0;
    for (uint32_t b = 0; b < M; b++) {
      C a = ci[b], c = cj[b];
      sr += a.x * c.x + a.y * c.y;
      si += a.y * c.x - a.x * c.y;
    }
    A[i * lda + j] = mk<T>(sr, si);
  }
  __syncthreads();

  // right-looking Cholesky A = L L^H in place (lower)
  for (uint32_t j = 0; j < K; j++) {
    if (tid == 0) {
      T d = A[j * lda + j].x;
      if (!(d > (T)0)) {
        not_pd = 1;
        d = (T)1;
      }
      A[j * lda + j] = mk<T>(sqrt(d), (T)0);
    }
    __syncthreads();
    const T inv = (T)1 / A[j * lda + j].x;
    for (uint32_t i = j + 1 + tid; i < K; i += nt) {
      C v = A[i * lda + j];
      A[i * lda + j] = mk<T>(v.x * inv, v.y * inv);
    }
    __syncthreads();
    const uint32_t rem = K - j - 1;
    for (uint32_t q = tid; q < rem * rem; q += nt) {
      uint32_t i = j + 1 + q / rem, k = j + 1 + q % rem;
      if (k > i) continue;
      C a = A[i * lda + j], b = A[k * lda + j];
      // A[i][k] -= L[i][j] * conj(L[k][j])
      C c = A[i * lda + k];
      c.x -= a.x * b.x + a.y * b.y;
      c.y -= a.y * b.x - a.x * b.y;
      A[i * lda + k] = c;
    }
    __syncthreads();
  }

  // W = A^{-1} C: thread per column b, solve in place in Cs[:, b]
  for (uint32_t b = tid; b < M; b += nt) {
    for (uint32_t i = 0; i < K; i++) {
      C s = Cs[i * ldc + b];
      for (uint32_t k = 0; k < i; k++) {
        C l = A[i * lda + k], z = Cs[k * ldc + b];
        s.x -= l.x * z.x - l.y * z.y;
        s.y -= l.x * z.y + l.y * z.x;
      }
      T d = A[i * lda + i].x;
      Cs[i * ldc + b] = mk<T>(s.x / d, s.y / d);
    }
    for (int i = (int)K - 1; i >= 0; i--) {
      C s = Cs[i * ldc + b];
      for (uint32_t k = i + 1; k < K; k++) {
        C l = A[k * lda + i], z = Cs[k * ldc + b];  // conj(L[k][i]) * z
        s.x -= l.x * z.x + l.y * z.y;
        s.y -= l.x * z.y - l.y * z.x;
      }
      T d = A[i * lda + i].x;
      Cs[i * ldc + b] = mk<T>(s.x / d, s.y / d);
    }
  }
  __syncthreads();

  const bool bad = not_pd != 0;
  // write W back in the CSI layout; track max |W| for the precoder
  float mx = 0.f;
  for (uint32_t e = tid; e < M * K; e += nt) {
    uint32_t b = e / K, u = e % K;
    C w = Cs[u * ldc + b];
    float2 o = bad ? make_float2(0.f, 0.f) : make_float2((float)w.x, (float)w.y);
    cg[e] = o;
    mx = fmaxf(mx, sqrtf(o.x * o.x + o.y * o.y));
  }
  if (status && tid == 0) status[g] = bad ? 1 : 0;
  if (cond_out && tid == 0) {
    // cheap estimate from the Cholesky diagonal: (max l_ii / min l_ii)^2
    T lo = A[0].x, hi = A[0].x;
    for (uint32_t i = 1; i < K; i++) {
      T d = A[i * lda + i].x;
      lo = d < lo ? d : lo;
      hi = d > hi ? d : hi;
    }
    cond_out[g] = bad ? INFINITY : (float)((hi / lo) * (hi / lo));
  }
  if (!precoder) return;
  red[tid] = mx;
  __syncthreads();
  for (int s = nt / 2; s > 0; s >>= 1) {
    if (tid < s) red[tid] = fmaxf(red[tid], red[tid + s]);
    __syncthreads();
  }
  const float inv = 1.0f / red[0];
  float2 *pg = precoder + (uint64_t)g * M * K;
  for (uint32_t e = tid; e < M * K; e += nt) {
    uint32_t u = e / M, b = e % M;
    C w = Cs[u * ldc + b];
    float2 o = bad ? make_float2(0.f, 0.f) : make_float2((float)w.x, (float)w.y);
    pg[e] = make_float2(o.x * inv, o.y * inv);
  }
}

// beam_utils.cuh:40-80 as a standalone kernel: one CTA per group.
__global__ void __launch_bounds__(256)
    precoder_kernel(const float2 *W, float2 *P, uint32_t M, uint32_t K) {
  __shared__ float red[256];
  const uint32_t g = blockIdx.x;
  const float2 *wg = W + (uint64_t)g * M * K;
  float2 *pg = P + (uint64_t)g * M * K;
  float mx = 0.f;
  for (uint32_t e = threadIdx.x; e < M * K; e += blockDim.x) {
    float2 v = wg[e];
    mx = fmaxf(mx, sqrtf(v.x * v.x + v.y * v.y));
  }
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  const float inv = 1.0f / red[0];
  // P[u][b] = W[b][u] * inv through 32 x 32 shared-memory tiles, so both the
  // reads (along u) and the writes (along b) are coalesced
  __shared__ float2 tile[32][33];
  const uint32_t tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 8 rows of 32
  for (uint32_t b0 = 0; b0 < M; b0 += 32)
    for (uint32_t u0 = 0; u0 < K; u0 += 32) {
      __syncthreads();
      for (uint32_t r = ty; r < 32; r += 8) {
        const uint32_t b = b0 + r, u = u0 + tx;
        tile[r][tx] = (b < M && u < K) ? wg[(uint64_t)b * K + u] : make_float2(0.f, 0.f);
      }
      __syncthreads();
      for (uint32_t r = ty; r < 32; r += 8) {
        const uint32_t u = u0 + r, b = b0 + tx;
        if (u < K && b < M) {
          const float2 v = tile[tx][r];
          pg[(uint64_t)u * M + b] = make_float2(v.x * inv, v.y * inv);
        }
      }
    }
}

// P[g][u][b] = W[g][b][u] / wmax[g]: one CTA per (group, 32 x 32 tile),
// transposed through shared memory
__global__ void __launch_bounds__(256)
    precoder_scale_kernel(const float2 *W, float2 *P, const float *wmax, uint32_t M, uint32_t K,
                          uint32_t tiles_b) {
  __shared__ float2 tile[32][33];
  const uint32_t g = blockIdx.x;
  const uint32_t b0 = (blockIdx.y % tiles_b) * 32, u0 = (blockIdx.y / tiles_b) * 32;
  const uint32_t tx = threadIdx.x % 32, ty = threadIdx.x / 32;
  const float2 *wg = W + (uint64_t)g * M * K;
  float2 *pg = P + (uint64_t)g * M * K;
  const float inv = 1.0f / wmax[g];  // as precoder_kernel
  for (uint32_t r = ty; r < 32; r += 8) {
    const uint32_t b = b0 + r, u = u0 + tx;
    tile[r][tx] = (b < M && u < K) ? wg[(uint64_t)b * K + u] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  for (uint32_t r = ty; r < 32; r += 8) {
    const uint32_t u = u0 + r, b = b0 + tx;
    if (u < K && b < M) {
      const float2 v = tile[tx][r];
      pg[(uint64_t)u * M + b] = make_float2(v.x * inv, v.y * inv);
    }
  }
}

size_t zf_chol_smem(uint32_t M, uint32_t K, bool dbl) {
  size_t c = dbl ? 16 : 8;
  return c * ((size_t)K * (M + 1) + (size_t)K * (K + 1)) + 256 * sizeof(float);
}

mb_status zf_fill_tail(float2 *csi, uint32_t groups, uint32_t S, uint32_t sg,
                       uint32_t M, uint32_t K, cudaStream_t st) {
  if (groups < 2) return MB_OK;
  uint64_t full = (uint64_t)(groups - 1) * sg;
  if (S <= full || S - full >= sg) return MB_OK;
  uint32_t rem = (uint32_t)(S - full);
  uint64_t total = (uint64_t)M * K;
  unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 1024);
  zf_fill_tail_kernel<<<blocks, 256, 0, st>>>(csi, groups, M, K, rem, sg);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

template <typename T>
static mb_status set_smem_attr(size_t smem) {
  static std::atomic<uint64_t> configured{0};
  int dev = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  if (!(configured.load() & bit)) {
    int maxs = 0;
    cudaFuncAttributes fa;
    MB_CUDA_TRY(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    MB_CUDA_TRY(cudaFuncGetAttributes(&fa, zf_chol_kernel<T>));
    MB_CUDA_TRY(cudaFuncSetAttribute(zf_chol_kernel<T>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     maxs - (int)fa.sharedSizeBytes));
    configured.fetch_or(bit);
  }
  (void)smem;
  return MB_OK;
}

mb_status zf_chol(float2 *csi, float2 *precoder, uint32_t groups, uint32_t M,
                  uint32_t K, bool dbl, int32_t *status, float *cond,
                  cudaStream_t st) {
  size_t smem = zf_chol_smem(M, K, dbl);
  int dev = 0, maxs = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  MB_CUDA_TRY(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (smem + 64 > (size_t)maxs) return MB_UNSUPPORTED;
  if (groups == 0) return MB_OK;
  if (dbl) {
    mb_status s = set_smem_attr<double>(smem);
    if (s != MB_OK) return s;
    zf_chol_kernel<double><<<groups, 256, smem, st>>>(csi, precoder, M, K, status, cond);
  } else {
    mb_status s = set_smem_attr<float>(smem);
    if (s != MB_OK) return s;
    zf_chol_kernel<float><<<groups, 256, smem, st>>>(csi, precoder, M, K, status, cond);
  }
  MB_LAUNCH_CHECK();
  return MB_OK;
}

mb_status precoder_scale(const float2 *W, float2 *P, const float *wmax, uint32_t M, uint32_t K,
                         uint32_t groups, cudaStream_t st) {
  if (groups == 0) return MB_OK;
  const uint32_t tb = (M + 31) / 32, tu = (K + 31) / 32;
  precoder_scale_kernel<<<dim3(groups, tb * tu), 256, 0, st>>>(W, P, wmax, M, K, tb);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

mb_status precoder_launch(const float2 *W, float2 *P, uint32_t M, uint32_t K,
                          uint32_t groups, cudaStream_t st) {
  if (groups == 0) return MB_OK;
  precoder_kernel<<<groups, 256, 0, st>>>(W, P, M, K);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

}  // namespace mb

using namespace mb;

struct mb_zf {
  uint32_t M, K, max_groups;
  void *img_w;        // mixed-precision detector images, sized for max_groups
  const mb_mlp *net;  // network of the learned initial iterate (not owned), or null
};

extern "C" mb_status mb_zf_create(uint32_t num_bs, uint32_t num_ue,
                                  uint32_t max_groups, mb_zf **out) {
  if (!out) return MB_BAD_ARG;
  *out = nullptr;
  if (num_bs == 0 || num_ue == 0 || num_ue > num_bs || num_ue > 64)
    return MB_BAD_SHAPE;
  if (!device_tables()) return MB_CUDA_ERROR;
  mb_zf *z = new mb_zf{num_bs, num_ue, max_groups, nullptr, nullptr};
  const uint64_t bytes = zf_mixed_scratch_bytes(max_groups, num_bs, num_ue);
  cudaError_t e = cudaSuccess;
  if (bytes) e = cudaMalloc(&z->img_w, bytes);
  if (e != cudaSuccess) {
    cudaFree(z->img_w);
    delete z;
    return record_error(e);
  }
  *out = z;
  return MB_OK;
}

extern "C" mb_status mb_zf_destroy(mb_zf *z) {
  if (!z) return MB_BAD_ARG;
  cudaFree(z->img_w);
  delete z;
  return MB_OK;
}

extern "C" mb_status mb_zf_uplink(mb_zf *z, mb_c32 *csi, uint32_t groups,
                                  uint32_t S, uint32_t sg,
                                  const mb_zf_opts *opts, int32_t *status,
                                  float *cond, void *stream) {
  if (!z || !csi) return MB_BAD_ARG;
  if (groups > z->max_groups) return MB_BAD_SHAPE;  // beamform.cu:144-152
  if (sg == 0 || (uint64_t)groups * sg < S || (uint64_t)(groups - 1) * sg >= S)
    return MB_BAD_SHAPE;
  uint32_t prec = opts ? opts->precision : MB_ZF_FP32;
  cudaStream_t st = as_stream(stream);
  float2 *c = reinterpret_cast<float2 *>(csi);
  mb_status s = zf_fill_tail(c, groups, S, sg, z->M, z->K, st);
  if (s != MB_OK) return s;
  switch (prec) {
    case MB_ZF_FP32:
      return zf_chol(c, nullptr, groups, z->M, z->K, false, status, cond, st);
    case MB_ZF_FP64:
      return zf_chol(c, nullptr, groups, z->M, z->K, true, status, cond, st);
    case MB_ZF_MIXED: {
      ZfNetView v{};
      if (opts && opts->init == 1) {
        if (!z->net) return MB_BAD_ARG;
        const mb_status r = mlp_zf_init_view(z->net, &v);
        if (r != MB_OK) return r;
      }
      return zf_mixed_run(c, z->img_w, groups, z->M, z->K, opts, status, cond, st, true, nullptr, &v);
    }
  }
  return MB_BAD_ARG;
}

extern "C" mb_status mb_zf_set_init_net(mb_zf *z, const mb_mlp *net) {
  if (!z) return MB_BAD_ARG;
  if (net) {
    ZfNetView v;
    const mb_status r = mlp_zf_init_view(net, &v);
    if (r != MB_OK) return r;
  }
  z->net = net;
  return MB_OK;
}

extern "C" mb_status mb_zf_precoder(const mb_c32 *W, mb_c32 *P, uint32_t M,
                                    uint32_t K, uint32_t groups, void *stream) {
  if (!W || !P || M == 0 || K == 0) return MB_BAD_ARG;
  return precoder_launch(reinterpret_cast<const float2 *>(W),
                         reinterpret_cast<float2 *>(P), M, K, groups,
                         as_stream(stream));
}

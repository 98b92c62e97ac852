// lzf.cu -- per-subcarrier zero forcing with a learned initial iterate.
//
// The reference computes one ZF detector per group of sg subcarriers from
// the comb pilots (beamform/beamform.cu:74-122), which loses accuracy when
// the channel changes within a group (large delay spread).  This module
// builds a detector per subcarrier instead, without a full inversion per
// subcarrier (no counterpart in the reference):
//  1. interpolate each user's comb-pilot estimates linearly along frequency
//     (user u's pilot of group g sits on subcarrier g sg + u mod sg) to a
//     CSI estimate c_s [M][K] for every data subcarrier s (the pilot FFT's
//     CSI convention: the conjugate channel);
//  2. per subcarrier Gram G_s = C C^H with C[u][b] = c_s[b][u], the
//     reference's Gram (FP32; FP64 for training targets);
//  3. exact inverses X_g of the Grams at the group centres only (Gauss-Jordan
//     per matrix);
//  4. an initial iterate per subcarrier X0_s = sum_j alpha_j X_{g+j},
//     j = -1..2 (group indices clamped at the band edges), where alpha comes
//     from the MLP (mlp.cu) evaluated on features of the neighbouring centre
//     Grams and the subcarrier's offset in its group ("learned"), or alpha =
//     (0, 1, 0, 0) ("coarse": the group's own inverse, i.e. the per-group
//     ZF), or X0_s = G_s^{-1} ("exact");
//  5. ns_iters Newton-Schulz steps X <- X (2I - G_s X) per subcarrier;
//  6. the detector W_s = X_s C, stored [S][M][K] like the per-group W with
//     sg = 1, so the existing equalizer applies it unchanged.
// Training targets come from the same interpolation in FP64: with Y_j the
// four centre inverses and X* = G_s^{-1} (FP64), the loss of a blend alpha
// is ||sum_j alpha_j Y_j - X*||_F^2 / ||X*||_F^2 = alpha^T A alpha - 2 b^T
// alpha + 1 with A_jk = Re tr(Y_j^H Y_k) / ||X*||^2, b_j = Re tr(Y_j^H X*) /
// ||X*||^2.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace mb {
namespace {

constexpr int kBlend = 4;  // centre inverses g-1, g, g+1, g+2

template <typename T> struct CT { using V = float2; };
template <> struct CT<double> { using V = double2; };

template <typename V> __device__ __forceinline__ V cz() { V r; r.x = 0; r.y = 0; return r; }
template <typename V> __device__ __forceinline__ V cmake(double x, double y) {
  V r;
  r.x = (decltype(r.x))x;
  r.y = (decltype(r.y))y;
  return r;
}
template <typename V> __device__ __forceinline__ V cfma(V a, V b, V c) {  // c + a b
  c.x += a.x * b.x - a.y * b.y;
  c.y += a.x * b.y + a.y * b.x;
  return c;
}
template <typename V> __device__ __forceinline__ V cjfma(V a, V b, V c) {  // c + conj(a) b
  c.x += a.x * b.x + a.y * b.y;
  c.y += a.x * b.y - a.y * b.x;
  return c;
}

// 1. c_s[b][u] by linear interpolation of csi[g][b][u] along the pilots of u
template <typename T>
__global__ void interp_kernel(const float2 *csi, typename CT<T>::V *H, uint32_t M, uint32_t K,
                              uint32_t S, uint32_t sg, uint32_t G) {
  using V = typename CT<T>::V;
  const uint64_t total = (uint64_t)S * M * K;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = (uint32_t)(e % K), b = (uint32_t)((e / K) % M), s = (uint32_t)(e / ((uint64_t)K * M));
    const double p = ((double)s - (double)(u % sg)) / (double)sg;  // pilot index coordinate
    int g0 = (int)floor(p);
    g0 = max(0, min(g0, (int)G - 2));
    double t = G > 1 ? p - g0 : 0.0;
    t = fmin(fmax(t, 0.0), 1.0);
    const float2 a = csi[((uint64_t)g0 * M + b) * K + u];
    const float2 c = G > 1 ? csi[((uint64_t)(g0 + 1) * M + b) * K + u] : a;
    H[e] = cmake<V>((1.0 - t) * a.x + t * c.x, (1.0 - t) * a.y + t * c.y);
  }
}

// 2. G_s[u][v] = sum_b c_s[b][u] conj(c_s[b][v]) (the reference's Gram C C^H
// of the CSI, beamform.cu:74-122), one CTA per subcarrier, c_s staged in
// shared memory
template <typename T>
__global__ void gram_kernel(const typename CT<T>::V *H, typename CT<T>::V *Gm, uint32_t M, uint32_t K) {
  using V = typename CT<T>::V;
  extern __shared__ __align__(16) unsigned char gsm[];
  V *h = reinterpret_cast<V *>(gsm);
  const uint32_t s = blockIdx.x;
  const V *Hs = H + (uint64_t)s * M * K;
  for (uint32_t e = threadIdx.x; e < M * K; e += blockDim.x) h[e] = Hs[e];
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < K * K; e += blockDim.x) {
    const uint32_t u = e / K, v = e % K;
    V acc = cz<V>();
    for (uint32_t b = 0; b < M; b++) acc = cjfma(h[b * K + v], h[b * K + u], acc);
    Gm[(uint64_t)s * K * K + e] = acc;
  }
}

// 3. X = G^{-1} for matrices src[idx[i]] (or i when idx is null) by
// Gauss-Jordan on [G | I] without pivoting (G is Hermitian positive
// definite), one CTA per matrix, rows in shared memory; flag[i] = 1 when a
// pivot is not positive
template <typename T>
__global__ void inverse_kernel(const typename CT<T>::V *src, const uint32_t *idx,
                               typename CT<T>::V *X, uint32_t K, int *flag) {
  using V = typename CT<T>::V;
  extern __shared__ __align__(16) unsigned char ism[];
  V *A = reinterpret_cast<V *>(ism);  // K x 2K
  __shared__ int bad;
  const uint32_t i = blockIdx.x, m = idx ? idx[i] : i;
  const V *Gm = src + (uint64_t)m * K * K;
  const uint32_t W = 2 * K;
  if (threadIdx.x == 0) bad = 0;
  for (uint32_t e = threadIdx.x; e < K * W; e += blockDim.x) {
    const uint32_t r = e / W, c = e % W;
    A[e] = c < K ? Gm[r * K + c] : cmake<V>(c - K == r ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  for (uint32_t k = 0; k < K; k++) {
    const T p = A[k * W + k].x;
    if (!(p > (T)0)) {
      if (threadIdx.x == 0) bad = 1;
      break;  // uniform: every thread read the same pivot
    }
    const T inv = (T)1 / p;
    __syncthreads();  // all threads have read the pivot
    for (uint32_t c = threadIdx.x; c < W; c += blockDim.x) {
      V v = A[k * W + c];
      v.x *= inv;
      v.y *= inv;
      A[k * W + c] = v;
    }
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < K * W; e += blockDim.x) {
      const uint32_t r = e / W, c = e % W;
      if (r == k || c == k) continue;  // column k is cleared below
      const V f = A[r * W + k];
      const V rk = A[k * W + c];
      V v = A[r * W + c];
      v.x -= f.x * rk.x - f.y * rk.y;
      v.y -= f.x * rk.y + f.y * rk.x;
      A[r * W + c] = v;
    }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < K; r += blockDim.x)
      if (r != k) A[r * W + k] = cz<V>();
    __syncthreads();
  }
  __syncthreads();
  if (threadIdx.x == 0 && flag) flag[i] = bad;
  for (uint32_t e = threadIdx.x; e < K * K; e += blockDim.x)
    X[(uint64_t)i * K * K + e] = A[(e / K) * W + K + e % K];
}

// Gc[g] = Gs[centre(g)]
__global__ void gather_kernel(const float2 *Gs, const uint32_t *cidx, float2 *Gc, uint32_t K, uint32_t G) {
  const uint64_t total = (uint64_t)G * K * K;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = (uint32_t)(e / (K * K)), r = (uint32_t)(e % (K * K));
    Gc[e] = Gs[(uint64_t)cidx[g] * K * K + r];
  }
}

// 4. features of subcarrier s: one-hot of its offset in the group (sg),
// then for j = -1, +1, +2: ||Gc[g+j] - Gc[g]||_F / ||Gc[g]||_F and
// tr Gc[g+j] / tr Gc[g] - 1 (0 where g+j leaves the band)
__global__ void features_kernel(const float2 *Gc, float *F, uint32_t K, uint32_t S, uint32_t sg,
                                uint32_t G) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const uint32_t g = s / sg, o = s % sg, nf = sg + 6;
  float *f = F + (uint64_t)s * nf;
  for (uint32_t q = 0; q < sg; q++) f[q] = q == o ? 1.f : 0.f;
  const float2 *C0 = Gc + (uint64_t)g * K * K;
  float n0 = 0.f, t0 = 0.f;
  for (uint32_t e = 0; e < K * K; e++) n0 += C0[e].x * C0[e].x + C0[e].y * C0[e].y;
  for (uint32_t u = 0; u < K; u++) t0 += C0[u * K + u].x;
  n0 = sqrtf(n0);
  const int js[3] = {-1, 1, 2};
  for (int q = 0; q < 3; q++) {
    const int gj = (int)g + js[q];
    float d = 0.f, tr = 0.f;
    if (gj >= 0 && gj < (int)G) {
      const float2 *Cj = Gc + (uint64_t)gj * K * K;
      for (uint32_t e = 0; e < K * K; e++) {
        const float dx = Cj[e].x - C0[e].x, dy = Cj[e].y - C0[e].y;
        d += dx * dx + dy * dy;
      }
      for (uint32_t u = 0; u < K; u++) tr += Cj[u * K + u].x;
      d = n0 > 0.f ? sqrtf(d) / n0 : 0.f;
      tr = t0 > 0.f ? tr / t0 - 1.f : 0.f;
    }
    f[sg + q] = d;
    f[sg + 3 + q] = tr;
  }
}

// 5. X0_s = sum_j alpha[s][j] Xc[clamp(g + j - 1)] (alpha null: coarse)
__global__ void blend_kernel(const float *alpha, const float2 *Xc, float2 *X, uint32_t K, uint32_t S,
                             uint32_t sg, uint32_t G) {
  const uint64_t total = (uint64_t)S * K * K;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = (uint32_t)(e / (K * K)), r = (uint32_t)(e % (K * K));
    const uint32_t g = s / sg;
    float2 acc = make_float2(0.f, 0.f);
    if (!alpha) {
      acc = Xc[(uint64_t)g * K * K + r];
    } else {
      for (int j = 0; j < kBlend; j++) {
        const int gj = min(max((int)g + j - 1, 0), (int)G - 1);
        const float a = alpha[(uint64_t)s * kBlend + j];
        const float2 x = Xc[(uint64_t)gj * K * K + r];
        acc.x += a * x.x;
        acc.y += a * x.y;
      }
    }
    X[e] = acc;
  }
}

// 6. Newton-Schulz per subcarrier, one CTA of K*K threads: X <- X (2I - G X)
__global__ void ns_kernel(const float2 *Gm, float2 *X, uint32_t K, uint32_t iters) {
  extern __shared__ __align__(16) unsigned char nsm[];
  float2 *g = reinterpret_cast<float2 *>(nsm), *x = g + K * K, *t = x + K * K;
  const uint32_t s = blockIdx.x, e = threadIdx.x, r = e / K, c = e % K;
  const bool on = e < K * K;
  if (on) {
    g[e] = Gm[(uint64_t)s * K * K + e];
    x[e] = X[(uint64_t)s * K * K + e];
  }
  __syncthreads();
  for (uint32_t it = 0; it < iters; it++) {
    float2 acc = make_float2(0.f, 0.f);
    if (on)
      for (uint32_t k = 0; k < K; k++) acc = cfma(g[r * K + k], x[k * K + c], acc);
    if (on) t[e] = make_float2((r == c ? 2.f : 0.f) - acc.x, -acc.y);
    __syncthreads();
    acc = make_float2(0.f, 0.f);
    if (on)
      for (uint32_t k = 0; k < K; k++) acc = cfma(x[r * K + k], t[k * K + c], acc);
    __syncthreads();
    if (on) x[e] = acc;
    __syncthreads();
  }
  if (on) X[(uint64_t)s * K * K + e] = x[e];
}

// ||I - G_s X_s||_F per subcarrier
__global__ void residual_kernel(const float2 *Gm, const float2 *X, float *res, uint32_t K, uint32_t S) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const float2 *g = Gm + (uint64_t)s * K * K, *x = X + (uint64_t)s * K * K;
  float acc = 0.f;
  for (uint32_t r = 0; r < K; r++)
    for (uint32_t c = 0; c < K; c++) {
      float2 v = make_float2(r == c ? -1.f : 0.f, 0.f);
      for (uint32_t k = 0; k < K; k++) v = cfma(g[r * K + k], x[k * K + c], v);
      acc += v.x * v.x + v.y * v.y;
    }
  res[s] = sqrtf(acc);
}

// 7. W_s[b][u] = sum_v X_s[u][v] c_s[b][v] (W = G^{-1} C in the CSI layout)
__global__ void detector_kernel(const float2 *X, const float2 *H, float2 *W, uint32_t M, uint32_t K,
                                uint32_t S) {
  const uint64_t total = (uint64_t)S * M * K;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = (uint32_t)(e % K);
    const uint64_t sb = e / K;  // s * M + b
    const uint32_t s = (uint32_t)(sb / M);
    const float2 *x = X + (uint64_t)s * K * K + (uint64_t)u * K;
    const float2 *h = H + sb * K;
    float2 acc = make_float2(0.f, 0.f);
    for (uint32_t v = 0; v < K; v++) acc = cfma(x[v], h[v], acc);
    W[e] = acc;
  }
}

// training targets: A [S][4][4], b [S][4] from the FP64 centre inverses Yc
// and the FP64 per-subcarrier inverses Xs
__global__ void targets_kernel(const double2 *Yc, const double2 *Xs, float *A, float *bv, uint32_t K,
                               uint32_t S, uint32_t sg, uint32_t G) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const uint32_t g = s / sg, KK = K * K;
  const double2 *Y[kBlend];
  for (int j = 0; j < kBlend; j++) Y[j] = Yc + (uint64_t)min(max((int)g + j - 1, 0), (int)G - 1) * KK;
  const double2 *x = Xs + (uint64_t)s * KK;
  double nx = 0.0;
  for (uint32_t e = 0; e < KK; e++) nx += x[e].x * x[e].x + x[e].y * x[e].y;
  const double inv = nx > 0.0 ? 1.0 / nx : 0.0;
  for (int j = 0; j < kBlend; j++) {
    double bj = 0.0;
    for (uint32_t e = 0; e < KK; e++) bj += Y[j][e].x * x[e].x + Y[j][e].y * x[e].y;
    bv[(uint64_t)s * kBlend + j] = (float)(bj * inv);
    for (int k = j; k < kBlend; k++) {
      double a = 0.0;
      for (uint32_t e = 0; e < KK; e++) a += Y[j][e].x * Y[k][e].x + Y[j][e].y * Y[k][e].y;
      A[((uint64_t)s * kBlend + j) * kBlend + k] = (float)(a * inv);
      A[((uint64_t)s * kBlend + k) * kBlend + j] = (float)(a * inv);
    }
  }
}

unsigned grid_for(uint64_t n) { return (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16); }

}  // namespace
}  // namespace mb

using namespace mb;


struct mb_lzf {
  uint32_t M, K, S, sg, G;
  float2 *H, *Gs, *Gc, *Xc, *X;   // FP32 working set
  float *feat, *alpha, *res;
  uint32_t *cidx;                 // centre subcarrier of each group
  int *flag;                      // per-inverse non-PD flags
  double2 *H64, *Gs64, *Yc64, *X64;  // FP64 training-target set (allocated on first use)
};

extern "C" mb_status mb_lzf_destroy(mb_lzf *z) {
  if (!z) return MB_BAD_ARG;
  for (void *p : {(void *)z->H, (void *)z->Gs, (void *)z->Gc, (void *)z->Xc, (void *)z->X,
                  (void *)z->feat, (void *)z->alpha, (void *)z->res, (void *)z->cidx, (void *)z->flag,
                  (void *)z->H64, (void *)z->Gs64, (void *)z->Yc64, (void *)z->X64})
    cudaFree(p);
  delete z;
  return MB_OK;
}

extern "C" mb_status mb_lzf_create(uint32_t M, uint32_t K, uint32_t S, uint32_t sg, mb_lzf **out) {
  if (!out) return MB_BAD_ARG;
  *out = nullptr;
  if (M == 0 || K == 0 || K > 32 || K > M || S == 0 || sg == 0 || sg > 64) return MB_BAD_SHAPE;
  mb_lzf *z = new mb_lzf();
  z->M = M;
  z->K = K;
  z->S = S;
  z->sg = sg;
  z->G = (S + sg - 1) / sg;
  mb_status st = MB_OK;
  auto alloc = [&](void **p, size_t bytes) {
    if (st != MB_OK) return;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) st = record_error(e);
  };
  const size_t smk = (size_t)S * M * K, skk = (size_t)S * K * K, gkk = (size_t)z->G * K * K;
  alloc((void **)&z->H, sizeof(float2) * smk);
  alloc((void **)&z->Gs, sizeof(float2) * skk);
  alloc((void **)&z->X, sizeof(float2) * skk);
  alloc((void **)&z->Gc, sizeof(float2) * gkk);
  alloc((void **)&z->Xc, sizeof(float2) * gkk);
  alloc((void **)&z->feat, sizeof(float) * (size_t)S * (sg + 6));
  alloc((void **)&z->alpha, sizeof(float) * (size_t)S * kBlend);
  alloc((void **)&z->res, sizeof(float) * S);
  alloc((void **)&z->cidx, sizeof(uint32_t) * z->G);
  alloc((void **)&z->flag, sizeof(int) * std::max(z->G, S));
  if (st == MB_OK) {
    std::vector<uint32_t> c(z->G);
    for (uint32_t g = 0; g < z->G; g++) c[g] = std::min(g * sg + sg / 2, S - 1);
    cudaError_t e = cudaMemcpy(z->cidx, c.data(), sizeof(uint32_t) * z->G, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) st = record_error(e);
  }
  if (st != MB_OK) {
    mb_lzf_destroy(z);
    return st;
  }
  *out = z;
  return MB_OK;
}

extern "C" uint32_t mb_lzf_num_features(uint32_t sg) { return sg + 6; }

// interpolation, Grams, centre Grams and their inverses (FP32)
static mb_status lzf_front(mb_lzf *z, const mb_c32 *csi, cudaStream_t st) {
  const uint32_t M = z->M, K = z->K, S = z->S;
  interp_kernel<float><<<grid_for((uint64_t)S * M * K), 256, 0, st>>>(
      reinterpret_cast<const float2 *>(csi), z->H, M, K, S, z->sg, z->G);
  gram_kernel<float><<<S, 256, sizeof(float2) * M * K, st>>>(z->H, z->Gs, M, K);
  gather_kernel<<<grid_for((uint64_t)z->G * K * K), 256, 0, st>>>(z->Gs, z->cidx, z->Gc, K, z->G);
  inverse_kernel<float><<<z->G, 256, sizeof(float2) * 2 * K * K, st>>>(z->Gc, nullptr, z->Xc, K, z->flag);
  MB_CUDA_TRY(cudaGetLastError());
  return MB_OK;
}

static mb_status lzf_shared_mem_ok(const mb_lzf *z) {
  // the Gram kernel stages one subcarrier's M x K channel (FP64 for targets)
  return (size_t)z->M * z->K * sizeof(double2) <= 48 * 1024 ? MB_OK : MB_UNSUPPORTED;
}

extern "C" mb_status mb_lzf_features(mb_lzf *z, const mb_c32 *csi, float *features, void *stream) {
  if (!z || !csi || !features) return MB_BAD_ARG;
  if (lzf_shared_mem_ok(z) != MB_OK) return MB_UNSUPPORTED;
  cudaStream_t st = as_stream(stream);
  mb_status r = lzf_front(z, csi, st);
  if (r != MB_OK) return r;
  features_kernel<<<(z->S + 127) / 128, 128, 0, st>>>(z->Gc, features, z->K, z->S, z->sg, z->G);
  MB_CUDA_TRY(cudaGetLastError());
  return MB_OK;
}

extern "C" mb_status mb_lzf_run(mb_lzf *z, const mb_c32 *csi, mb_mlp *mlp, int init,
                                uint32_t ns_iters, mb_c32 *W, void *stream) {
  if (!z || !csi || !W) return MB_BAD_ARG;
  if (init < MB_LZF_COARSE || init > MB_LZF_EXACT || (init == MB_LZF_LEARNED && !mlp)) return MB_BAD_ARG;
  if (lzf_shared_mem_ok(z) != MB_OK) return MB_UNSUPPORTED;
  cudaStream_t st = as_stream(stream);
  const uint32_t M = z->M, K = z->K, S = z->S;
  mb_status r = lzf_front(z, csi, st);
  if (r != MB_OK) return r;
  if (init == MB_LZF_EXACT) {
    inverse_kernel<float><<<S, 256, sizeof(float2) * 2 * K * K, st>>>(z->Gs, nullptr, z->X, K, z->flag);
  } else {
    const float *alpha = nullptr;
    if (init == MB_LZF_LEARNED) {
      features_kernel<<<(S + 127) / 128, 128, 0, st>>>(z->Gc, z->feat, K, S, z->sg, z->G);
      MB_CUDA_TRY(cudaGetLastError());
      r = mb_mlp_forward(mlp, z->feat, S, z->alpha, st);
      if (r != MB_OK) return r;
      alpha = z->alpha;
    }
    blend_kernel<<<grid_for((uint64_t)S * K * K), 256, 0, st>>>(alpha, z->Xc, z->X, K, S, z->sg, z->G);
  }
  MB_CUDA_TRY(cudaGetLastError());
  if (ns_iters) {
    ns_kernel<<<S, ((K * K + 31) / 32) * 32, 3 * sizeof(float2) * K * K, st>>>(z->Gs, z->X, K, ns_iters);
    MB_CUDA_TRY(cudaGetLastError());
  }
  detector_kernel<<<grid_for((uint64_t)S * M * K), 256, 0, st>>>(z->X, z->H, reinterpret_cast<float2 *>(W),
                                                                 M, K, S);
  MB_CUDA_TRY(cudaGetLastError());
  return MB_OK;
}

extern "C" mb_status mb_lzf_residual(mb_lzf *z, float *res, void *stream) {
  if (!z || !res) return MB_BAD_ARG;
  residual_kernel<<<(z->S + 127) / 128, 128, 0, as_stream(stream)>>>(z->Gs, z->X, res, z->K, z->S);
  MB_CUDA_TRY(cudaGetLastError());
  return MB_OK;
}

extern "C" mb_status mb_lzf_targets(mb_lzf *z, const mb_c32 *csi, float *A, float *b, void *stream) {
  if (!z || !csi || !A || !b) return MB_BAD_ARG;
  if (lzf_shared_mem_ok(z) != MB_OK) return MB_UNSUPPORTED;
  cudaStream_t st = as_stream(stream);
  const uint32_t M = z->M, K = z->K, S = z->S;
  if (!z->H64) {
    const size_t smk = (size_t)S * M * K, skk = (size_t)S * K * K, gkk = (size_t)z->G * K * K;
    MB_CUDA_TRY(cudaMalloc(&z->H64, sizeof(double2) * smk));
    MB_CUDA_TRY(cudaMalloc(&z->Gs64, sizeof(double2) * skk));
    MB_CUDA_TRY(cudaMalloc(&z->X64, sizeof(double2) * skk));
    MB_CUDA_TRY(cudaMalloc(&z->Yc64, sizeof(double2) * gkk));
  }
  interp_kernel<double><<<grid_for((uint64_t)S * M * K), 256, 0, st>>>(
      reinterpret_cast<const float2 *>(csi), z->H64, M, K, S, z->sg, z->G);
  gram_kernel<double><<<S, 256, sizeof(double2) * M * K, st>>>(z->H64, z->Gs64, M, K);
  inverse_kernel<double><<<S, 256, sizeof(double2) * 2 * K * K, st>>>(z->Gs64, nullptr, z->X64, K, z->flag);
  inverse_kernel<double><<<z->G, 256, sizeof(double2) * 2 * K * K, st>>>(z->Gs64, z->cidx, z->Yc64, K,
                                                                        nullptr);
  targets_kernel<<<(S + 127) / 128, 128, 0, st>>>(z->Yc64, z->X64, A, b, K, S, z->sg, z->G);
  MB_CUDA_TRY(cudaGetLastError());
  return MB_OK;
}

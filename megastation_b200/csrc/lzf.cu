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
#include <atomic>
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

// interpolation position of subcarrier s for user u: c_s = (1 - t) csi[g0]
// + t csi[g0 + 1] (integer floor division, then one float division)
__device__ __forceinline__ void interp_pos(uint32_t s, uint32_t u, uint32_t sg, uint32_t G, int &g0,
                                           float &t) {
  const int num = (int)s - (int)(u % sg);
  int q = num >= 0 ? num / (int)sg : -(((-num) + (int)sg - 1) / (int)sg);
  const int gmax = (int)G - 2;
  g0 = max(0, min(q, gmax));
  t = G > 1 ? fminf(fmaxf((float)(num - g0 * (int)sg) / (float)sg, 0.f), 1.f) : 0.f;
}

// c_s [M][K] of subcarrier s into shared memory; ig / iw: per (s, u) the
// lower pilot group and the weight of the upper one (interp_pos, tabulated)
__device__ __forceinline__ void interp_smem(const float2 *csi, const int *ig, const float *iw, float2 *c,
                                            uint32_t s, uint32_t M, uint32_t K, uint32_t G) {
  for (uint32_t e = threadIdx.x; e < M * K; e += blockDim.x) {
    const uint32_t b = e / K, u = e % K;
    const int g0 = ig[s * K + u];
    const float t = iw[s * K + u];
    const float2 a = csi[((uint64_t)g0 * M + b) * K + u];
    const float2 d = G > 1 ? csi[((uint64_t)(g0 + 1) * M + b) * K + u] : a;
    c[e] = make_float2((1.f - t) * a.x + t * d.x, (1.f - t) * a.y + t * d.y);
  }
}

__global__ void interp_table_kernel(int *ig, float *iw, uint32_t K, uint32_t S, uint32_t sg, uint32_t G) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= S * K) return;
  int g0;
  float t;
  interp_pos(e / K, e % K, sg, G, g0, t);
  ig[e] = g0;
  iw[e] = t;
}

// Gauss-Jordan inverse of the K x K matrix in the first K columns of A
// (K x 2K, row-major, the right half set to I by the caller) by all
// threads; returns false when a pivot is not positive
template <typename V, typename T>
__device__ bool gj_smem(V *A, uint32_t K, int *bad) {
  const uint32_t W = 2 * K;
  if (threadIdx.x == 0) *bad = 0;
  __syncthreads();
  for (uint32_t k = 0; k < K; k++) {
    const T p = A[k * W + k].x;
    if (!(p > (T)0)) {
      if (threadIdx.x == 0) *bad = 1;
      break;  // uniform: every thread read the same pivot
    }
    const T inv = (T)1 / p;
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < W; c += blockDim.x) {
      V v = A[k * W + c];
      v.x *= inv;
      v.y *= inv;
      A[k * W + c] = v;
    }
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < K * W; e += blockDim.x) {
      const uint32_t r = e / W, c = e % W;
      if (r == k || c == k) continue;
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
  return *bad == 0;
}

// per subcarrier: interpolated CSI in shared memory, then its Gram
__global__ void sub_gram_kernel(const float2 *csi, const int *ig, const float *iw, float2 *Gm, uint32_t M,
                                uint32_t K, uint32_t G) {
  extern __shared__ __align__(16) unsigned char sgm[];
  float2 *c = reinterpret_cast<float2 *>(sgm);
  const uint32_t s = blockIdx.x;
  interp_smem(csi, ig, iw, c, s, M, K, G);
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < K * K; e += blockDim.x) {
    const uint32_t u = e / K, v = e % K;
    float2 acc = make_float2(0.f, 0.f);
    for (uint32_t b = 0; b < M; b++) acc = cjfma(c[b * K + v], c[b * K + u], acc);
    Gm[(uint64_t)s * K * K + e] = acc;
  }
}

// per group g: ||Gc[g]||_F, and for j = -1, +1, +2 the relative distance
// ||Gc[g+j] - Gc[g]|| / ||Gc[g]|| and trace ratio minus 1 -> st[g][6]
__global__ void group_stats_kernel(const float2 *Gc, float *st, uint32_t K, uint32_t G) {
  __shared__ float red[8][256];
  const uint32_t g = blockIdx.x, KK = K * K;
  const float2 *C0 = Gc + (uint64_t)g * KK;
  const int js[3] = {-1, 1, 2};
  float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // n0, t0, d[-1], d[1], d[2], t[-1], t[1], t[2]
  for (uint32_t e = threadIdx.x; e < KK; e += blockDim.x) {
    const float2 a = C0[e];
    const bool diag = e / K == e % K;
    v[0] += a.x * a.x + a.y * a.y;
    if (diag) v[1] += a.x;
    for (int q = 0; q < 3; q++) {
      const int gj = (int)g + js[q];
      if (gj < 0 || gj >= (int)G) continue;
      const float2 b = Gc[(uint64_t)gj * KK + e];
      v[2 + q] += (b.x - a.x) * (b.x - a.x) + (b.y - a.y) * (b.y - a.y);
      if (diag) v[5 + q] += b.x;
    }
  }
  for (int i = 0; i < 8; i++) red[i][threadIdx.x] = v[i];
  __syncthreads();
  for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int i = 0; i < 8; i++) red[i][threadIdx.x] += red[i][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const float n0 = sqrtf(red[0][0]), t0 = red[1][0];
    for (int q = 0; q < 3; q++) {
      const int gj = (int)g + js[q];
      const bool in = gj >= 0 && gj < (int)G;
      st[g * 6 + q] = in && n0 > 0.f ? sqrtf(red[2 + q][0]) / n0 : 0.f;
      st[g * 6 + 3 + q] = in && t0 > 0.f ? red[5 + q][0] / t0 - 1.f : 0.f;
    }
  }
}

// features [S][sg + 6]: one-hot offset, then the group's six statistics
__global__ void features2_kernel(const float *st, float *F, uint32_t S, uint32_t sg) {
  const uint32_t nf = sg + 6;
  const uint64_t total = (uint64_t)S * nf;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = (uint32_t)(e / nf), f = (uint32_t)(e % nf);
    F[e] = f < sg ? (f == s % sg ? 1.f : 0.f) : st[(s / sg) * 6 + (f - sg)];
  }
}

// per subcarrier: initial iterate (coarse / learned blend / exact
// Gauss-Jordan), Newton-Schulz steps, then the detector W_s = X C, all in
// shared memory; X is also stored for the residual diagnostic
__global__ void sub_detect_kernel(const float2 *csi, const int *ig, const float *iw, const float2 *Gm,
                                  const float2 *Xc, const float *alpha, int mode, uint32_t iters,
                                  float2 *Xout, float2 *W, uint32_t M, uint32_t K, uint32_t sg,
                                  uint32_t G, int *flag) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ int bad;
  const uint32_t KK = K * K;
  float2 *g = reinterpret_cast<float2 *>(dsm), *x = g + KK, *t = x + KK, *aug = t + KK;
  float2 *c = aug;  // K x 2K for the exact inverse, then M x K of CSI
  const uint32_t s = blockIdx.x, grp = s / sg;
  for (uint32_t e = threadIdx.x; e < KK; e += blockDim.x) g[e] = Gm[(uint64_t)s * KK + e];
  if (mode == 2) {
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < 2 * KK; e += blockDim.x) {
      const uint32_t r = e / (2 * K), q = e % (2 * K);
      aug[e] = q < K ? g[r * K + q] : make_float2(q - K == r ? 1.f : 0.f, 0.f);
    }
    __syncthreads();
    const bool ok = gj_smem<float2, float>(aug, K, &bad);
    if (threadIdx.x == 0 && flag) flag[s] = ok ? 0 : 1;
    for (uint32_t e = threadIdx.x; e < KK; e += blockDim.x) x[e] = aug[(e / K) * 2 * K + K + e % K];
  } else {
    for (uint32_t e = threadIdx.x; e < KK; e += blockDim.x) {
      float2 acc = make_float2(0.f, 0.f);
      if (mode == 0) {
        acc = Xc[(uint64_t)grp * KK + e];
      } else {
        for (int j = 0; j < kBlend; j++) {
          const int gj = min(max((int)grp + j - 1, 0), (int)G - 1);
          const float a = alpha[(uint64_t)s * kBlend + j];
          const float2 v = Xc[(uint64_t)gj * KK + e];
          acc.x += a * v.x;
          acc.y += a * v.y;
        }
      }
      x[e] = acc;
    }
  }
  __shared__ float e0sq;  // ||I - G X0||_F^2 of the initial iterate
  if (threadIdx.x == 0) {
    e0sq = 0.f;
    if (mode != 2 && flag) flag[s] = 0;
  }
  __syncthreads();
  for (uint32_t it = 0; it < iters; it++) {
    float part = 0.f;
    for (uint32_t e = threadIdx.x; e < KK; e += blockDim.x) {
      const uint32_t r = e / K, q = e % K;
      float2 acc = make_float2(0.f, 0.f);
      for (uint32_t k = 0; k < K; k++) acc = cfma(g[r * K + k], x[k * K + q], acc);
      t[e] = make_float2((r == q ? 2.f : 0.f) - acc.x, -acc.y);
      const float ex = (r == q ? 1.f : 0.f) - acc.x;
      part += ex * ex + acc.y * acc.y;
    }
    if (it == 0 && mode != 2) {
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      if ((threadIdx.x & 31) == 0) atomicAdd(&e0sq, part);
    }
    __syncthreads();
    if (it == 0 && mode != 2 && !(e0sq < 1.f)) {
      // Newton-Schulz converges only from ||I - G X0|| < 1: a start further
      // off (the blend of neighbouring groups' inverses under a channel that
      // changes too fast across the band) takes the exact inverse instead,
      // flagged 2 (uniform: every thread read the same sum)
      for (uint32_t e = threadIdx.x; e < 2 * KK; e += blockDim.x) {
        const uint32_t r = e / (2 * K), q = e % (2 * K);
        aug[e] = q < K ? g[r * K + q] : make_float2(q - K == r ? 1.f : 0.f, 0.f);
      }
      __syncthreads();
      const bool ok = gj_smem<float2, float>(aug, K, &bad);
      if (threadIdx.x == 0 && flag) flag[s] = ok ? 2 : 1;
      for (uint32_t e = threadIdx.x; e < KK; e += blockDim.x) x[e] = aug[(e / K) * 2 * K + K + e % K];
      __syncthreads();
      break;
    }
    float2 nx[4];
    uint32_t n = 0;
    for (uint32_t e = threadIdx.x; e < KK; e += blockDim.x, n++) {
      const uint32_t r = e / K, q = e % K;
      float2 acc = make_float2(0.f, 0.f);
      for (uint32_t k = 0; k < K; k++) acc = cfma(x[r * K + k], t[k * K + q], acc);
      nx[n] = acc;
    }
    __syncthreads();
    n = 0;
    for (uint32_t e = threadIdx.x; e < KK; e += blockDim.x, n++) x[e] = nx[n];
    __syncthreads();
  }
  // X transposed into t (xt[v][u]) so that the lanes of a warp, which hold
  // consecutive users u, read consecutive words
  for (uint32_t e = threadIdx.x; e < KK; e += blockDim.x) {
    if (Xout) Xout[(uint64_t)s * KK + e] = x[e];
    t[(e % K) * K + e / K] = x[e];
  }
  interp_smem(csi, ig, iw, c, s, M, K, G);
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < M * K; e += blockDim.x) {
    const uint32_t b = e / K, u = e % K;
    float2 acc = make_float2(0.f, 0.f);
    for (uint32_t v = 0; v < K; v++) acc = cfma(t[v * K + u], c[b * K + v], acc);
    W[(uint64_t)s * M * K + e] = acc;
  }
}

unsigned grid_for(uint64_t n) { return (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16); }

}  // namespace
}  // namespace mb

using namespace mb;


struct mb_lzf {
  uint32_t M, K, S, sg, G;
  float2 *Gs, *Gc, *Xc, *X;       // FP32 working set: per-subcarrier and centre Grams, inverses
  float *feat, *alpha, *res, *stats;  // stats: per-group feature statistics [G][6]
  uint32_t *cidx;                 // centre subcarrier of each group
  int *ig;                        // [S][K] lower pilot group of the interpolation
  float *iw;                      // [S][K] weight of the upper pilot group
  int *flag;                      // per-inverse non-PD flags
  double2 *H64, *Gs64, *Yc64, *X64;  // FP64 training-target set (allocated on first use)
};

extern "C" mb_status mb_lzf_destroy(mb_lzf *z) {
  if (!z) return MB_BAD_ARG;
  for (void *p : {(void *)z->ig, (void *)z->iw, (void *)z->stats, (void *)z->Gs, (void *)z->Gc, (void *)z->Xc, (void *)z->X,
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
  const size_t skk = (size_t)S * K * K, gkk = (size_t)z->G * K * K;
  alloc((void **)&z->Gs, sizeof(float2) * skk);
  alloc((void **)&z->X, sizeof(float2) * skk);
  alloc((void **)&z->Gc, sizeof(float2) * gkk);
  alloc((void **)&z->Xc, sizeof(float2) * gkk);
  alloc((void **)&z->feat, sizeof(float) * (size_t)S * (sg + 6));
  alloc((void **)&z->alpha, sizeof(float) * (size_t)S * kBlend);
  alloc((void **)&z->res, sizeof(float) * S);
  alloc((void **)&z->stats, sizeof(float) * 6 * z->G);
  alloc((void **)&z->ig, sizeof(int) * (size_t)S * K);
  alloc((void **)&z->iw, sizeof(float) * (size_t)S * K);
  if (st == MB_OK) {
    interp_table_kernel<<<(S * K + 255) / 256, 256>>>(z->ig, z->iw, K, S, sg, z->G);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) st = record_error(e);
  }
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

// interpolated CSI and Grams per subcarrier, centre Grams and their
// inverses, per-group feature statistics (FP32)
static mb_status lzf_front(mb_lzf *z, const mb_c32 *csi, cudaStream_t st) {
  const uint32_t M = z->M, K = z->K, S = z->S;
  sub_gram_kernel<<<S, 256, sizeof(float2) * M * K, st>>>(reinterpret_cast<const float2 *>(csi), z->ig, z->iw,
                                                          z->Gs, M, K, z->G);
  gather_kernel<<<grid_for((uint64_t)z->G * K * K), 256, 0, st>>>(z->Gs, z->cidx, z->Gc, K, z->G);
  inverse_kernel<float><<<z->G, 256, sizeof(float2) * 2 * K * K, st>>>(z->Gc, nullptr, z->Xc, K, z->flag);
  group_stats_kernel<<<z->G, 256, 0, st>>>(z->Gc, z->stats, K, z->G);
  MB_CUDA_TRY(cudaGetLastError());
  return MB_OK;
}

static size_t detect_smem(const mb_lzf *z) {
  return sizeof(float2) * (3 * (size_t)z->K * z->K + std::max<size_t>(2 * (size_t)z->K * z->K,
                                                                     (size_t)z->M * z->K));
}

// The kernels that stage one subcarrier's M x K CSI in shared memory take
// up to the device's opt-in limit (raised once per device): 256 x 32 needs
// 64 KB (FP32 Gram), 88 KB (detector) and 128 KB (FP64 Gram of the targets).
static mb_status lzf_configure(size_t *limit) {
  static std::atomic<uint64_t> configured{0};
  static std::atomic<int> lim[64] = {};
  int dev = 0, maxs = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  if (!(configured.load() & bit)) {
    MB_CUDA_TRY(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    int l = maxs;
    const void *ks[3] = {(const void *)sub_gram_kernel, (const void *)sub_detect_kernel,
                         (const void *)gram_kernel<double>};
    for (const void *k : ks) {
      cudaFuncAttributes fa;
      MB_CUDA_TRY(cudaFuncGetAttributes(&fa, k));
      MB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs - (int)fa.sharedSizeBytes));
      l = std::min(l, maxs - (int)fa.sharedSizeBytes);
    }
    lim[dev & 63].store(l);
    configured.fetch_or(bit);
  }
  *limit = (size_t)lim[dev & 63].load();
  return MB_OK;
}

static mb_status lzf_shared_mem_ok(const mb_lzf *z) {
  // one subcarrier's M x K CSI is staged in shared memory (FP64 for targets)
  size_t limit = 0;
  const mb_status r = lzf_configure(&limit);
  if (r != MB_OK) return r;
  return (size_t)z->M * z->K * sizeof(double2) <= limit && detect_smem(z) <= limit ? MB_OK : MB_UNSUPPORTED;
}

extern "C" mb_status mb_lzf_features(mb_lzf *z, const mb_c32 *csi, float *features, void *stream) {
  if (!z || !csi || !features) return MB_BAD_ARG;
  if (lzf_shared_mem_ok(z) != MB_OK) return MB_UNSUPPORTED;
  cudaStream_t st = as_stream(stream);
  mb_status r = lzf_front(z, csi, st);
  if (r != MB_OK) return r;
  features2_kernel<<<grid_for((uint64_t)z->S * (z->sg + 6)), 256, 0, st>>>(z->stats, features, z->S, z->sg);
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
  if (init == MB_LZF_LEARNED) {
    features2_kernel<<<grid_for((uint64_t)S * (z->sg + 6)), 256, 0, st>>>(z->stats, z->feat, S, z->sg);
    MB_CUDA_TRY(cudaGetLastError());
    r = mb_mlp_forward(mlp, z->feat, S, z->alpha, st);
    if (r != MB_OK) return r;
  }
  const size_t smem = detect_smem(z);
  sub_detect_kernel<<<S, 256, smem, st>>>(reinterpret_cast<const float2 *>(csi), z->ig, z->iw, z->Gs, z->Xc,
                                          init == MB_LZF_LEARNED ? z->alpha : nullptr, init, ns_iters, z->X,
                                          reinterpret_cast<float2 *>(W), M, K, z->sg, z->G, z->flag);
  MB_CUDA_TRY(cudaGetLastError());
  return MB_OK;
}

extern "C" mb_status mb_lzf_flags(mb_lzf *z, int32_t *flags, void *stream) {
  if (!z || !flags) return MB_BAD_ARG;
  MB_CUDA_TRY(cudaMemcpyAsync(flags, z->flag, sizeof(int) * z->S, cudaMemcpyDeviceToDevice, as_stream(stream)));
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

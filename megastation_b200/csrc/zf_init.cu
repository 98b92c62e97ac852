// zf_init.cu -- training data of the learned initial iterate of the mixed
// ZF (no counterpart in the reference).
//
// For a group's Gram G = C C^H (C[u][b] = csi[g][b][u], the reference's
// Gram of beamform/beamform.cu:74-122) with tau = tr(G) / K and Gn = G / tau,
// the initial iterate X0 = (a0 I + a1 Gn + a2 Gn^2 + a3 Gn^3) / tau leaves
// the residual I - G X0 = I - sum_i a_i Gn^(i+1), whose squared Frobenius
// norm over K is the quadratic form a^T A a - 2 b^T a + 1 with
// A_ij = t_(i+j+2), b_i = t_(i+1) and t_k = tr(Gn^k) / K.  One CTA per group
// forms the Gram in FP64, the powers Gn^2 and Gn^3 in shared memory and the
// traces t_1..t_8 (t_7 and t_8 from Gn^4 = Gn^2 Gn^2 entry by entry), and
// writes A, b and the six features the ZF kernel's network reads
// (zf_mixed.cu, poly_init): t2 - 1, t3 - 3 t2 + 2, t4 - 4 t3 + 6 t2 - 3,
// min and max of diag(Gn) minus 1, and K / M.
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "zf.cuh"

namespace mb {
namespace {

constexpr int kTT = 256;

// C = A B, K x K complex (row-major, leading dimension K), all threads
__device__ void dmatmul(const double2 *A, const double2 *B, double2 *C, uint32_t K) {
  for (uint32_t e = threadIdx.x; e < K * K; e += kTT) {
    const uint32_t i = e / K, j = e % K;
    double re = 0.0, im = 0.0;
    for (uint32_t k = 0; k < K; k++) {
      const double2 a = A[i * K + k], b = B[k * K + j];
      re += a.x * b.x - a.y * b.y;
      im += a.x * b.y + a.y * b.x;
    }
    C[e] = make_double2(re, im);
  }
}

__global__ void __launch_bounds__(kTT) zf_init_targets_kernel(const float2 *csi, uint32_t M, uint32_t K,
                                                              float *feat, float *A, float *bv) {
  extern __shared__ __align__(16) unsigned char zsm[];
  double2 *Gd = reinterpret_cast<double2 *>(zsm), *P2 = Gd + K * K, *P3 = P2 + K * K;
  __shared__ double red[7][kTT];
  __shared__ double sc[4];  // tau, dmin, dmax
  const uint32_t g = blockIdx.x, tid = threadIdx.x;
  const float2 *c = csi + (uint64_t)g * M * K;
  for (uint32_t e = tid; e < K * K; e += kTT) {
    const uint32_t u = e / K, v = e % K;
    double re = 0.0, im = 0.0;
    for (uint32_t b = 0; b < M; b++) {
      const float2 x = c[b * K + u], y = c[b * K + v];  // x conj(y)
      re += (double)x.x * y.x + (double)x.y * y.y;
      im += (double)x.y * y.x - (double)x.x * y.y;
    }
    Gd[e] = make_double2(re, im);
  }
  __syncthreads();
  if (tid == 0) {
    double tr = 0.0, mn = INFINITY, mx = -INFINITY;
    for (uint32_t i = 0; i < K; i++) {
      const double d = Gd[i * K + i].x;
      tr += d;
      mn = fmin(mn, d);
      mx = fmax(mx, d);
    }
    sc[0] = tr / K;
    sc[1] = mn;
    sc[2] = mx;
  }
  __syncthreads();
  const double tau = sc[0], it = tau > 0.0 ? 1.0 / tau : 0.0;
  for (uint32_t e = tid; e < K * K; e += kTT) Gd[e] = make_double2(Gd[e].x * it, Gd[e].y * it);
  __syncthreads();
  dmatmul(Gd, Gd, P2, K);
  __syncthreads();
  dmatmul(Gd, P2, P3, K);
  __syncthreads();
  // t2..t8 (all real for Hermitian powers)
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
  for (uint32_t e = tid; e < K * K; e += kTT) {
    const uint32_t i = e / K, j = e % K;
    const double2 a = Gd[e], p = P2[e], q = P3[e];
    double4 p4 = make_double4(0, 0, 0, 0);  // (Gn^4)_ij = sum_k P2_ik P2_kj
    for (uint32_t k = 0; k < K; k++) {
      const double2 x = P2[i * K + k], y = P2[k * K + j];
      p4.x += x.x * y.x - x.y * y.y;
      p4.y += x.x * y.y + x.y * y.x;
    }
    s[0] += a.x * a.x + a.y * a.y;        // tr Gn^2 = ||Gn||^2
    s[1] += a.x * p.x + a.y * p.y;        // tr Gn^3 = <Gn, Gn^2>
    s[2] += p.x * p.x + p.y * p.y;        // tr Gn^4 = ||Gn^2||^2
    s[3] += p.x * q.x + p.y * q.y;        // tr Gn^5 = <Gn^2, Gn^3>
    s[4] += q.x * q.x + q.y * q.y;        // tr Gn^6 = ||Gn^3||^2
    s[5] += q.x * p4.x + q.y * p4.y;      // tr Gn^7 = <Gn^3, Gn^4>
    s[6] += p4.x * p4.x + p4.y * p4.y;    // tr Gn^8 = ||Gn^4||^2
  }
  for (int k = 0; k < 7; k++) red[k][tid] = s[k];
  __syncthreads();
  for (uint32_t o = kTT / 2; o > 0; o >>= 1) {
    if (tid < o)
      for (int k = 0; k < 7; k++) red[k][tid] += red[k][tid + o];
    __syncthreads();
  }
  if (tid == 0) {
    double t[9];
    t[0] = 1.0;
    t[1] = 1.0;
    for (int k = 0; k < 7; k++) t[k + 2] = red[k][0] / K;
    for (int i = 0; i < 4; i++) {
      bv[(uint64_t)g * 4 + i] = (float)t[i + 1];
      for (int j = 0; j < 4; j++) A[((uint64_t)g * 4 + i) * 4 + j] = (float)t[i + j + 2];
    }
    float *f = feat + (uint64_t)g * kZfInitFeatures;
    f[0] = (float)(t[2] - 1.0);
    f[1] = (float)(t[3] - 3.0 * t[2] + 2.0);
    f[2] = (float)(t[4] - 4.0 * t[3] + 6.0 * t[2] - 3.0);
    f[3] = (float)(sc[1] * it - 1.0);
    f[4] = (float)(sc[2] * it - 1.0);
    f[5] = (float)K / (float)M;
  }
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" mb_status mb_zf_init_targets(const mb_c32 *csi, uint32_t groups, uint32_t M, uint32_t K,
                                        float *features, float *A, float *b, void *stream) {
  if (!csi || !features || !A || !b) return MB_BAD_ARG;
  if (M == 0 || K == 0 || K > 64 || K > M) return MB_BAD_SHAPE;
  if (groups == 0) return MB_OK;
  const size_t smem = 3 * (size_t)K * K * sizeof(double2);
  // the static reductions (14 KB) and up to 192 KB of powers need the opt-in
  // limit whatever K is: raise it once per device to the K = 64 size
  static std::atomic<uint64_t> configured{0};
  int dev = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  if (!(configured.load() & bit)) {
    MB_CUDA_TRY(cudaFuncSetAttribute(zf_init_targets_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(3 * 64 * 64 * sizeof(double2))));
    configured.fetch_or(bit);
  }
  zf_init_targets_kernel<<<groups, kTT, smem, as_stream(stream)>>>(reinterpret_cast<const float2 *>(csi), M,
                                                                   K, features, A, b);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

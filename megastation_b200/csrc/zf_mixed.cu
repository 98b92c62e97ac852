// zf_mixed.cu -- mixed-precision zero forcing on the tensor cores.
//
// The reference computes W = (C C^H)^{-1} C per subcarrier group with cuBLAS
// Cgemm + cuSOLVER potrf/potrs in FP32 (beamform/beamform.cu:74-122).  Here
// one CTA per group does, in one kernel:
//  1. Gram on tcgen05: with R(C) the real embedding of C (row 2u = [Re C_u,
//     -Im C_u], row 2u+1 = [Im C_u, Re C_u] over the reduction index
//     kk = plane*Mp + b), R(G) = R(C) R(C)^T.  Plane 1 of R(C) is P times
//     plane 0 (P = diag of [[0,-1],[1,0]] blocks), so only the plane-0 tiles
//     T are multiplied: A = sum T T^T and R(G) = A + P A P^T.  T is split
//     into BF16 hi + lo parts and A ~ hi hi^T + hi lo^T + lo hi^T
//     accumulates in FP32 in tensor memory: BF16 operands, FP32
//     accumulation, and a Gram accurate to ~2^-16 (a plain BF16 Gram costs
//     ~0.25 dB of EVM at 256x32, which the split removes).  The same
//     shared-memory tile is both MMA operands (A = T, B^T = T, both K-major).
//  2. FP32 Gauss-Jordan inverse X of G (registers, one barrier per pivot)
//     or the learned polynomial start, ns_iters Newton-Schulz steps
//     X <- X (2I - G X), then the 1-norm condition estimate ||G||_1 ||X||_1.
//     For K <= 32 every matrix product of this step (the powers of G of the
//     learned start and both products of each Newton-Schulz step) runs on
//     tcgen05 as 64 x 64 x 64 products of split-BF16 real embeddings, on
//     the normalised Gn = G / tau and Y = tau X; W then reads Y's BF16
//     image and scales by 1 / tau.  For 32 < K <= 64 they run on the CUDA
//     cores.
//  3. W = X C on tcgen05: D0 = R(X) T over the plane-0 tiles, which stay in
//     shared memory from step 1 (re-built from the CSI when they do not
//     fit), gives row for row the plane-0 half of the detector image the
//     tensor-core equalizer consumes (eq_tc.cu); the plane-1 half is P D0.
//     The epilogue stores that image (BF16) and W in the CSI layout (FP32).
//  4. Groups whose Gram is not positive definite in FP32, or whose condition
//     estimate exceeds cond_threshold, are redone in FP64 (Gram, Cholesky,
//     solve) and reported with status 2 (1 if even FP64 fails).
#include <algorithm>
#include <atomic>
#include <cstring>

#include "common.cuh"
#include "eq_tc.cuh"
#include "eq_tc_epi.cuh"
#include "tc.cuh"
#include "zf.cuh"

namespace mb {

namespace {
constexpr int kKT = 64;        // reduction elements per k tile
constexpr float kPolyAccept = 0.04f;  // ||I - G X||_F before the last step of an accepted learned iterate
constexpr int kThreads = 256;  // 8 warps; warps w and w+4 share TMEM lane quadrant w
constexpr uint32_t kZfStageWidth = 64;  // networks up to this width are staged in shared memory
constexpr uint32_t kTcMinK = 16;        // K above this (and <= 32): the inverse's products on the tensor cores

struct ZfmParams {
  ZfNetView net;      // network of the learned initial iterate (used when learned)
  uint32_t learned;   // 1: initial iterate from the learned polynomial, exact inverse as fallback
  float2 *csi;        // [G][M][K]: in CSI, out W (FP32)
  uint8_t *img_w;     // [G] detector images for the equalizer (BF16)
  int32_t *status;
  float *cond;
  float *wmax;        // per group max |W| (precoder scaling), or null
  int *err;
  uint32_t M, K, Mp, nkt, ns_iters;
  uint32_t nh;        // plane-0 k tiles: Mp / 64
  uint32_t resident;  // 1: all nh hi tiles stay in shared memory for W = X C
  uint32_t write_w;   // 1: also store W (FP32, CSI layout); 0: the detector image only
  uint32_t net_bulk;  // 1: the network's six arrays come into shared memory by bulk copies (MM == 64)
  uint32_t csi_nst;   // MM == 64: CSI k tiles staged by bulk copies, csi_nst at a time (0: register loads)
  uint32_t tcns;      // MM == 64: 1 the inverse's products on the tensor cores, 0 on the CUDA cores
  float cond_thr;
  // fused equalize (kernels with QMF > 0): the LLR layout and outputs of
  // the group's eq_nb symbols, eq_spc of them per 128-column tile, eq_nct
  // tiles; eq_N = 2K padded to 16
  EqParams ep;
  uint32_t eq_nb, eq_spc, eq_nct, eq_N;
};

__device__ __forceinline__ uint32_t img_off(uint32_t r, uint32_t kk, uint32_t MM) {
  // canonical K-major, no swizzle: [k tile][row group][k chunk][row][8]
  const uint32_t kt = kk / kKT, kin = kk % kKT;
  return kt * (MM * kKT * 2) + (r / 8) * 1024 + (kin / 8) * 128 + (r % 8) * 16 + (kin % 8) * 2;
}

// In-place Cholesky of the K x K Hermitian matrix A (lower, leading dim lda)
// by all threads; returns false when a pivot is not positive.
template <typename C, typename R>
__device__ bool chol_smem(C *A, uint32_t K, uint32_t lda, int *flag) {
  const int tid = threadIdx.x, nt = blockDim.x;
  if (tid == 0) *flag = 0;
  __syncthreads();
  for (uint32_t j = 0; j < K; j++) {
    if (tid == 0) {
      R d = A[j * lda + j].x;
      if (!(d > (R)0)) {
        *flag = 1;
        d = (R)1;
      }
      A[j * lda + j].x = sqrt(d);
      A[j * lda + j].y = 0;
    }
    __syncthreads();
    const R inv = (R)1 / A[j * lda + j].x;
    for (uint32_t i = j + 1 + tid; i < K; i += nt) {
      A[i * lda + j].x *= inv;
      A[i * lda + j].y *= inv;
    }
    __syncthreads();
    const uint32_t rem = K - j - 1;
    for (uint32_t q = tid; q < rem * rem; q += nt) {
      const uint32_t i = j + 1 + q / rem, k = j + 1 + q % rem;
      if (k > i) continue;
      const C a = A[i * lda + j], b = A[k * lda + j];
      A[i * lda + k].x -= a.x * b.x + a.y * b.y;
      A[i * lda + k].y -= a.y * b.x - a.x * b.y;
    }
    __syncthreads();
  }
  return *flag == 0;
}

// Inverse of the K x K Hermitian positive definite matrix G (leading dim ld)
// into X by in-place Gauss-Jordan without pivoting (every pivot of a
// positive definite matrix is real and positive): at pivot k the pivot row
// becomes a_kj / a_kk with a_kk <- 1 / a_kk, and every other row i becomes
// a_ij - a_ik a_kj' with a_ik <- -a_ik / a_kk, so column k of G is replaced
// by column k of the inverse and no identity half is carried.  The matrix is
// padded to KP x KP with an identity block.  Thread t holds row t / TPR in
// registers, columns t % TPR + TPR m; the pivot row goes through shared
// memory (prow, two buffers of KP), so each pivot costs one barrier.  The
// register row is rotated by one slot after every TPR pivots, so the pivot
// column always sits in slot 0 and the loop body indexes registers
// statically without being unrolled over the row (a short body: the
// unrolled form stalled on instruction fetch at KP = 64).
// Returns false when a pivot is not positive (the output is then garbage).
template <int KP>
__device__ __forceinline__ bool gj_inverse(const float2 *G, float2 *X, uint32_t K, uint32_t ld,
                                           float2 *prow, int *bad) {
  constexpr int TPR = kThreads / KP, NC = KP / TPR;
  const uint32_t i = threadIdx.x / TPR, sub = threadIdx.x % TPR;
  // v[m] holds column sub + TPR ((m + r) % NC) after r rotations
  float2 v[NC];
#pragma unroll
  for (int m = 0; m < NC; m++) {
    const uint32_t c = sub + TPR * m;
    v[m] = (i < K && c < K) ? G[i * ld + c] : make_float2(i == c ? 1.f : 0.f, 0.f);
  }
#pragma unroll 1
  for (uint32_t r = 0; r < (uint32_t)NC; r++) {
#pragma unroll
    for (int s = 0; s < TPR; s++) {
      const uint32_t k = r * TPR + s;
      float2 f;  // this row's entry in column k
      f.x = __shfl_sync(0xffffffffu, v[0].x, s, TPR);
      f.y = __shfl_sync(0xffffffffu, v[0].y, s, TPR);
      float2 *pr = prow + (k & 1) * KP;
      if (i == k) {
        if (!(f.x > 0.f)) *bad = 1;
        const float inv = __frcp_rn(f.x);
        if (sub == (uint32_t)s) v[0] = make_float2(1.f, 0.f);
#pragma unroll
        for (int m = 0; m < NC; m++) {
          v[m].x *= inv;
          v[m].y *= inv;
          pr[sub + TPR * m] = v[m];
        }
      }
      __syncthreads();
      if (i != k) {
        if (sub == (uint32_t)s) v[0] = make_float2(0.f, 0.f);
#pragma unroll
        for (int m = 0; m < NC; m++) {
          const float2 w = pr[sub + TPR * m];
          v[m].x -= f.x * w.x - f.y * w.y;
          v[m].y -= f.x * w.y + f.y * w.x;
        }
      }
    }
    const float2 t = v[0];
#pragma unroll
    for (int m = 0; m < NC - 1; m++) v[m] = v[m + 1];
    v[NC - 1] = t;
  }
  __syncthreads();
  const bool ok = *bad == 0;
  if (i < K) {
#pragma unroll
    for (int m = 0; m < NC; m++) {
      const uint32_t c = sub + TPR * m;
      if (c < K) X[i * ld + c] = v[m];
    }
  }
  __syncthreads();
  return ok;
}

// C = A B for K x K complex matrices in shared memory (leading dims given);
// out(i, j, c) receives each entry.  Thread t owns the outputs
// (t / 16 + 16a, t % 16 + 16b), a, b < T: T*T independent accumulators that
// share each A and B load.  Needs 256 threads and K <= 16 T.  HERM: C is
// known to be Hermitian, so only the 16 x 16 blocks a <= b are computed and
// the blocks below the diagonal are written as their conjugate transposes.
template <int T, bool HERM, typename Out>
__device__ __forceinline__ void cmatmul(const float2 *A, uint32_t lda, const float2 *B, uint32_t ldb,
                                        uint32_t K, Out out) {
  const uint32_t ti = threadIdx.x / 16, tj = threadIdx.x % 16;
  float2 acc[T][T];
#pragma unroll
  for (int a = 0; a < T; a++)
#pragma unroll
    for (int b = 0; b < T; b++) acc[a][b] = make_float2(0.f, 0.f);
#pragma unroll 4
  for (uint32_t k = 0; k < K; k++) {
    float2 av[T], bv[T];
#pragma unroll
    for (int a = 0; a < T; a++) {
      const uint32_t i = ti + 16 * a;
      av[a] = i < K ? A[i * lda + k] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int b = 0; b < T; b++) {
      const uint32_t j = tj + 16 * b;
      bv[b] = j < K ? B[k * ldb + j] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int a = 0; a < T; a++)
#pragma unroll
      for (int b = 0; b < T; b++) {
        if (HERM && a > b) continue;
        acc[a][b].x = fmaf(av[a].x, bv[b].x, fmaf(-av[a].y, bv[b].y, acc[a][b].x));
        acc[a][b].y = fmaf(av[a].x, bv[b].y, fmaf(av[a].y, bv[b].x, acc[a][b].y));
      }
  }
#pragma unroll
  for (int a = 0; a < T; a++)
#pragma unroll
    for (int b = 0; b < T; b++) {
      if (HERM && a > b) continue;
      const uint32_t i = ti + 16 * a, j = tj + 16 * b;
      if (i < K && j < K) {
        out(i, j, acc[a][b]);
        if (HERM && a < b) out(j, i, make_float2(acc[a][b].x, -acc[a][b].y));
      }
    }
}

// K <= MM / 2: MM = 64 covers K <= 32, MM = 128 covers K <= 64
template <int MM, bool HERM = false, typename Out>
__device__ __forceinline__ void cmatmul_any(const float2 *A, uint32_t lda, const float2 *B, uint32_t ldb,
                                            uint32_t K, Out out) {
  if (MM == 64) {
    if (K <= 16)
      cmatmul<1, HERM>(A, lda, B, ldb, K, out);
    else
      cmatmul<2, HERM>(A, lda, B, ldb, K, out);
  } else {
    if (K <= 48)
      cmatmul<3, HERM>(A, lda, B, ldb, K, out);
    else
      cmatmul<4, HERM>(A, lda, B, ldb, K, out);
  }
}

// Block sums of three values and the block min / max of two; every thread
// gets the results.  sred holds 5 x 8 floats.
__device__ __forceinline__ void block_reduce5(float &a, float &b, float &c, float &mn, float &mx,
                                              float *sred) {
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if (lane == 0) {
    sred[warp] = a;
    sred[8 + warp] = b;
    sred[16 + warp] = c;
    sred[24 + warp] = mn;
    sred[32 + warp] = mx;
  }
  __syncthreads();
  a = b = c = 0.f;
  mn = INFINITY;
  mx = -INFINITY;
#pragma unroll
  for (int w = 0; w < kThreads / 32; w++) {
    a += sred[w];
    b += sred[8 + w];
    c += sred[16 + w];
    mn = fminf(mn, sred[24 + w]);
    mx = fmaxf(mx, sred[32 + w]);
  }
  __syncthreads();
}

// The learned iterate's network on the CTA's threads: the six features in
// coef[0..5] -> the four coefficients in coef[8..11].  BF16 weights, and
// features and hidden activations rounded to BF16 into every product, FP32
// accumulation, ReLU hidden layers (the arithmetic of mb_mlp_forward,
// mlp.cu).  act holds 2 kZfInitMaxWidth floats.
__device__ __forceinline__ void zf_net_eval(const ZfNetView &net, float *act, float *coef) {
  const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
  const uint32_t W = net.width;
  auto bf = [](float x) { return __bfloat162float(__float2bfloat16_rn(x)); };
  if ((uint32_t)tid < W) {
    float h = net.b1[tid];
#pragma unroll
    for (uint32_t k = 0; k < kZfInitFeatures; k++) h = fmaf(bf(coef[k]), __bfloat162float(net.w1[k * W + tid]), h);
    act[tid] = bf(fmaxf(h, 0.f));
  }
  __syncthreads();
  if ((uint32_t)tid < W) {
    float h = net.b2[tid];
#pragma unroll 8
    for (uint32_t k = 0; k < W; k++) h = fmaf(act[k], __bfloat162float(net.w2[k * W + tid]), h);
    act[kZfInitMaxWidth + tid] = bf(fmaxf(h, 0.f));
  }
  __syncthreads();
  if (warp < (int)kZfInitCoeffs) {
    float y = 0.f;
    for (uint32_t k = lane; k < W; k += 32)
      y = fmaf(act[kZfInitMaxWidth + k], __bfloat162float(net.w3[k * kZfInitCoeffs + warp]), y);
    for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
    if (lane == 0) coef[8 + warp] = y + net.b3[warp];
  }
  __syncthreads();
}

// ---- 64 x 64 real matrices on the tensor cores (K <= 32).  The real
// embeddings R(Z) (row 2u: [Re Z_uv, -Im Z_uv], row 2u+1: [Im Z_uv, Re Z_uv]
// over columns 2v, 2v+1; R(A B) = R(A) R(B)) of the K x K complex matrices
// of the inverse, zero-padded to 64 x 64, are held in shared memory as
// BF16 images in the canonical no-swizzle layout of img_off (8 KB each), a
// matrix M as hi = bf16(M) and lo = bf16(M - hi).  A product A B is then
// A_hi B_hi + A_hi B_lo + A_lo B_hi accumulated in FP32 in tensor memory:
// BF16 operands, an error of ~2^-16 of the entries (the split-BF16 Gram's
// accuracy) and one 64 x 64 x 64 MMA per term.  The left operand is read
// K-major (its rows), the right one MN-major (its rows are the reduction
// index), so every product is exact as written, symmetric or not.
constexpr uint32_t kSqImg = 64 * 64 * 2;

// one term: D (+)= A B, a0 / b0 the images' shared-memory addresses
__device__ __forceinline__ void sq_mma(uint32_t tmem, uint32_t a0, uint32_t b0, bool acc, uint32_t idesc) {
#pragma unroll
  for (int ks = 0; ks < 4; ks++) {
    // A: K core matrices 128 B apart, 8-row groups 1024 B apart; B: 8-row
    // K groups 1024 B apart, 8-column MN chunks 128 B apart
    const uint64_t ad = tc::smem_desc(a0 + ks * 256, 128, 1024);
    const uint64_t bd = tc::smem_desc(b0 + ks * 2048, 1024, 128);
    tc::mma_f16(tmem, ad, bd, idesc, (acc || ks) ? 1u : 0u);
  }
}

// D = A B for split A (ah, al) and B (bh, bl)
__device__ __forceinline__ void sq_mma3(uint32_t tmem, const uint8_t *ah, const uint8_t *al, const uint8_t *bh,
                                        const uint8_t *bl, uint32_t idesc) {
  sq_mma(tmem, tc::smem_u32(ah), tc::smem_u32(bh), false, idesc);
  sq_mma(tmem, tc::smem_u32(ah), tc::smem_u32(bl), true, idesc);
  sq_mma(tmem, tc::smem_u32(al), tc::smem_u32(bh), true, idesc);
}

// 8 values of one row (8 consecutive columns, one 16-byte core row) into
// the split images (lo may be null)
__device__ __forceinline__ void sq_put8(uint8_t *hi, uint8_t *lo, uint32_t off, const float *v) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const __nv_bfloat162 a = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
    const float2 f = __bfloat1622float2(a);
    const __nv_bfloat162 b = __floats2bfloat162_rn(v[2 * e] - f.x, v[2 * e + 1] - f.y);
    h[e] = *reinterpret_cast<const uint32_t *>(&a);
    l[e] = *reinterpret_cast<const uint32_t *>(&b);
  }
  *reinterpret_cast<uint4 *>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
  if (lo) *reinterpret_cast<uint4 *>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

// hi + lo of 8 values of one row
__device__ __forceinline__ void sq_get8(const uint8_t *hi, const uint8_t *lo, uint32_t off, float *v) {
  const uint4 a = *reinterpret_cast<const uint4 *>(hi + off), b = *reinterpret_cast<const uint4 *>(lo + off);
  const uint32_t aw[4] = {a.x, a.y, a.z, a.w}, bw[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const float2 fa = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&aw[e]));
    const float2 fb = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&bw[e]));
    v[2 * e] = fa.x + fb.x;
    v[2 * e + 1] = fa.y + fb.y;
  }
}

// two neighbouring values (c even) of one row into the split images
__device__ __forceinline__ void sq_put2(uint8_t *hi, uint8_t *lo, uint32_t r, uint32_t c, float x, float y) {
  const __nv_bfloat162 a = __floats2bfloat162_rn(x, y);
  const float2 f = __bfloat1622float2(a);
  const uint32_t off = img_off(r, c, 64);
  *reinterpret_cast<__nv_bfloat162 *>(hi + off) = a;
  *reinterpret_cast<__nv_bfloat162 *>(lo + off) = __floats2bfloat162_rn(x - f.x, y - f.y);
}

__device__ __forceinline__ float2 sq_get2(const uint8_t *hi, const uint8_t *lo, uint32_t r, uint32_t c) {
  const uint32_t off = img_off(r, c, 64);
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(hi + off));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(lo + off));
  return make_float2(a.x + b.x, a.y + b.y);
}

// this thread's part of a 64 x 64 FP32 accumulator at tmem: row r = 16
// (warp % 4) + lane of the 16 lanes per quadrant an M = 64 MMA writes,
// 16-column chunks warp / 4 and warp / 4 + 2; f(r, c0, v) gets the 16
// values of columns c0 .. c0 + 15 (lanes 16..31 only take part in the
// warp-collective loads).  Two 16-column loads measured faster here than
// one 32-column load.
template <typename F>
__device__ __forceinline__ void sq_readout(uint32_t tmem, F f) {
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const uint32_t r = (warp % 4) * 16 + lane;
#pragma unroll 1
  for (uint32_t j = 0; j < 2; j++) {
    const uint32_t ch = warp / 4 + 2 * j;
    float v[16];
    tc::tmem_ld16(tmem + ((uint32_t)((warp % 4) * 32) << 16) + ch * 16, v);
    if (lane < 16) f(r, ch * 16, v);
  }
}

// Learned polynomial initial iterate (no reference counterpart).  With
// tau = tr(G) / K and Gn = G / tau, the initial iterate is
// X0 = (a0 I + a1 Gn + a2 Gn^2 + a3 Gn^3) / tau, whose coefficients a come
// from the network evaluated on six scale-free features of the group:
// with t_k = tr(Gn^k) / K (t_1 = 1), the central moments of Gn's
// eigenvalues t2 - 1, t3 - 3 t2 + 2 and t4 - 4 t3 + 6 t2 - 3 (Gn^2 is
// needed for the iterate anyway, so t3 = <Gn, Gn^2> / K and t4 =
// ||Gn^2||^2 / K cost no product of their own), the smallest and largest
// diagonal entry of Gn minus 1, and K / M.  ns_iters Newton-Schulz steps
// X <- X (2I - G X) follow, and at most two more while the residual is
// below 0.3 but above the acceptance bound; X stays a polynomial in G, so
// both products are Hermitian and only their upper blocks are computed.
// The Frobenius norm of E = I - G X comes with every step's first product;
// the iterate is accepted when the last one is at most kPolyAccept = 0.04
// (the returned X then has ||I - G X||_F <= 1.6e-3, below the BF16 rounding
// of the detector image), otherwise the caller falls back to the exact
// inverse.  The network: BF16 weights and activations into every product,
// FP32 accumulation, ReLU hidden layers (the arithmetic of mb_mlp_forward).
// Result in Xs.  This CUDA-core form serves 32 < K <= 64 (MM = 128); for
// K <= 32 the kernel takes the same steps with its products on the tensor
// cores (the sq_* helpers above).
template <int MM>
__device__ bool poly_init(const float2 *Gs, uint32_t ld, float2 *Xs, float2 *P2, float2 *P3, float2 *Ts,
                          float2 *Xn, uint32_t K, uint32_t M, const ZfNetView &net, uint32_t ns_iters,
                          float *sred, float *act, float *coef) {
  const int tid = threadIdx.x;
  // tau and the diagonal's range
  float d = 0.f, z1 = 0.f, z2 = 0.f, dmin = INFINITY, dmax = -INFINITY;
  for (uint32_t i = tid; i < K; i += kThreads) {
    const float g = Gs[i * ld + i].x;
    d += g;
    dmin = fminf(dmin, g);
    dmax = fmaxf(dmax, g);
  }
  block_reduce5(d, z1, z2, dmin, dmax, sred);
  const float tau = d / (float)K;
  if (!(tau > 0.f) || !(dmin > 0.f)) return false;  // uniform
  const float it = 1.f / tau, it2 = it * it;
  // Gn^2 (Hermitian)
  cmatmul_any<MM, true>(Gs, ld, Gs, ld, K,
                        [&](uint32_t i, uint32_t j, float2 s) { P2[i * K + j] = make_float2(s.x * it2, s.y * it2); });
  __syncthreads();
  // t2, t3, t4
  float a2 = 0.f, a3 = 0.f, a4 = 0.f, n0 = INFINITY, n1 = -INFINITY;
  for (uint32_t e = tid; e < K * K; e += kThreads) {
    const float2 g = Gs[(e / K) * ld + e % K], p = P2[e];
    const float gx = g.x * it, gy = g.y * it;
    a2 += gx * gx + gy * gy;
    a3 += gx * p.x + gy * p.y;
    a4 += p.x * p.x + p.y * p.y;
  }
  block_reduce5(a2, a3, a4, n0, n1, sred);
  const float t2 = a2 / (float)K, t3 = a3 / (float)K, t4 = a4 / (float)K;
  // the network: layer 1 (6 -> width), layer 2 (width -> width), layer 3
  // (width -> 4), hidden activations in act[0..width) and act[256..)
  if (tid == 0) {
    coef[0] = t2 - 1.f;
    coef[1] = t3 - 3.f * t2 + 2.f;
    coef[2] = t4 - 4.f * t3 + 6.f * t2 - 3.f;
    coef[3] = dmin * it - 1.f;
    coef[4] = dmax * it - 1.f;
    coef[5] = (float)K / (float)M;
  }
  __syncthreads();
  zf_net_eval(net, act, coef);
  const float c0 = coef[8], c1 = coef[9], c2 = coef[10], c3 = coef[11];
  // Gn^3 = Gn Gn^2 (Hermitian)
  cmatmul_any<MM, true>(Gs, ld, P2, K, K,
                        [&](uint32_t i, uint32_t j, float2 s) { P3[i * K + j] = make_float2(s.x * it, s.y * it); });
  __syncthreads();
  for (uint32_t e = tid; e < K * K; e += kThreads) {
    const uint32_t i = e / K, j = e % K;
    const float2 g = Gs[i * ld + j], p2 = P2[e], p3 = P3[e];
    const float re = (i == j ? c0 : 0.f) + c1 * g.x * it + c2 * p2.x + c3 * p3.x;
    const float im = c1 * g.y * it + c2 * p2.y + c3 * p3.y;
    Xs[i * ld + j] = make_float2(re * it, im * it);
  }
  __syncthreads();
  float2 *xc = Xs, *xn = Xn;
  uint32_t ldc = ld, ldn = K;
  float e_last = INFINITY;
  // ns_iters steps, then up to two more only to rescue a near miss
  // (0.04 < ||E|| < 0.3); a start further off goes to the exact inverse
  for (uint32_t s = 0; s < ns_iters + 2; s++) {
    if (s >= ns_iters && (e_last <= kPolyAccept || e_last >= 0.3f)) break;  // uniform
    float en = 0.f;
    cmatmul_any<MM, true>(Gs, ld, xc, ldc, K, [&](uint32_t i, uint32_t j, float2 v) {
      const float ex = (i == j ? 1.f : 0.f) - v.x, ey = -v.y;  // E = I - G X; T = I + E
      en += ex * ex + ey * ey;
      Ts[i * K + j] = make_float2((i == j ? 1.f : 0.f) + ex, ey);
    });
    float u0 = 0.f, u1 = 0.f, m0 = INFINITY, m1 = -INFINITY;
    block_reduce5(en, u0, u1, m0, m1, sred);  // also orders the Ts writes before their reads
    e_last = sqrtf(en);
    if (!(e_last < 1.f)) return false;  // uniform: the iteration would not converge
    cmatmul_any<MM, true>(xc, ldc, Ts, K, K, [&](uint32_t i, uint32_t j, float2 v) { xn[i * ldn + j] = v; });
    __syncthreads();
    float2 *t = xc;
    xc = xn;
    xn = t;
    const uint32_t l = ldc;
    ldc = ldn;
    ldn = l;
  }
  if (xc != Xs) {
    for (uint32_t e = tid; e < K * K; e += kThreads) Xs[(e / K) * ld + e % K] = xc[e];
    __syncthreads();
  }
  return e_last <= kPolyAccept;
}
}  // namespace

// QMF > 0: the fused form (MM == 64), which keeps the detector image in
// shared memory and equalizes the group's symbols (modulation order QMF)
// from the planar BF16 samples that ymap describes
template <int MM, int QMF>
__global__ void __launch_bounds__(kThreads, MM == 64 ? 2 : 1)
    zf_mixed_kernel(const ZfmParams q, const __grid_constant__ CUtensorMap ymap) {
  static_assert(QMF == 0 || MM == 64, "the fused equalize needs K <= 32");
  extern __shared__ __align__(1024) uint8_t zsm[];
  __shared__ __align__(8) uint64_t tile_bar[2];
  __shared__ __align__(8) uint64_t mma_bar;
  __shared__ __align__(8) uint64_t stage_bar[4];  // CSI tiles staged by bulk copies
  __shared__ __align__(8) uint64_t net_bar;       // the network's weights
  __shared__ float ns_acc[2];                     // residual norms, alternating
  __shared__ __align__(8) uint64_t eq_full[2], eq_empty[2], eq_done;  // fused equalize pipeline
  __shared__ int eq_to;
  __shared__ uint32_t tmem_slot;
  __shared__ int flag, fail, piv_bad;
  __shared__ float red[kThreads], red2[kThreads];
  __shared__ float2 prow[MM];  // Gauss-Jordan pivot rows, two buffers of KP <= MM / 2
  __shared__ float zi_red[40], zi_coef[16];     // learned initial iterate: reductions, features, coefficients
  __shared__ float zi_act[2 * kZfInitMaxWidth];  // and the network's hidden activations

  constexpr uint32_t tile_bytes = MM * kKT * 2;
  constexpr uint32_t TC = 256;             // TMEM columns: the Gram (MM) or TCH W tiles
  constexpr uint32_t TCH = TC / kKT;       // W tiles per TMEM pass
  constexpr int kIpt = MM / 2 * 8 / kThreads;  // tile items per thread (8K <= 4 MM)
  const uint32_t g = blockIdx.x, K = q.K, M = q.M, Mp = q.Mp, nh = q.nh;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const uint32_t ld = K + 1;
  const uint32_t HS = q.resident ? nh : 2;  // hi-tile slots
  // shared memory carve-up
  uint8_t *hi_base = zsm;
  uint8_t *lo_t[2] = {zsm + HS * tile_bytes, zsm + (HS + 1) * tile_bytes};
  // MM == 64 (K <= 32): behind the tiles the split images of Gn = G / tau
  // and of the iterate Y = tau X, then G (K x ld), then K x ld float2 more
  // (the FP64 fallback's Gram spans both) that hold the network's weights
  // when the kernel runs learned.  With the inverse on the tensor cores
  // (16 < K <= 32) X of the exact start and the residual's image go in the
  // lo tiles and W = X C reads the iterate's hi image; with the CUDA-core
  // products (K <= 16: a 16 x 16 product is a fraction of one tensor-core
  // round trip) X and the powers Gn^2, Gn^3 take the Gn images' place and
  // R(X) the iterate's.
  const bool tcns = MM == 64 && q.tcns;  // uniform
  uint8_t *gn_img = zsm + (HS + 2) * tile_bytes;
  uint8_t *y_img = gn_img + 2 * kSqImg;
  // MM == 128: R(X) (MM x MM BF16), G, X, and the powers Gn^2, Gn^3 of the
  // learned initial iterate (allotted only when the kernel runs learned);
  // Newton-Schulz temporaries (leading dim K): T in the lo tiles, the other
  // iterate in the R(X) image (both free between the Gram and W = X C)
  uint8_t *ximg = MM == 64 ? y_img : zsm + (HS + 2) * tile_bytes;
  float2 *Gs = reinterpret_cast<float2 *>(MM == 64 ? y_img + 2 * kSqImg : ximg + MM * MM * 2);
  float2 *Xs = MM == 64 ? reinterpret_cast<float2 *>(tcns ? lo_t[0] : gn_img) : Gs + K * ld;
  float2 *Ts = reinterpret_cast<float2 *>(lo_t[0]);
  float2 *Xn = reinterpret_cast<float2 *>(ximg);
  float2 *P2 = Xs + K * ld, *P3 = P2 + K * K;
  uint8_t *wsm = reinterpret_cast<uint8_t *>(Gs + K * ld);

  float2 *cg = q.csi + (uint64_t)g * M * K;
  // the detector image: global memory, or (fused) shared memory from 0,
  // over the tiles and the Gn images, which are free once W = X C is done
  uint8_t *imgw = QMF ? zsm : q.img_w + (uint64_t)g * q.nkt * tile_bytes;
  // CSI k tile kt (64 antennas x K users, contiguous in [M][K]) staged in
  // the image region, which is free during the Gram
  const uint32_t nst = MM == 64 ? q.csi_nst : 0;
  const uint32_t nstd = nst ? nst : 1;  // divisor of the stage arithmetic (used only when nst > 0)
  const uint32_t ctile = kKT * K * (uint32_t)sizeof(float2);
  auto csi_rows = [&](uint32_t kt) { return min((uint32_t)kKT, M - kt * kKT); };
  auto stage_csi = [&](uint32_t kt) {
    const uint32_t ss = kt % nstd, bytes = csi_rows(kt) * K * (uint32_t)sizeof(float2);
    tc::mbar_arrive_expect_tx(&stage_bar[ss], bytes);
    tc::bulk_g2s(gn_img + ss * ctile, cg + (uint64_t)kt * kKT * K, bytes, &stage_bar[ss]);
  };
  // the network's arrays in shared memory: w1, w2, w3 (BF16), b1, b2, b3
  const uint32_t NW = q.net.width;
  const uint32_t net_sz[6] = {kZfInitFeatures * NW * 2, NW * NW * 2, NW * kZfInitCoeffs * 2, NW * 4, NW * 4,
                              kZfInitCoeffs * 4};
  const void *net_src[6] = {q.net.w1, q.net.w2, q.net.w3, q.net.b1, q.net.b2, q.net.b3};
  const bool net_bulk = MM == 64 && q.learned && q.net_bulk;

  if (tid == 0) {
    tc::mbar_init(&tile_bar[0], 1);
    tc::mbar_init(&tile_bar[1], 1);
    tc::mbar_init(&mma_bar, 1);
    for (int i = 0; i < 4; i++) tc::mbar_init(&stage_bar[i], 1);
    tc::mbar_init(&net_bar, 1);
    if (QMF) {
      for (int i = 0; i < 2; i++) {
        tc::mbar_init(&eq_full[i], 1);
        tc::mbar_init(&eq_empty[i], 1);
      }
      tc::mbar_init(&eq_done, 1);
      eq_to = 0;
      tc::prefetch_tmap(&ymap);
    }
    tc::fence_mbar_init();
    fail = 0;
    piv_bad = 0;
    ns_acc[0] = ns_acc[1] = 0.f;
    for (uint32_t kt = 0; kt < min(nst, nh); kt++) stage_csi(kt);
    if (net_bulk) {
      uint32_t tot = 0;
      for (int i = 0; i < 6; i++) tot += net_sz[i];
      tc::mbar_arrive_expect_tx(&net_bar, tot);
      uint32_t o = 0;
      for (int i = 0; i < 6; i++) {
        tc::bulk_g2s(wsm + o, net_src[i], net_sz[i], &net_bar);
        o += net_sz[i];
      }
    }
  }
  // rows 2K..MM-1 of the R(C) tiles are padding: zero them once
  for (uint32_t c = tid; c < (HS + 2) * tile_bytes / 16; c += kThreads)
    reinterpret_cast<uint4 *>(zsm)[c] = make_uint4(0, 0, 0, 0);
  if (warp == 0) tc::tmem_alloc(&tmem_slot, TC);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;
  uint32_t tiles_used = 0;  // double-buffer uses issued so far
  uint32_t mma_phase = 0;
  bool ok = true;
  // the network the learned start evaluates: its bulk-copied shared-memory
  // copy (waited for after the Gram), else global memory
  ZfNetView netv = q.net;
  if (net_bulk) {
    const __nv_bfloat16 *sw = reinterpret_cast<const __nv_bfloat16 *>(wsm);
    const float *sb = reinterpret_cast<const float *>(wsm + net_sz[0] + net_sz[1] + net_sz[2]);
    netv = ZfNetView{sw, sw + kZfInitFeatures * NW, sw + kZfInitFeatures * NW + NW * NW, sb, sb + NW, sb + 2 * NW, NW};
  }

  // Tile item e < 8K: user u = e % K and antennas 8 (e / K) .. +7 of the
  // k tile, i.e. 16 bytes of rows 2u (Re C) and 2u+1 (Im C).
  auto load_items = [&](uint32_t kt, float2 (&pf)[kIpt][8]) {
#pragma unroll
    for (int j = 0; j < kIpt; j++) {
      const uint32_t e = tid + j * kThreads, u = e % K, b0 = kt * kKT + (e / K) * 8;
#pragma unroll
      for (int i = 0; i < 8; i++)
        pf[j][i] = (e < 8 * K && b0 + i < M) ? cg[(b0 + i) * K + u] : make_float2(0.f, 0.f);
    }
  };
  auto store_items = [&](const float2 (&pf)[kIpt][8], uint8_t *hi, uint8_t *lo) {
#pragma unroll
    for (int j = 0; j < kIpt; j++) {
      const uint32_t e = tid + j * kThreads, u = e % K, bc = e / K;
      if (e >= 8 * K) continue;
      uint32_t h0[4], h1[4], l0[4], l1[4];
#pragma unroll
      for (int i = 0; i < 8; i += 2) {
        const __nv_bfloat162 a0 = __floats2bfloat162_rn(pf[j][i].x, pf[j][i + 1].x);
        const __nv_bfloat162 a1 = __floats2bfloat162_rn(pf[j][i].y, pf[j][i + 1].y);
        const float2 f0 = __bfloat1622float2(a0), f1 = __bfloat1622float2(a1);
        const __nv_bfloat162 r0 = __floats2bfloat162_rn(pf[j][i].x - f0.x, pf[j][i + 1].x - f0.y);
        const __nv_bfloat162 r1 = __floats2bfloat162_rn(pf[j][i].y - f1.x, pf[j][i + 1].y - f1.y);
        h0[i / 2] = *reinterpret_cast<const uint32_t *>(&a0);
        h1[i / 2] = *reinterpret_cast<const uint32_t *>(&a1);
        l0[i / 2] = *reinterpret_cast<const uint32_t *>(&r0);
        l1[i / 2] = *reinterpret_cast<const uint32_t *>(&r1);
      }
      const uint32_t o0 = img_off(2 * u, bc * 8, MM), o1 = img_off(2 * u + 1, bc * 8, MM);
      *reinterpret_cast<uint4 *>(hi + o0) = make_uint4(h0[0], h0[1], h0[2], h0[3]);
      *reinterpret_cast<uint4 *>(hi + o1) = make_uint4(h1[0], h1[1], h1[2], h1[3]);
      if (lo) {
        *reinterpret_cast<uint4 *>(lo + o0) = make_uint4(l0[0], l0[1], l0[2], l0[3]);
        *reinterpret_cast<uint4 *>(lo + o1) = make_uint4(l1[0], l1[1], l1[2], l1[3]);
      }
    }
  };

  // ---------------------------------------------------------------- Gram
  // A = sum over the plane-0 tiles of T T^T (hi hi + hi lo + lo hi); the
  // next tile's CSI loads are in flight while the current one is multiplied
  const uint32_t idesc_g = tc::idesc_bf16(MM, MM, false, false);
  uint32_t staged = min(nst, nh);  // CSI tiles whose bulk copies were issued
  uint32_t consumed = 0;            // and waited for
  {
    float2 pf[kIpt][8];
    if (!nst) load_items(0, pf);
    for (uint32_t kt = 0; kt < nh; kt++, tiles_used++) {
      const uint32_t s = tiles_used % 2, use = tiles_used / 2;
      if (use >= 1 && !tc::mbar_wait(&tile_bar[s], (use - 1) & 1)) ok = false;
      if (nst) {
        if (!tc::mbar_wait(&stage_bar[kt % nstd], (kt / nstd) & 1)) ok = false;
        else consumed = kt + 1;
      }
      if (__syncthreads_or(!ok)) break;
      if (nst) {
        // the staged tile, [antenna][user], rows beyond M read as zero
        const float2 *st = reinterpret_cast<const float2 *>(gn_img + (kt % nstd) * ctile);
        const uint32_t rows = csi_rows(kt);
#pragma unroll
        for (int j = 0; j < kIpt; j++) {
          const uint32_t e = tid + j * kThreads, u = e % K, r0 = (e / K) * 8;
#pragma unroll
          for (int i = 0; i < 8; i++)
            pf[j][i] = (e < 8 * K && r0 + i < rows) ? st[(r0 + i) * K + u] : make_float2(0.f, 0.f);
        }
      }
      uint8_t *hi = hi_base + (q.resident ? kt : s) * tile_bytes;
      store_items(pf, hi, lo_t[s]);
      if (!nst && kt + 1 < nh) load_items(kt + 1, pf);
      tc::fence_proxy_async_smem();
      __syncthreads();
      if (tid == 0) {
        // the stage just read takes the tile nst further on
        if (nst && kt + nst < nh) {
          stage_csi(kt + nst);
          staged = kt + nst + 1;
        }
        tc::fence_after_sync();
        const uint32_t h0 = tc::smem_u32(hi), l0 = tc::smem_u32(lo_t[s]);
#pragma unroll
        for (int ks = 0; ks < kKT / 16; ks++) {
          const uint64_t dh = tc::smem_desc(h0 + ks * 256, 128, 1024);
          const uint64_t dl = tc::smem_desc(l0 + ks * 256, 128, 1024);
          tc::mma_f16(tmem, dh, dh, idesc_g, (kt | ks) != 0);
          tc::mma_f16(tmem, dh, dl, idesc_g, 1);
          tc::mma_f16(tmem, dl, dh, idesc_g, 1);
        }
        tc::mma_commit(&tile_bar[s]);
      }
    }
  }
  // bulk copies land before their shared memory is read or reused or the
  // CTA exits: the network's (issued at the start, long done by now) and,
  // after a wait that gave up, CSI tiles still in flight
  if (net_bulk && !tc::mbar_wait(&net_bar, 0)) ok = false;
  if (tid == 0)
    for (uint32_t kt = consumed; kt < staged; kt++) tc::mbar_wait(&stage_bar[kt % nstd], (kt / nstd) & 1);
  if (ok) {
    if (tid == 0) tc::mma_commit(&mma_bar);
    if (!tc::mbar_wait(&mma_bar, mma_phase & 1)) ok = false;
    mma_phase++;
  }
  if (__syncthreads_or(!ok)) fail = 1;
  tc::fence_after_sync();

  // ----------------------------------------- Gram out, inverse, refinement
  float cond_est = INFINITY;
  int st = 0;
  bool used_learned = false;  // the learned initial iterate was accepted
  float wmx = 0.f;  // this thread's max |W| over the values it stored
  float wscale = 1.f;  // W = wscale * (the R(X) image times C)
  if (!fail) {
    // R(G) = A + P A P^T (plane 1 of R(C) is P times plane 0): rows 2u and
    // 2u+1 of A sit in neighbouring TMEM lanes
    if (warp < 4) {
      const int rows_per_warp = MM == 64 ? 16 : 32;
      const uint32_t r = warp * rows_per_warp + lane;
      for (uint32_t ch = 0; ch < MM / 16; ch++) {
        float v[16], nb[16];
        tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + ch * 16, v);
#pragma unroll
        for (int i = 0; i < 16; i++) nb[i] = __shfl_xor_sync(0xffffffffu, v[i], 1);
        if (lane < rows_per_warp && !(r & 1) && r / 2 < K) {
#pragma unroll
          for (int i = 0; i < 16; i += 2) {
            const uint32_t vcol = (ch * 16 + i) / 2;
            if (vcol < K) Gs[(r / 2) * ld + vcol] = make_float2(v[i] + nb[i + 1], nb[i] - v[i + 1]);
          }
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (tcns) {
      // ---- the inverse on the tensor cores (16 < K <= 32)
      uint8_t *gh = gn_img, *gl = gn_img + kSqImg, *yh = y_img, *yl = y_img + kSqImg;
      uint8_t *eimg = lo_t[0];  // E = I - Gn Y (hi only)
      const uint32_t two_k = 2 * K;
      const uint32_t idesc_s = tc::idesc_bf16(64, 64, false, true);
      bool tc_ok = true;  // uniform: every MMA wait so far succeeded
      auto issue = [&](auto f) {
        if (tid == 0) {
          tc::fence_after_sync();
          f();
          tc::mma_commit(&mma_bar);
        }
      };
      auto mma_wait = [&]() {
        const bool w = tc::mbar_wait(&mma_bar, mma_phase & 1);
        mma_phase++;
        if (__syncthreads_or(!w)) tc_ok = false;
        tc::fence_after_sync();
        return tc_ok;
      };
      // complex entries (u8, j8 + 8 m) of the 32 x 32 grid: eight threads a row
      const uint32_t u8 = tid / 8, j8 = tid % 8;
      // tau = tr(G) / K and the diagonal's range
      float d = 0.f, z1 = 0.f, z2 = 0.f, dmin = INFINITY, dmax = -INFINITY;
      for (uint32_t i = tid; i < K; i += kThreads) {
        const float g = Gs[i * ld + i].x;
        d += g;
        dmin = fminf(dmin, g);
        dmax = fmaxf(dmax, g);
      }
      block_reduce5(d, z1, z2, dmin, dmax, zi_red);
      const float tau = d / (float)K;
      bool pd = false;
      if (tau > 0.f && dmin > 0.f) {  // uniform
        const float it = 1.f / tau;
        // Gn images; ||Gn||_F^2 and the 1-norm (largest row sum of |Gn_uv|)
        float f2 = 0.f, rs = 0.f;
#pragma unroll
        for (uint32_t m = 0; m < 4; m++) {
          const uint32_t v = j8 + 8 * m;
          float2 g = make_float2(0.f, 0.f);
          if (u8 < K && v < K) g = make_float2(Gs[u8 * ld + v].x * it, Gs[u8 * ld + v].y * it);
          f2 += g.x * g.x + g.y * g.y;
          rs += sqrtf(g.x * g.x + g.y * g.y);
          sq_put2(gh, gl, 2 * u8, 2 * v, g.x, -g.y);
          sq_put2(gh, gl, 2 * u8 + 1, 2 * v, g.y, g.x);
        }
        rs += __shfl_xor_sync(0xffffffffu, rs, 1);
        rs += __shfl_xor_sync(0xffffffffu, rs, 2);
        rs += __shfl_xor_sync(0xffffffffu, rs, 4);
        tc::fence_proxy_async_smem();
        float a0 = 0.f, a1 = 0.f, n0 = INFINITY, gn1 = rs;
        block_reduce5(f2, a0, a1, n0, gn1, zi_red);
        const float t2 = f2 / (float)K;
        // E = I - Gn Y into its image; returns ||E||_F (complex).  The warps'
        // sums meet in ns_acc[n_res % 2] (the other entry is cleared for the
        // next call: every thread has read it before the barrier below)
        uint32_t n_res = 0;
        auto residual = [&]() {
          issue([&] { sq_mma3(tmem, gh, gl, yh, yl, idesc_s); });
          float en = 0.f;
          if (mma_wait()) {
            sq_readout(tmem, [&](uint32_t r, uint32_t c0, float *v) {
#pragma unroll
              for (int i = 0; i < 16; i++) {
                const float e = ((r == c0 + i && r < two_k) ? 1.f : 0.f) - v[i];
                en += e * e;
                v[i] = e;
              }
              sq_put8(eimg, nullptr, img_off(r, c0, 64), v);
              sq_put8(eimg, nullptr, img_off(r, c0 + 8, 64), v + 8);
            });
          }
          for (int o = 16; o > 0; o >>= 1) en += __shfl_xor_sync(0xffffffffu, en, o);
          if (lane == 0) atomicAdd(&ns_acc[n_res & 1], en);
          if (tid == 0) ns_acc[(n_res + 1) & 1] = 0.f;
          tc::fence_proxy_async_smem();
          tc::fence_before_sync();
          __syncthreads();
          en = ns_acc[n_res & 1];
          n_res++;
          return sqrtf(0.5f * en);  // each complex entry is four real ones
        };
        // Y <- Y + Y E = Y (2I - Gn Y)
        auto refine = [&]() {
          issue([&] {
            sq_mma(tmem, tc::smem_u32(yh), tc::smem_u32(eimg), false, idesc_s);
            sq_mma(tmem, tc::smem_u32(yl), tc::smem_u32(eimg), true, idesc_s);
          });
          if (mma_wait()) {
            sq_readout(tmem, [&](uint32_t r, uint32_t c0, float *v) {
#pragma unroll
              for (int h = 0; h < 2; h++) {
                const uint32_t off = img_off(r, c0 + 8 * h, 64);
                float y[8];
                sq_get8(yh, yl, off, y);
#pragma unroll
                for (int i = 0; i < 8; i++) y[i] += v[8 * h + i];
                sq_put8(yh, yl, off, y);
              }
            });
          }
          tc::fence_proxy_async_smem();
          tc::fence_before_sync();
          __syncthreads();
        };
        if (q.learned) {
          // Gn^2 = Gn Gn into the iterate's images; t3 = <Gn, Gn^2> / K and
          // t4 = ||Gn^2||_F^2 / K (each complex entry is four real ones)
          issue([&] { sq_mma3(tmem, gh, gl, gh, gl, idesc_s); });
          float a3 = 0.f, a4 = 0.f;
          if (mma_wait()) {
            sq_readout(tmem, [&](uint32_t r, uint32_t c0, float *v) {
#pragma unroll
              for (int h = 0; h < 2; h++) {
                const uint32_t off = img_off(r, c0 + 8 * h, 64);
                float g[8];
                sq_get8(gh, gl, off, g);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                  a3 += g[i] * v[8 * h + i];
                  a4 += v[8 * h + i] * v[8 * h + i];
                }
                sq_put8(yh, yl, off, v + 8 * h);
              }
            });
          }
          tc::fence_proxy_async_smem();
          tc::fence_before_sync();
          float b0 = 0.f, m0 = INFINITY, m1 = -INFINITY;
          block_reduce5(a3, a4, b0, m0, m1, zi_red);
          // Gn^3 = Gn Gn^2 on the tensor cores while the network runs
          if (tc_ok) issue([&] { sq_mma3(tmem, gh, gl, yh, yl, idesc_s); });
          const float t3 = a3 / (2.f * K), t4 = a4 / (2.f * K);
          if (tid == 0) {
            zi_coef[0] = t2 - 1.f;
            zi_coef[1] = t3 - 3.f * t2 + 2.f;
            zi_coef[2] = t4 - 4.f * t3 + 6.f * t2 - 3.f;
            zi_coef[3] = dmin * it - 1.f;
            zi_coef[4] = dmax * it - 1.f;
            zi_coef[5] = (float)K / (float)M;
          }
          __syncthreads();
          zf_net_eval(netv, zi_act, zi_coef);
          const float c0 = zi_coef[8], c1 = zi_coef[9], c2 = zi_coef[10], c3 = zi_coef[11];
          // Y0 = c0 I + c1 Gn + c2 Gn^2 + c3 Gn^3, in place of Gn^2
          if (tc_ok && mma_wait()) {
            sq_readout(tmem, [&](uint32_t r, uint32_t cb, float *v) {
#pragma unroll
              for (int h = 0; h < 2; h++) {
                const uint32_t off = img_off(r, cb + 8 * h, 64);
                float g[8], p[8];
                sq_get8(gh, gl, off, g);
                sq_get8(yh, yl, off, p);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                  const uint32_t c = cb + 8 * h + i;
                  p[i] = ((r == c && r < two_k) ? c0 : 0.f) + c1 * g[i] + c2 * p[i] + c3 * v[8 * h + i];
                }
                sq_put8(yh, yl, off, p);
              }
            });
          }
          tc::fence_proxy_async_smem();
          tc::fence_before_sync();
          __syncthreads();
          // ns_iters steps, then up to two more only to rescue a near miss
          // (0.04 < ||E|| < 0.3); a start further off goes to the exact inverse
          float e_last = INFINITY;
          bool conv = tc_ok;
          for (uint32_t s = 0; s < q.ns_iters + 2 && conv; s++) {
            if (s >= q.ns_iters && (e_last <= kPolyAccept || e_last >= 0.3f)) break;  // uniform
            e_last = residual();
            if (!(e_last < 1.f) || !tc_ok) conv = false;  // uniform: the iteration would not converge
            else refine();
          }
          used_learned = conv && tc_ok && e_last <= kPolyAccept;
        }
        if (!used_learned && tc_ok) {
          // exact start: Gauss-Jordan X of G (into the lo tiles), Y = tau X
          pd = K <= 16 ? gj_inverse<16>(Gs, Xs, K, ld, prow, &piv_bad) : gj_inverse<32>(Gs, Xs, K, ld, prow, &piv_bad);
          if (pd) {
#pragma unroll
            for (uint32_t m = 0; m < 4; m++) {
              const uint32_t v = j8 + 8 * m;
              float2 x = make_float2(0.f, 0.f);
              if (u8 < K && v < K) x = make_float2(Xs[u8 * ld + v].x * tau, Xs[u8 * ld + v].y * tau);
              sq_put2(yh, yl, 2 * u8, 2 * v, x.x, -x.y);
              sq_put2(yh, yl, 2 * u8 + 1, 2 * v, x.y, x.x);
            }
            tc::fence_proxy_async_smem();
            __syncthreads();
            for (uint32_t s = 0; s < q.ns_iters && tc_ok; s++) {
              residual();
              if (tc_ok) refine();
            }
          }
        }
        if ((pd || used_learned) && tc_ok) {
          // 1-norm condition estimate ||G||_1 ||X||_1 = ||Gn||_1 ||Y||_1
          float ys = 0.f;
#pragma unroll
          for (uint32_t m = 0; m < 4; m++) {
            const float2 y = sq_get2(yh, yl, 2 * u8, 2 * (j8 + 8 * m));
            ys += sqrtf(y.x * y.x + y.y * y.y);
          }
          ys += __shfl_xor_sync(0xffffffffu, ys, 1);
          ys += __shfl_xor_sync(0xffffffffu, ys, 2);
          ys += __shfl_xor_sync(0xffffffffu, ys, 4);
          float b0 = 0.f, b1 = 0.f, b2 = 0.f, m0 = INFINITY;
          block_reduce5(b0, b1, b2, m0, ys, zi_red);
          cond_est = gn1 * ys;
          if (!(cond_est <= q.cond_thr)) st = 2;
          wscale = it;  // W = X C = (Y C) / tau
        } else {
          st = 2;
        }
      } else {
        st = 2;  // G is not positive definite in FP32
      }
      if (!tc_ok) fail = 1;
    } else {
      bool pd = false;
      if (q.learned)
        used_learned = poly_init<MM>(Gs, ld, Xs, P2, P3, Ts, Xn, K, M, netv, q.ns_iters, zi_red, zi_act, zi_coef);
      if (!used_learned) {
        if (MM == 64)
          pd = K <= 16 ? gj_inverse<16>(Gs, Xs, K, ld, prow, &piv_bad)
                       : gj_inverse<32>(Gs, Xs, K, ld, prow, &piv_bad);
        else
          pd = gj_inverse<64>(Gs, Xs, K, ld, prow, &piv_bad);
      }
      if (pd) {
        // Newton-Schulz: T = 2I - G X; X <- X T, ping-ponging Xs and Xn
        float2 *xc = Xs, *xn = Xn;
        uint32_t ldc = ld, ldn = K;
        for (uint32_t it = 0; it < q.ns_iters; it++) {
          cmatmul_any<MM>(Gs, ld, xc, ldc, K, [&](uint32_t i, uint32_t j, float2 s) {
            Ts[i * K + j] = make_float2((i == j ? 2.f : 0.f) - s.x, -s.y);
          });
          __syncthreads();
          // X T = 2X - X G X is Hermitian for Hermitian X: upper blocks only
          cmatmul_any<MM, true>(xc, ldc, Ts, K, K,
                                [&](uint32_t i, uint32_t j, float2 s) { xn[i * ldn + j] = s; });
          __syncthreads();
          float2 *t = xc;
          xc = xn;
          xn = t;
          const uint32_t l = ldc;
          ldc = ldn;
          ldn = l;
        }
        if (xc != Xs) {
          for (uint32_t e = tid; e < K * K; e += kThreads) Xs[(e / K) * ld + e % K] = xc[e];
          __syncthreads();
        }
      }
      if (pd || used_learned) {
        // 1-norm condition estimate ||G||_1 ||X||_1 (both Hermitian): thread
        // t sums column j0 + t % 32 over rows t / 32, t / 32 + 8, ...; warp 0
        // adds the eight partial sums and takes the maximum over columns
        float gmax = 0.f, xmax = 0.f;
        for (uint32_t j0 = 0; j0 < K; j0 += 32) {
          const uint32_t j = j0 + lane;
          float sg = 0.f, sx = 0.f;
          if (j < K)
            for (uint32_t i = warp; i < K; i += kThreads / 32) {
              const float2 gv = Gs[i * ld + j], xv = Xs[i * ld + j];
              sg += sqrtf(gv.x * gv.x + gv.y * gv.y);
              sx += sqrtf(xv.x * xv.x + xv.y * xv.y);
            }
          red[tid] = sg;
          red2[tid] = sx;
          __syncthreads();
          if (warp == 0) {
            float a = 0.f, c = 0.f;
            for (uint32_t w = 0; w < kThreads / 32; w++) {
              a += red[w * 32 + lane];
              c += red2[w * 32 + lane];
            }
            for (int o = 16; o > 0; o >>= 1) {
              a = fmaxf(a, __shfl_xor_sync(0xffffffffu, a, o));
              c = fmaxf(c, __shfl_xor_sync(0xffffffffu, c, o));
            }
            if (lane == 0) {
              red[0] = a;
              red2[0] = c;
            }
          }
          __syncthreads();
          gmax = fmaxf(gmax, red[0]);
          xmax = fmaxf(xmax, red2[0]);
          __syncthreads();
        }
        cond_est = gmax * xmax;
        if (!(cond_est <= q.cond_thr)) st = 2;
      } else {
        st = 2;
      }
    }
  }

  // ----------------------------------------------------- W = X C (tensor)
  // D0 = R(X) T0 over the plane-0 tiles; plane 1 of the detector image is
  // P D0 (R(X) commutes with P), so it needs no multiply of its own
  if (!fail && st == 0) {
    // R(X) image, K-major over the reduction index 2v + rj; rows/columns
    // beyond 2K are padding and stay zero.  MM == 64: the iterate's hi image
    // R(Y) = tau R(X) is already there (the epilogue scales by 1 / tau).
    if (!tcns) {
      for (uint32_t c = tid; c < MM * MM * 2 / 16; c += kThreads)
        reinterpret_cast<uint4 *>(ximg)[c] = make_uint4(0, 0, 0, 0);
      __syncthreads();
      for (uint32_t e = tid; e < K * K; e += kThreads) {
        const uint32_t u = e / K, v = e % K;
        const float2 x = Xs[u * ld + v];
        *reinterpret_cast<__nv_bfloat162 *>(ximg + img_off(2 * u, 2 * v, MM)) = __floats2bfloat162_rn(x.x, -x.y);
        *reinterpret_cast<__nv_bfloat162 *>(ximg + img_off(2 * u + 1, 2 * v, MM)) =
            __floats2bfloat162_rn(x.y, x.x);
      }
      tc::fence_proxy_async_smem();
      __syncthreads();
    }
    const uint32_t idesc_w = tc::idesc_bf16(MM, kKT, false, true);
    for (uint32_t kt0 = 0; kt0 < nh && ok; kt0 += TCH) {
      const uint32_t nt = min(TCH, nh - kt0);
      for (uint32_t t = 0; t < nt; t++) {
        uint8_t *hi;
        uint32_t s = 0;
        if (q.resident) {
          hi = hi_base + (kt0 + t) * tile_bytes;
        } else {
          // rebuild the hi tile from the CSI (not yet overwritten: W rows
          // of a tile are stored only after all of its pass is multiplied)
          s = tiles_used % 2;
          const uint32_t use = tiles_used / 2;
          tiles_used++;
          if (use >= 1 && !tc::mbar_wait(&tile_bar[s], (use - 1) & 1)) ok = false;
          if (__syncthreads_or(!ok)) break;
          hi = hi_base + s * tile_bytes;
          float2 pf[kIpt][8];
          load_items(kt0 + t, pf);
          store_items(pf, hi, nullptr);
          tc::fence_proxy_async_smem();
          __syncthreads();
        }
        if (tid == 0) {
          tc::fence_after_sync();
          const uint32_t xa = tc::smem_u32(ximg), cb = tc::smem_u32(hi);
#pragma unroll
          for (int ks = 0; ks < MM / 16; ks++) {
            // A = R(X): k tile ks/4, k chunk pair ks%4
            const uint64_t ad = tc::smem_desc(xa + (ks / 4) * MM * 128 + (ks % 4) * 256, 128, 1024);
            // B = hi tile read MN-major: K groups (8 rows) 1024 B apart,
            // MN chunks (8 kk) 128 B apart
            const uint64_t bd = tc::smem_desc(cb + ks * 2 * 1024, 1024, 128);
            tc::mma_f16(tmem + t * kKT, ad, bd, idesc_w, ks != 0);
          }
          if (!q.resident) tc::mma_commit(&tile_bar[s]);
        }
      }
      if (!ok) break;
      if (tid == 0) tc::mma_commit(&mma_bar);
      if (!tc::mbar_wait(&mma_bar, mma_phase & 1)) ok = false;
      mma_phase++;
      if (__syncthreads_or(!ok)) break;
      tc::fence_after_sync();
      // epilogue: warp w reads lanes of quadrant w % 4, column chunks
      // w / 4, w / 4 + 2, ...; row r, column = antenna b of plane 0
      const int rows_per_warp = MM == 64 ? 16 : 32;
      const uint32_t quad = warp % 4;
      const uint32_t r = quad * rows_per_warp + lane;
      const uint32_t u = r / 2;
      const float sgn = (r & 1) ? 1.f : -1.f;  // plane 1: row 2u = -D0[2u+1], row 2u+1 = D0[2u]
      for (uint32_t ch = warp / 4; ch < nt * kKT / 16; ch += kThreads / 128) {
        float v[16], nb[16];
        tc::tmem_ld16(tmem + ((uint32_t)(quad * 32) << 16) + ch * 16, v);
#pragma unroll
        for (int i = 0; i < 16; i++) {
          v[i] *= wscale;
          nb[i] = __shfl_xor_sync(0xffffffffu, v[i], 1);
        }
        if (lane >= rows_per_warp) continue;
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const uint32_t kk = kt0 * kKT + ch * 16 + h * 8;
          uint32_t p0[4], p1[4];
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const __nv_bfloat162 a = __floats2bfloat162_rn(v[h * 8 + 2 * e], v[h * 8 + 2 * e + 1]);
            const __nv_bfloat162 c =
                __floats2bfloat162_rn(sgn * nb[h * 8 + 2 * e], sgn * nb[h * 8 + 2 * e + 1]);
            p0[e] = *reinterpret_cast<const uint32_t *>(&a);
            p1[e] = *reinterpret_cast<const uint32_t *>(&c);
          }
          *reinterpret_cast<uint4 *>(imgw + img_off(r, kk, MM)) = make_uint4(p0[0], p0[1], p0[2], p0[3]);
          *reinterpret_cast<uint4 *>(imgw + img_off(r, Mp + kk, MM)) = make_uint4(p1[0], p1[1], p1[2], p1[3]);
          if (q.write_w && !(r & 1) && u < K) {
#pragma unroll
            for (int e = 0; e < 8; e++) {
              const uint32_t b = kk + e;
              if (b < M) {
                cg[b * K + u] = make_float2(v[h * 8 + e], nb[h * 8 + e]);
                wmx = fmaxf(wmx, sqrtf(v[h * 8 + e] * v[h * 8 + e] + nb[h * 8 + e] * nb[h * 8 + e]));
              }
            }
          }
        }
      }
      tc::fence_before_sync();
      __syncthreads();
    }
    if (!ok) fail = 1;
  }

  // ------------------------------------------------- FP64 fallback groups
  if (!fail && st == 2) {
    using D2 = double2;
    D2 *Gd = reinterpret_cast<D2 *>(Gs);  // reuses Gs and Xs (2 K*ld float2)
    const uint32_t ldd = K + 1;
    for (uint32_t e = tid; e < K * K; e += kThreads) {
      const uint32_t i = e / K, j = e % K;
      if (j > i) continue;
      double sr = 0, si = 0;
      for (uint32_t b = 0; b < M; b++) {
        const float2 a = cg[b * K + i], c = cg[b * K + j];
        sr += (double)a.x * c.x + (double)a.y * c.y;
        si += (double)a.y * c.x - (double)a.x * c.y;
      }
      Gd[i * ldd + j] = make_double2(sr, si);
    }
    __syncthreads();
    const bool pd = chol_smem<D2, double>(Gd, K, ldd, &flag);
    for (uint32_t c = tid; c < q.nkt * tile_bytes / 16; c += kThreads)
      reinterpret_cast<uint4 *>(imgw)[c] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    if (!pd) st = 1;
    for (uint32_t b = tid; b < M; b += kThreads) {
      D2 z[64];
      for (uint32_t i = 0; i < K; i++) {
        const float2 cv = cg[b * K + i];
        D2 s = make_double2(cv.x, cv.y);
        for (uint32_t k = 0; k < i && pd; k++) {
          const D2 l = Gd[i * ldd + k];
          s.x -= l.x * z[k].x - l.y * z[k].y;
          s.y -= l.x * z[k].y + l.y * z[k].x;
        }
        const double d = pd ? Gd[i * ldd + i].x : 1.0;
        z[i] = make_double2(s.x / d, s.y / d);
      }
      for (int i = (int)K - 1; i >= 0 && pd; i--) {
        D2 s = z[i];
        for (uint32_t k = i + 1; k < K; k++) {
          const D2 l = Gd[k * ldd + i];
          s.x -= l.x * z[k].x + l.y * z[k].y;
          s.y -= l.x * z[k].y - l.y * z[k].x;
        }
        const double d = Gd[i * ldd + i].x;
        z[i] = make_double2(s.x / d, s.y / d);
      }
      // every thread reads its own column b of C before overwriting it
      for (uint32_t u = 0; u < K; u++) {
        const float2 w = pd ? make_float2((float)z[u].x, (float)z[u].y) : make_float2(0.f, 0.f);
        cg[b * K + u] = w;
        wmx = fmaxf(wmx, sqrtf(w.x * w.x + w.y * w.y));
        *reinterpret_cast<__nv_bfloat16 *>(imgw + img_off(2 * u, b, MM)) = __float2bfloat16_rn(w.x);
        *reinterpret_cast<__nv_bfloat16 *>(imgw + img_off(2 * u, Mp + b, MM)) = __float2bfloat16_rn(-w.y);
        *reinterpret_cast<__nv_bfloat16 *>(imgw + img_off(2 * u + 1, b, MM)) = __float2bfloat16_rn(w.y);
        *reinterpret_cast<__nv_bfloat16 *>(imgw + img_off(2 * u + 1, Mp + b, MM)) = __float2bfloat16_rn(w.x);
      }
    }
  }

  if (q.wmax) {
    // block maximum of |W| for the precoder's scaling (beam_utils.cuh:40-80)
    __syncthreads();
    red[tid] = wmx;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
      if (tid < o) red[tid] = fmaxf(red[tid], red[tid + o]);
      __syncthreads();
    }
    if (tid == 0) q.wmax[g] = fail ? 0.f : red[0];
  }
  if (tid == 0) {
    if (q.status) q.status[g] = fail ? 1 : (st == 0 && used_learned ? 3 : st);
    if (q.cond) q.cond[g] = cond_est;
    if (fail && q.err) atomicOr(q.err, tc::kErrTimeout);
  }

  // ------------------------------------------------ fused equalize (QMF)
  // The tensor-core equalizer of eq_tc.cu on this group's columns, with
  // the detector image from shared memory: D (128 x N) = Y (128 x 2Mp) A^T
  // per tile of up to 128 (symbol, subcarrier) columns, the samples in
  // 16-subcarrier x 64-antenna TMA boxes (32-byte swizzle) through two
  // 16 KB stages behind the iterate's images, tile ct accumulating in TMEM
  // columns 64 ct.  One thread loads, one issues the MMAs; then every
  // thread runs the shared epilogue (demap, LLRs, descrambled hard bits).
  if constexpr (QMF > 0) {
    tc::fence_proxy_async_smem();  // the image's generic writes before the MMAs read it
    tc::fence_before_sync();
    __syncthreads();
    if (!fail) {
      const EqParams &p = q.ep;
      constexpr uint32_t kCols = 128, y_tile = kCols * kKT * 2;
      uint8_t *ystage = y_img;
      const uint32_t s_base = g * p.sg, nct = q.eq_nct, total = nct * q.nkt;
      auto tile_cols = [&](uint32_t ct) { return min(q.eq_spc, q.eq_nb - ct * q.eq_spc) * p.sg; };
      uint32_t issued = 0;  // stage loads the loading thread issued
      if (warp == 0 && lane == 0) {
        tc::fence_after_sync();
        for (uint32_t i = 0; i < total; i++) {
          const uint32_t ct = i / q.nkt, kt = i % q.nkt, sgi = i % 2, use = i / 2;
          if (use >= 1 && !tc::mbar_wait(&eq_empty[sgi], (use - 1) & 1)) {
            eq_to = 1;
            break;
          }
          const uint32_t ncols = tile_cols(ct), l_off = ct * q.eq_spc;
          uint8_t *sy = ystage + sgi * y_tile;
          tc::mbar_arrive_expect_tx(&eq_full[sgi], ncols * kKT * 2);
          const uint32_t kk0 = kt * kKT, plane = kk0 / Mp, b0 = kk0 % Mp;
          for (uint32_t j = 0; j < ncols / 16; j++) {
            const uint32_t col0 = j * 16, l = col0 / p.sg, sl = col0 % p.sg;
            const int32_t row = (int32_t)(((l_off + l) * 2 + plane) * M + b0);
            tc::tma_load_2d(sy + j * 16 * 128, &ymap, (int32_t)(s_base + sl), row, &eq_full[sgi]);
          }
          issued = i + 1;
        }
      } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = tc::idesc_bf16(kCols, q.eq_N, true, false);
        bool good = true;
        for (uint32_t i = 0; i < total; i++) {
          const uint32_t ct = i / q.nkt, kt = i % q.nkt, sgi = i % 2, use = i / 2;
          if (!tc::mbar_wait(&eq_full[sgi], use & 1)) {
            good = false;
            break;
          }
          tc::fence_after_sync();
          const uint32_t y0 = tc::smem_u32(ystage + sgi * y_tile), a0 = tc::smem_u32(zsm + kt * tile_bytes);
#pragma unroll
          for (int ks = 0; ks < kKT / 16; ks++) {
            // Y: 32-byte atoms of 16 columns 2048 B apart, 8-antenna K groups
            // 256 B apart; image: K core matrices 128 B apart, row groups 1024 B
            const uint64_t yd = tc::smem_desc_mn_sw32(y0 + ks * 512, 2048, 256);
            const uint64_t ad = tc::smem_desc(a0 + ks * 256, 128, 1024);
            tc::mma_f16(tmem + ct * 64, yd, ad, idesc, (kt | ks) != 0);
          }
          tc::mma_commit(&eq_empty[sgi]);
        }
        // eq_done also after a wait that gave up: it then marks the end of
        // the MMAs that were issued
        tc::mma_commit(&eq_done);
        if (!good) eq_to = 1;
      }
      __syncwarp();
      // everyone: wait for the accumulators (bounded), then the epilogues
      const bool got = tc::mbar_wait(&eq_done, 0);
      if (__syncthreads_or(!got || eq_to)) {
        // give up: the loads still in flight land before the CTA exits.  A
        // stage is reloaded only after its previous load was consumed, so
        // those are among the last two issued, each the current phase of
        // its stage.
        if (warp == 0 && lane == 0)
          for (uint32_t i = issued >= 2 ? issued - 2 : 0u; i < issued; i++)
            tc::mbar_wait(&eq_full[i % 2], (i / 2) & 1);
        if (tid == 0 && q.err) atomicOr(q.err, tc::kErrTimeout);
      } else {
        tc::fence_after_sync();
        for (uint32_t ct = 0; ct < nct; ct++) {
          EqTcEpilogue<64, QMF == 0 ? 2 : QMF> epi;
          epi.prepare(p, s_base, ct * q.eq_spc, tile_cols(ct), 0, q.eq_N, warp, lane);
          epi.run(p, tmem + ct * 64, warp, lane);
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TC);
}

// dynamic shared memory of the kernel (its carve-up at the top of the kernel)
static size_t zfm_smem(uint32_t K, uint32_t MM, uint32_t hi_slots, bool learned, uint32_t width) {
  const size_t tile = (size_t)MM * kKT * 2, gk = (size_t)K * (K + 1) * sizeof(float2);
  if (MM == 64) {
    // tiles, the Gn and iterate images, G, then the FP64 Gram's second half
    // or the staged network (BF16 weights, FP32 biases)
    size_t net = 0;
    if (learned && width <= kZfStageWidth) {
      const size_t nw = (size_t)width * (kZfInitFeatures + width + kZfInitCoeffs);
      net = (nw + 1) / 2 * 2 * 2 + (2 * (size_t)width + kZfInitCoeffs) * 4;
    }
    return (hi_slots + 2) * tile + 4 * (size_t)kSqImg + gk + std::max(gk, net);
  }
  return (hi_slots + 2) * tile + (size_t)MM * MM * 2 + 2 * gk + (learned ? 2 * (size_t)K * K * sizeof(float2) : 0);
}

uint64_t zf_mixed_scratch_bytes(uint32_t groups, uint32_t M, uint32_t K) {
  const TcShape s = tc_shape(M, K);
  return (uint64_t)groups * s.img_group_bytes;
}

using ZfmKernel = void (*)(const ZfmParams, const CUtensorMap);

static ZfmKernel zfm_kernel_of(uint32_t MM, uint32_t qmf, int *which) {
  switch (MM == 64 ? qmf : 0) {
    case 2: *which = 2; return zf_mixed_kernel<64, 2>;
    case 4: *which = 3; return zf_mixed_kernel<64, 4>;
    case 6: *which = 4; return zf_mixed_kernel<64, 6>;
    case 8: *which = 5; return zf_mixed_kernel<64, 8>;
    default: break;
  }
  *which = MM == 64 ? 0 : 1;
  return MM == 64 ? zf_mixed_kernel<64, 0> : zf_mixed_kernel<128, 0>;
}

// the fused equalize of zf_mixed_eq_run
struct ZfmFused {
  const EqParams *p;
  const void *y_lp;
  uint32_t S_pad, nb;
};

static mb_status zf_mixed_launch(float2 *csi, void *img_w, uint32_t groups, uint32_t M, uint32_t K,
                                 const mb_zf_opts *opts, int32_t *status, float *cond, cudaStream_t st,
                                 bool write_w, float *wmax, const ZfNetView *net, const ZfmFused *fe,
                                 uint32_t path) {
  if (path > 2) return MB_BAD_ARG;
  if (K == 0 || K > 64) return MB_UNSUPPORTED;
  const bool learned = opts && opts->init == 1;
  if (opts && opts->init > 1) return MB_BAD_ARG;
  if (learned && (!net || !net->w1 || net->width == 0 || net->width > kZfInitMaxWidth)) return MB_BAD_ARG;
  const TcShape s = tc_shape(M, K);
  const DeviceTables *tab = device_tables();
  if (!tab) return MB_CUDA_ERROR;
  ZfmParams q{};
  q.net = learned ? *net : ZfNetView{};
  q.learned = learned ? 1 : 0;
  q.csi = csi;
  q.img_w = reinterpret_cast<uint8_t *>(img_w);
  q.status = status;
  q.cond = cond;
  q.wmax = write_w ? wmax : nullptr;
  q.err = tab->err;
  q.M = M;
  q.K = K;
  q.Mp = s.Mp;
  q.nkt = s.nkt;
  q.nh = s.Mp / kKT;
  q.ns_iters = opts ? opts->ns_iters : 2;
  q.cond_thr = opts && opts->cond_threshold > 0 ? opts->cond_threshold : 1e4f;
  // bulk copies want 16-byte aligned addresses and sizes: the network's six
  // arrays (width a multiple of 4), and CSI k tiles (K even)
  auto a16 = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  q.net_bulk = 0;
  if (s.MM == 64 && learned && net->width <= kZfStageWidth && net->width % 4 == 0 && a16(net->w1) &&
      a16(net->w2) && a16(net->w3) && a16(net->b1) && a16(net->b2) && a16(net->b3))
    q.net_bulk = 1;
  // the inverse's products: tensor cores for 16 < K <= 32 unless the caller
  // picks (path 1: CUDA cores, 2: tensor cores for any K <= 32)
  q.tcns = s.MM == 64 && (path == 2 || (path == 0 && K > kTcMinK)) ? 1 : 0;
  q.csi_nst = 0;
  if (s.MM == 64 && K % 2 == 0 && a16(csi))
    q.csi_nst = std::min<uint32_t>(4, 4 * kSqImg / (kKT * K * (uint32_t)sizeof(float2)));
  // the fused equalize: K <= 32, at most 256 antennas (the whole detector
  // image, 2 Mp / 64 k tiles of 8 KB, in shared memory over the tiles),
  // whole 16-subcarrier boxes per group, at most four 128-column tiles
  uint32_t qmf = 0;
  CUtensorMap ymap;
  memset(&ymap, 0, sizeof(ymap));
  if (fe) {
    const EqParams &p = *fe->p;
    if (s.MM != 64 || q.nh > 4 || p.sg == 0 || p.sg % 16 || p.sg > 128 || fe->nb == 0 ||
        !(p.Qm == 2 || p.Qm == 4 || p.Qm == 6 || p.Qm == 8) || fe->S_pad % 8 || fe->S_pad < p.S ||
        p.M != M || p.K != K)
      return MB_UNSUPPORTED;
    const uint32_t spc_max = 128 / p.sg, ny = (fe->nb + spc_max - 1) / spc_max;
    q.eq_spc = (fe->nb + ny - 1) / ny;
    q.eq_nct = (fe->nb + q.eq_spc - 1) / q.eq_spc;
    // one 128-column tile per group: with two (or more) the CTA's two 16 KB
    // sample stages leave the loads latency-bound and the separate
    // equalizer (three CTAs of three stages per SM) is faster (measured at
    // 256x32: fused -2.4 / -3.0 / -0.4 us per slot at 2 / 4 / 8 symbols,
    // +13.5 us at 12)
    if (q.eq_nct > 1) return MB_UNSUPPORTED;
    q.eq_nb = fe->nb;
    q.eq_N = (2 * K + 15) / 16 * 16;
    q.ep = p;
    qmf = p.Qm;
    // rows [nb][re|im][M] of S_pad subcarriers; boxes of 16 x 64, 32-byte swizzle
    mb_status tr = make_tmap_2d_bf16(&ymap, fe->y_lp, fe->S_pad, (uint64_t)fe->nb * 2 * M, fe->S_pad, 16, kKT,
                                     true);
    if (tr != MB_OK) return tr;
  }
  int dev = 0, maxs = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  MB_CUDA_TRY(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  static std::atomic<uint64_t> configured[6] = {};
  static std::atomic<int> static_smem[6] = {};
  int which = 0;
  const ZfmKernel kern = zfm_kernel_of(s.MM, qmf, &which);
  const uint64_t bit = 1ull << (dev & 63);
  if (!(configured[which].load() & bit)) {
    cudaFuncAttributes fa;
    MB_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    MB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     maxs - (int)fa.sharedSizeBytes));
    static_smem[which] = (int)fa.sharedSizeBytes;
    configured[which].fetch_or(bit);
  }
  const size_t avail = (size_t)maxs - (size_t)static_smem[which].load();
  // keep every hi tile in shared memory when it fits, else stream two
  const uint32_t width = learned ? net->width : 0;
  q.resident = zfm_smem(K, s.MM, q.nh, learned, width) <= avail ? 1 : 0;
  q.write_w = write_w ? 1 : 0;
  size_t smem = zfm_smem(K, s.MM, q.resident ? q.nh : 2, learned, width);
  if (qmf) {
    // the two 16 KB sample stages behind the Gn images
    if (!q.resident) return MB_UNSUPPORTED;
    smem = std::max(smem, (size_t)(q.nh + 2) * s.MM * kKT * 2 + 2 * kSqImg + 2 * 128 * kKT * 2);
  }
  if (smem > avail) return MB_UNSUPPORTED;
  if (groups == 0) return MB_OK;
  kern<<<groups, kThreads, smem, st>>>(q, ymap);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

mb_status zf_mixed_run(float2 *csi, void *img_w, uint32_t groups, uint32_t M, uint32_t K,
                       const mb_zf_opts *opts, int32_t *status, float *cond, cudaStream_t st,
                       bool write_w, float *wmax, const ZfNetView *net, uint32_t path) {
  return zf_mixed_launch(csi, img_w, groups, M, K, opts, status, cond, st, write_w, wmax, net, nullptr, path);
}

mb_status zf_mixed_eq_run(float2 *csi, uint32_t groups, uint32_t M, uint32_t K, const mb_zf_opts *opts,
                          int32_t *status, float *cond, cudaStream_t st, bool write_w, float *wmax,
                          const ZfNetView *net, const EqParams &p, const void *y_lp, uint32_t S_pad,
                          uint32_t nb, uint32_t path) {
  const ZfmFused fe{&p, y_lp, S_pad, nb};
  return zf_mixed_launch(csi, nullptr, groups, M, K, opts, status, cond, st, write_w, wmax, net, &fe, path);
}

}  // namespace mb

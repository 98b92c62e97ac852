// zf_mixed.cu -- mixed-precision zero forcing on the tensor cores.
//
// The reference computes W = (C C^H)^{-1} C per subcarrier group with cuBLAS
// Cgemm + cuSOLVER potrf/potrs in FP32 (beamform/beamform.cu:74-122).  Here
// one CTA per group does, in one kernel:
//  1. Gram on tcgen05: with R(C) the real embedding of C (row 2u = [Re C_u,
//     -Im C_u], row 2u+1 = [Im C_u, Re C_u] over the reduction index
//     kk = plane*Mp + b), R(G) = R(C) R(C)^T.  R(C) is split into BF16
//     hi + lo parts and R(G) ~ hi hi^T + hi lo^T + lo hi^T accumulates in
//     FP32 in tensor memory: BF16 operands, FP32 accumulation, and a Gram
//     accurate to ~2^-16 (a plain BF16 Gram costs ~0.25 dB of EVM at
//     256x32, which the split removes).  The same shared-memory tile is both
//     MMA operands (A = R(C), B^T = R(C), both K-major).
//  2. FP32 Cholesky of G, explicit inverse X, 1-norm condition estimate
//     ||G||_1 ||X||_1, then ns_iters Newton-Schulz steps X <- X (2I - G X).
//  3. W = X C on tcgen05: D = R(X) R(C) gives, row for row, the detector
//     image the tensor-core equalizer consumes (eq_tc.cu); the hi image of
//     R(C) written in step 1 is re-read as the MN-major B operand.  The
//     epilogue stores that image (BF16) and W in the CSI layout (FP32).
//  4. Groups whose Gram is not positive definite in FP32, or whose condition
//     estimate exceeds cond_threshold, are redone in FP64 (Gram, Cholesky,
//     solve) and reported with status 2 (1 if even FP64 fails).
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "eq_tc.cuh"
#include "tc.cuh"
#include "zf.cuh"

namespace mb {

namespace {
constexpr int kKT = 64;        // reduction elements per k tile
constexpr int kThreads = 256;  // 8 warps; warps w and w+4 share TMEM lane quadrant w

struct ZfmParams {
  float2 *csi;       // [G][M][K]: in CSI, out W (FP32)
  uint8_t *img_w;    // [G] detector images for the equalizer (BF16)
  uint8_t *img_c;    // [G] scratch: hi image of R(C)
  int32_t *status;
  float *cond;
  int *err;
  uint32_t M, K, Mp, nkt, ns_iters;
  float cond_thr;
};

__device__ __forceinline__ uint32_t img_off(uint32_t r, uint32_t kk, uint32_t MM) {
  // canonical K-major, no swizzle: [k tile][row group][k chunk][row][8]
  const uint32_t kt = kk / kKT, kin = kk % kKT;
  return kt * (MM * kKT * 2) + (r / 8) * 1024 + (kin / 8) * 128 + (r % 8) * 16 + (kin % 8) * 2;
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
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
}  // namespace

template <int MM>
__global__ void __launch_bounds__(kThreads, 1) zf_mixed_kernel(const ZfmParams q) {
  extern __shared__ __align__(1024) uint8_t zsm[];
  __shared__ __align__(8) uint64_t tile_bar[2];
  __shared__ __align__(8) uint64_t mma_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int flag, fail;
  __shared__ float red[kThreads];

  const uint32_t g = blockIdx.x, K = q.K, M = q.M, Mp = q.Mp;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const uint32_t tile_bytes = MM * kKT * 2;
  const uint32_t TC = MM == 64 ? 128 : 256;  // TMEM columns
  const uint32_t ld = K + 1;
  // shared memory carve-up
  uint8_t *hi_t[2] = {zsm, zsm + tile_bytes};
  uint8_t *lo_t[2] = {zsm + 2 * tile_bytes, zsm + 3 * tile_bytes};
  uint8_t *ximg = zsm + 4 * tile_bytes;                        // R(X): MM x MM BF16
  float2 *Gs = reinterpret_cast<float2 *>(ximg + MM * MM * 2);  // K x ld
  float2 *Ls = Gs + K * ld;
  float2 *Xs = Ls + K * ld;
  // K x K temporary (leading dim K) in the lo tiles, free after the Gram
  float2 *Ts = reinterpret_cast<float2 *>(lo_t[0]);

  float2 *cg = q.csi + (uint64_t)g * M * K;
  uint8_t *imgc = q.img_c + (uint64_t)g * q.nkt * tile_bytes;
  uint8_t *imgw = q.img_w + (uint64_t)g * q.nkt * tile_bytes;

  if (tid == 0) {
    tc::mbar_init(&tile_bar[0], 1);
    tc::mbar_init(&tile_bar[1], 1);
    tc::mbar_init(&mma_bar, 1);
    tc::fence_mbar_init();
    fail = 0;
  }
  // rows 2K..MM-1 of the R(C) tiles are padding: zero them once
  for (uint32_t c = tid; c < 4 * tile_bytes / 16; c += kThreads)
    reinterpret_cast<uint4 *>(zsm)[c] = make_uint4(0, 0, 0, 0);
  if (warp == 0) tc::tmem_alloc(&tmem_slot, TC);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;
  uint32_t tiles_used = 0;  // double-buffer uses issued so far
  uint32_t mma_phase = 0;
  bool ok = true;

  // ---------------------------------------------------------------- Gram
  const uint32_t idesc_g = tc::idesc_bf16(MM, MM, false, false);
  for (uint32_t kt = 0; kt < q.nkt; kt++, tiles_used++) {
    const uint32_t s = tiles_used % 2, use = tiles_used / 2;
    if (use >= 1 && !tc::mbar_wait(&tile_bar[s], (use - 1) & 1)) ok = false;
    if (__syncthreads_or(!ok)) break;
    const uint32_t kk0 = kt * kKT, plane = kk0 / Mp, b0 = kk0 % Mp;
    // item (u, 8-antenna chunk): rows 2u and 2u+1, 16 bytes each, hi and lo
    for (uint32_t e = tid; e < 8 * K; e += kThreads) {
      const uint32_t u = e % K, bc = e / K;
      uint32_t h0[4], h1[4], l0[4], l1[4];
#pragma unroll
      for (int i = 0; i < 8; i += 2) {
        float v0[2], v1[2];
#pragma unroll
        for (int t = 0; t < 2; t++) {
          const uint32_t b = b0 + bc * 8 + i + t;
          const float2 c = b < M ? cg[b * K + u] : make_float2(0.f, 0.f);
          // row 2u: plane 0 -> Re, plane 1 -> -Im; row 2u+1: Im, Re
          v0[t] = plane == 0 ? c.x : -c.y;
          v1[t] = plane == 0 ? c.y : c.x;
        }
        const __nv_bfloat162 a0 = __floats2bfloat162_rn(v0[0], v0[1]);
        const __nv_bfloat162 a1 = __floats2bfloat162_rn(v1[0], v1[1]);
        const float2 f0 = __bfloat1622float2(a0), f1 = __bfloat1622float2(a1);
        const __nv_bfloat162 r0 = __floats2bfloat162_rn(v0[0] - f0.x, v0[1] - f0.y);
        const __nv_bfloat162 r1 = __floats2bfloat162_rn(v1[0] - f1.x, v1[1] - f1.y);
        h0[i / 2] = *reinterpret_cast<const uint32_t *>(&a0);
        h1[i / 2] = *reinterpret_cast<const uint32_t *>(&a1);
        l0[i / 2] = *reinterpret_cast<const uint32_t *>(&r0);
        l1[i / 2] = *reinterpret_cast<const uint32_t *>(&r1);
      }
      const uint32_t o0 = img_off(2 * u, bc * 8, MM), o1 = img_off(2 * u + 1, bc * 8, MM);
      *reinterpret_cast<uint4 *>(hi_t[s] + o0) = make_uint4(h0[0], h0[1], h0[2], h0[3]);
      *reinterpret_cast<uint4 *>(hi_t[s] + o1) = make_uint4(h1[0], h1[1], h1[2], h1[3]);
      *reinterpret_cast<uint4 *>(lo_t[s] + o0) = make_uint4(l0[0], l0[1], l0[2], l0[3]);
      *reinterpret_cast<uint4 *>(lo_t[s] + o1) = make_uint4(l1[0], l1[1], l1[2], l1[3]);
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t h0 = tc::smem_u32(hi_t[s]), l0 = tc::smem_u32(lo_t[s]);
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
    // keep the hi tile for the W product (overlaps the MMAs)
    for (uint32_t c = tid; c < tile_bytes / 16; c += kThreads)
      reinterpret_cast<uint4 *>(imgc + kt * tile_bytes)[c] = reinterpret_cast<const uint4 *>(hi_t[s])[c];
  }
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
  if (!fail) {
    const int rows_per_warp = MM == 64 ? 16 : 32;
    if (warp < 4) {
      const uint32_t r = warp * rows_per_warp + lane;
      for (uint32_t ch = 0; ch < MM / 16; ch++) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + ch * 16, v);
        if (lane < rows_per_warp && r / 2 < K) {
#pragma unroll
          for (int i = 0; i < 16; i += 2) {
            const uint32_t vcol = (ch * 16 + i) / 2;  // column 2v: Re/Im G[u][v]
            if (vcol < K) {
              if (r & 1)
                Gs[(r / 2) * ld + vcol].y = v[i];
              else
                Gs[(r / 2) * ld + vcol].x = v[i];
            }
          }
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();
    // warp 0: Cholesky G = L L^H (row-oriented, lane owns rows lane and
    // lane+32), then T = L^{-1} (lane owns columns), no block barriers
    if (warp == 0) {
      bool pd = true;
      for (uint32_t j = 0; j < K; j++) {
        if ((j & 31) == (uint32_t)lane) {
          // four partial sums break the dependent shared-memory chain
          float d0 = 0.f, d1 = 0.f, d2 = 0.f, d3 = 0.f;
          uint32_t k = 0;
          for (; k + 4 <= j; k += 4) {
            const float2 l0 = Ls[j * ld + k], l1 = Ls[j * ld + k + 1];
            const float2 l2 = Ls[j * ld + k + 2], l3 = Ls[j * ld + k + 3];
            d0 += l0.x * l0.x + l0.y * l0.y;
            d1 += l1.x * l1.x + l1.y * l1.y;
            d2 += l2.x * l2.x + l2.y * l2.y;
            d3 += l3.x * l3.x + l3.y * l3.y;
          }
          for (; k < j; k++) {
            const float2 l = Ls[j * ld + k];
            d0 += l.x * l.x + l.y * l.y;
          }
          float d = Gs[j * ld + j].x - ((d0 + d1) + (d2 + d3));
          if (!(d > 0.f)) d = -1.f;
          Ls[j * ld + j] = make_float2(d > 0.f ? sqrtf(d) : -1.f, 0.f);
        }
        __syncwarp();
        const float ljj = Ls[j * ld + j].x;
        if (!(ljj > 0.f)) {
          pd = false;
          break;
        }
        for (uint32_t i = j + 1 + lane; i < K; i += 32) {
          float2 s0 = make_float2(0.f, 0.f), s1 = make_float2(0.f, 0.f);
          uint32_t k = 0;
          for (; k + 2 <= j; k += 2) {  // L_ik conj(L_jk), two chains
            const float2 a0 = Ls[i * ld + k], b0 = Ls[j * ld + k];
            const float2 a1 = Ls[i * ld + k + 1], b1 = Ls[j * ld + k + 1];
            s0.x += a0.x * b0.x + a0.y * b0.y;
            s0.y += a0.y * b0.x - a0.x * b0.y;
            s1.x += a1.x * b1.x + a1.y * b1.y;
            s1.y += a1.y * b1.x - a1.x * b1.y;
          }
          if (k < j) {
            const float2 a0 = Ls[i * ld + k], b0 = Ls[j * ld + k];
            s0.x += a0.x * b0.x + a0.y * b0.y;
            s0.y += a0.y * b0.x - a0.x * b0.y;
          }
          const float2 gij = Gs[i * ld + j];
          Ls[i * ld + j] = make_float2((gij.x - s0.x - s1.x) / ljj, (gij.y - s0.y - s1.y) / ljj);
        }
        __syncwarp();
      }
      if (pd) {
        for (uint32_t c = lane; c < K; c += 32) {
          Ts[c * K + c] = make_float2(1.f / Ls[c * ld + c].x, 0.f);
          for (uint32_t i = c + 1; i < K; i++) {
            float2 s0 = make_float2(0.f, 0.f), s1 = make_float2(0.f, 0.f);
            uint32_t k = c;
            for (; k + 2 <= i; k += 2) {
              s0 = cadd(s0, cmulf(Ls[i * ld + k], Ts[k * K + c]));
              s1 = cadd(s1, cmulf(Ls[i * ld + k + 1], Ts[(k + 1) * K + c]));
            }
            if (k < i) s0 = cadd(s0, cmulf(Ls[i * ld + k], Ts[k * K + c]));
            const float d = Ls[i * ld + i].x;
            Ts[i * K + c] = make_float2(-(s0.x + s1.x) / d, -(s0.y + s1.y) / d);
          }
        }
      }
      if (lane == 0) flag = pd ? 0 : 1;
    }
    __syncthreads();
    const bool pd = flag == 0;
    if (pd) {
      // X = T^H T (T lower triangular)
      for (uint32_t e = tid; e < K * K; e += kThreads) {
        const uint32_t i = e / K, j = e % K;
        float2 s = make_float2(0.f, 0.f);
        for (uint32_t k = i > j ? i : j; k < K; k++)
          s = cadd(s, cmulf(cconj(Ts[k * K + i]), Ts[k * K + j]));
        Xs[i * ld + j] = s;
      }
      __syncthreads();
      // Newton-Schulz: T = 2I - G X; X = X T
      for (uint32_t it = 0; it < q.ns_iters; it++) {
        for (uint32_t e = tid; e < K * K; e += kThreads) {
          const uint32_t i = e / K, j = e % K;
          float2 s = make_float2(0.f, 0.f);
          for (uint32_t k = 0; k < K; k++) s = cadd(s, cmulf(Gs[i * ld + k], Xs[k * ld + j]));
          Ts[i * K + j] = make_float2((i == j ? 2.f : 0.f) - s.x, -s.y);
        }
        __syncthreads();
        for (uint32_t e = tid; e < K * K; e += kThreads) {
          const uint32_t i = e / K, j = e % K;
          float2 s = make_float2(0.f, 0.f);
          for (uint32_t k = 0; k < K; k++) s = cadd(s, cmulf(Xs[i * ld + k], Ts[k * K + j]));
          Ls[i * ld + j] = s;  // L is no longer needed
        }
        __syncthreads();
        for (uint32_t e = tid; e < K * K; e += kThreads) Xs[(e / K) * ld + e % K] = Ls[(e / K) * ld + e % K];
        __syncthreads();
      }
      // 1-norm condition estimate ||G||_1 ||X||_1 (both Hermitian)
      float gcol = 0.f, xcol = 0.f;
      for (uint32_t j = tid; j < K; j += kThreads) {
        float sg = 0.f, sx = 0.f;
        for (uint32_t i = 0; i < K; i++) {
          const float2 gv = Gs[i * ld + j], xv = Xs[i * ld + j];
          sg += sqrtf(gv.x * gv.x + gv.y * gv.y);
          sx += sqrtf(xv.x * xv.x + xv.y * xv.y);
        }
        gcol = fmaxf(gcol, sg);
        xcol = fmaxf(xcol, sx);
      }
      red[tid] = gcol;
      __syncthreads();
      for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (tid < o) red[tid] = fmaxf(red[tid], red[tid + o]);
        __syncthreads();
      }
      const float gn = red[0];
      __syncthreads();
      red[tid] = xcol;
      __syncthreads();
      for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (tid < o) red[tid] = fmaxf(red[tid], red[tid + o]);
        __syncthreads();
      }
      cond_est = gn * red[0];
      __syncthreads();
      if (!(cond_est <= q.cond_thr)) st = 2;
    } else {
      st = 2;
    }
  }

  // ----------------------------------------------------- W = X C (tensor)
  if (!fail && st == 0) {
    // R(X) image, K-major over the reduction index 2v + rj; rows/columns
    // beyond 2K are padding and stay zero
    for (uint32_t c = tid; c < MM * MM * 2 / 16; c += kThreads)
      reinterpret_cast<uint4 *>(ximg)[c] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    for (uint32_t e = tid; e < K * K; e += kThreads) {
      const uint32_t u = e / K, v = e % K;
      const float2 x = Xs[u * ld + v];
      *reinterpret_cast<__nv_bfloat162 *>(ximg + img_off(2 * u, 2 * v, MM)) = __floats2bfloat162_rn(x.x, -x.y);
      *reinterpret_cast<__nv_bfloat162 *>(ximg + img_off(2 * u + 1, 2 * v, MM)) = __floats2bfloat162_rn(x.y, x.x);
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    const uint32_t tiles_per_chunk = TC / kKT;
    const uint32_t idesc_w = tc::idesc_bf16(MM, kKT, false, true);
    for (uint32_t kt0 = 0; kt0 < q.nkt && ok; kt0 += tiles_per_chunk) {
      const uint32_t nt = min(tiles_per_chunk, q.nkt - kt0);
      for (uint32_t t = 0; t < nt; t++, tiles_used++) {
        const uint32_t s = tiles_used % 2, use = tiles_used / 2;
        if (use >= 1 && !tc::mbar_wait(&tile_bar[s], (use - 1) & 1)) ok = false;
        if (__syncthreads_or(!ok)) break;
        for (uint32_t c = tid; c < tile_bytes / 16; c += kThreads)
          reinterpret_cast<uint4 *>(hi_t[s])[c] =
              reinterpret_cast<const uint4 *>(imgc + (kt0 + t) * tile_bytes)[c];
        tc::fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
          tc::fence_after_sync();
          const uint32_t xa = tc::smem_u32(ximg), cb = tc::smem_u32(hi_t[s]);
#pragma unroll
          for (int ks = 0; ks < MM / 16; ks++) {
            // A = R(X): k tile ks/4, k chunk pair ks%4
            const uint64_t ad = tc::smem_desc(xa + (ks / 4) * MM * 128 + (ks % 4) * 256, 128, 1024);
            // B = hi tile read MN-major: K groups (8 rows) 1024 B apart,
            // MN chunks (8 kk) 128 B apart
            const uint64_t bd = tc::smem_desc(cb + ks * 2 * 1024, 1024, 128);
            tc::mma_f16(tmem + t * kKT, ad, bd, idesc_w, ks != 0);
          }
          tc::mma_commit(&tile_bar[s]);
        }
      }
      if (!ok) break;
      if (tid == 0) tc::mma_commit(&mma_bar);
      if (!tc::mbar_wait(&mma_bar, mma_phase & 1)) ok = false;
      mma_phase++;
      if (__syncthreads_or(!ok)) break;
      tc::fence_after_sync();
      // epilogue: warp w reads lanes of quadrant w % 4, column chunks
      // w / 4, w / 4 + 2, ...; row r, column = reduction index kk
      const int rows_per_warp = MM == 64 ? 16 : 32;
      const uint32_t quad = warp % 4;
      const uint32_t r = quad * rows_per_warp + lane;
      const uint32_t u = r / 2;
      for (uint32_t ch = warp / 4; ch < nt * kKT / 16; ch += kThreads / 128) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(quad * 32) << 16) + ch * 16, v);
        if (lane >= rows_per_warp) continue;
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const uint32_t kk = kt0 * kKT + ch * 16 + h * 8;
          uint4 pk;
          __nv_bfloat162 b01 = __floats2bfloat162_rn(v[h * 8 + 0], v[h * 8 + 1]);
          __nv_bfloat162 b23 = __floats2bfloat162_rn(v[h * 8 + 2], v[h * 8 + 3]);
          __nv_bfloat162 b45 = __floats2bfloat162_rn(v[h * 8 + 4], v[h * 8 + 5]);
          __nv_bfloat162 b67 = __floats2bfloat162_rn(v[h * 8 + 6], v[h * 8 + 7]);
          pk.x = *reinterpret_cast<uint32_t *>(&b01);
          pk.y = *reinterpret_cast<uint32_t *>(&b23);
          pk.z = *reinterpret_cast<uint32_t *>(&b45);
          pk.w = *reinterpret_cast<uint32_t *>(&b67);
          *reinterpret_cast<uint4 *>(imgw + img_off(r, kk, MM)) = pk;
          if (u < K && kk < Mp) {
#pragma unroll
            for (int e = 0; e < 8; e++) {
              const uint32_t b = kk + e;
              if (b < M) reinterpret_cast<float *>(cg + b * K + u)[r & 1] = v[h * 8 + e];
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
    D2 *Gd = reinterpret_cast<D2 *>(Gs);  // reuses Gs and Ls (2 K*ld float2)
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
        *reinterpret_cast<__nv_bfloat16 *>(imgw + img_off(2 * u, b, MM)) = __float2bfloat16_rn(w.x);
        *reinterpret_cast<__nv_bfloat16 *>(imgw + img_off(2 * u, Mp + b, MM)) = __float2bfloat16_rn(-w.y);
        *reinterpret_cast<__nv_bfloat16 *>(imgw + img_off(2 * u + 1, b, MM)) = __float2bfloat16_rn(w.y);
        *reinterpret_cast<__nv_bfloat16 *>(imgw + img_off(2 * u + 1, Mp + b, MM)) = __float2bfloat16_rn(w.x);
      }
    }
  }

  if (tid == 0) {
    if (q.status) q.status[g] = fail ? 1 : st;
    if (q.cond) q.cond[g] = cond_est;
    if (fail && q.err) atomicOr(q.err, tc::kErrTimeout);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, TC);
}

static size_t zfm_smem(uint32_t K, uint32_t MM) {
  const size_t tile = (size_t)MM * kKT * 2;
  return 4 * tile + (size_t)MM * MM * 2 + 3 * (size_t)K * (K + 1) * sizeof(float2);
}

uint64_t zf_mixed_scratch_bytes(uint32_t groups, uint32_t M, uint32_t K) {
  const TcShape s = tc_shape(M, K);
  return (uint64_t)groups * s.img_group_bytes;  // one of img_w / img_c
}

mb_status zf_mixed_run(float2 *csi, void *img_w, void *img_c, uint32_t groups, uint32_t M,
                       uint32_t K, const mb_zf_opts *opts, int32_t *status, float *cond,
                       cudaStream_t st) {
  if (K == 0 || K > 64) return MB_UNSUPPORTED;
  const TcShape s = tc_shape(M, K);
  const DeviceTables *tab = device_tables();
  if (!tab) return MB_CUDA_ERROR;
  ZfmParams q;
  q.csi = csi;
  q.img_w = reinterpret_cast<uint8_t *>(img_w);
  q.img_c = reinterpret_cast<uint8_t *>(img_c);
  q.status = status;
  q.cond = cond;
  q.err = tab->err;
  q.M = M;
  q.K = K;
  q.Mp = s.Mp;
  q.nkt = s.nkt;
  q.ns_iters = opts ? opts->ns_iters : 2;
  q.cond_thr = opts && opts->cond_threshold > 0 ? opts->cond_threshold : 1e4f;
  const size_t smem = zfm_smem(K, s.MM);
  int dev = 0, maxs = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  MB_CUDA_TRY(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  static std::atomic<uint64_t> configured[2] = {{0}, {0}};
  const int which = s.MM == 64 ? 0 : 1;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(configured[which].load() & bit)) {
    cudaFuncAttributes fa;
    if (which == 0) {
      MB_CUDA_TRY(cudaFuncGetAttributes(&fa, zf_mixed_kernel<64>));
      MB_CUDA_TRY(cudaFuncSetAttribute(zf_mixed_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       maxs - (int)fa.sharedSizeBytes));
    } else {
      MB_CUDA_TRY(cudaFuncGetAttributes(&fa, zf_mixed_kernel<128>));
      MB_CUDA_TRY(cudaFuncSetAttribute(zf_mixed_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       maxs - (int)fa.sharedSizeBytes));
    }
    configured[which].fetch_or(bit);
  }
  if (smem + 2048 > (size_t)maxs) return MB_UNSUPPORTED;
  if (groups == 0) return MB_OK;
  if (s.MM == 64)
    zf_mixed_kernel<64><<<groups, kThreads, smem, st>>>(q);
  else
    zf_mixed_kernel<128><<<groups, kThreads, smem, st>>>(q);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

}  // namespace mb

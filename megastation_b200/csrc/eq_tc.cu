// eq_tc.cu -- equalize + demodulate on the 5th-generation tensor cores.
//
// The mixed-precision replacement of the reference's SIMT equalizer
// (sgemv/equalize_kernel.cuh:27-481).  One CTA per subcarrier group g
// computes, for all nb symbols of the launch at once, the real-block GEMM
//     D (MM x N) = A_g (MM x 2*Mp) * B_g (2*Mp x N),   N = nb * sg,
// with BF16 operands and FP32 accumulation in tensor memory:
//   A_g = R(W_g^T) with rows interleaved (2u: real part of user u, 2u+1:
//         imaginary part) and reduction index kk = plane*Mp + b
//         (plane 0 multiplies Re y, plane 1 multiplies Im y); the ZF kernel
//         writes A_g into global memory already in the shared-memory image
//         of the K-major no-swizzle canonical layout, one 64-wide k tile at
//         a time, so the CTA copies it with plain 16-byte loads;
//   B_g = the planar BF16 FFT output y_lp[sym][plane][b][s], MN-major: each
//         8 x 16-byte core matrix is 8 antennas x 8 consecutive subcarriers.
// Row pairs (2u, 2u+1) land in adjacent TMEM lanes, so after tcgen05.ld one
// shuffle gives each thread the complex x of 8 subcarriers, which it demaps
// (modulation/demodulation.h:30-67 in FP16), stores as LLRs in the code-block
// layout and packs into descrambled hard-bit bytes.
//
// Pipeline: 3 shared-memory stages; all 128 threads stage tile kt while the
// tensor core works on tile kt-1; one thread issues the 4 MMAs per tile and
// commits them to the stage's mbarrier.  Every wait is bounded in time and
// reports a timeout through the device error word.
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "demod.cuh"
#include "eq_tc.cuh"
#include "sgemv.cuh"
#include "tc.cuh"

namespace mb {

namespace {
constexpr int kStages = 3;
constexpr int kKT = 64;  // reduction elements per k tile (4 MMAs of K=16)

__device__ __forceinline__ void cp16(void *dst_smem, const void *src) {
  uint4 v = __ldg(reinterpret_cast<const uint4 *>(src));
  *reinterpret_cast<uint4 *>(dst_smem) = v;
}
}  // namespace

template <int MM>
__global__ void __launch_bounds__(128, 1) equalize_tc_kernel(const EqTcParams q) {
  extern __shared__ __align__(1024) uint8_t eq_smem[];
  __shared__ __align__(8) uint64_t empty_bar[kStages];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_base_slot;
  __shared__ int timed_out;

  const EqParams &p = q.p;
  const uint32_t g = blockIdx.x;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const uint32_t N = q.N;
  const uint32_t a_tile = MM * kKT * 2;   // bytes
  const uint32_t b_tile = kKT * N * 2;    // bytes
  uint8_t *stage_base = eq_smem;

  if (tid == 0) {
    for (int s = 0; s < kStages; s++) tc::mbar_init(&empty_bar[s], 1);
    tc::mbar_init(&done_bar, 1);
    tc::fence_mbar_init();
    timed_out = 0;
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base_slot, q.tmem_cols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base_slot;

  const uint8_t *a_g = q.a_img + (uint64_t)g * q.nkt * a_tile;
  const uint32_t s_base = g * p.sg;
  const uint32_t idesc = tc::idesc_bf16(MM, N, false, true);
  const uint32_t nchunk_b = (N / 8) * (kKT / 8) * 8;  // 16-byte chunks in a B tile
  bool ok = true;

  for (uint32_t kt = 0; kt < q.nkt; kt++) {
    const uint32_t st = kt % kStages;
    uint8_t *sa = stage_base + st * (a_tile + b_tile);
    uint8_t *sb = sa + a_tile;
    if (kt >= kStages) {
      if (!tc::mbar_wait(&empty_bar[st], ((kt / kStages) - 1) & 1)) ok = false;
    }
    if (__syncthreads_or(!ok)) break;
    // A tile: contiguous image
    const uint8_t *a_src = a_g + (uint64_t)kt * a_tile;
    for (uint32_t c = tid; c < a_tile / 16; c += blockDim.x) cp16(sa + c * 16, a_src + c * 16);
    // B tile: chunk (j, kg, i) -> smem j*1024-style canonical position
    for (uint32_t c = tid; c < nchunk_b; c += blockDim.x) {
      const uint32_t i = c % 8, kg = (c / 8) % (kKT / 8), j = c / kKT;
      const uint32_t kk = kt * kKT + kg * 8 + i;
      const uint32_t plane = kk / q.Mp, b = kk % q.Mp;
      const uint32_t col0 = j * 8, l = col0 / p.sg, sl = col0 % p.sg;
      uint8_t *dst = sb + j * (kKT / 8) * 128 + kg * 128 + i * 16;
      if (b < p.M) {
        const __nv_bfloat16 *src =
            q.y_lp + ((uint64_t)(l * 2 + plane) * p.M + b) * q.S_pad + s_base + sl;
        cp16(dst, src);
      } else {
        *reinterpret_cast<uint4 *>(dst) = make_uint4(0, 0, 0, 0);
      }
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t a0 = tc::smem_u32(sa), b0 = tc::smem_u32(sb);
#pragma unroll
      for (int ks = 0; ks < kKT / 16; ks++) {
        // A: K-major, K core matrices 128 B apart, 8-row groups 1024 B apart
        const uint64_t ad = tc::smem_desc(a0 + ks * 256, 128, 1024);
        // B: MN-major, K groups 128 B apart, MN chunks (kKT/8)*128 B apart
        const uint64_t bd = tc::smem_desc(b0 + ks * 256, 128, (kKT / 8) * 128);
        tc::mma_f16(tmem, ad, bd, idesc, (kt | ks) != 0);
      }
      tc::mma_commit(&empty_bar[st]);
    }
  }
  if (tid == 0 && ok) tc::mma_commit(&done_bar);
  if (ok && !tc::mbar_wait(&done_bar, 0)) ok = false;
  if (!ok) timed_out = 1;
  __syncthreads();
  tc::fence_after_sync();

  if (!timed_out) {
    // epilogue: warp w reads TMEM lanes 32w..32w+31
    const int rows_per_warp = MM == 64 ? 16 : 32;
    const bool lane_ok = lane < rows_per_warp;
    const uint32_t r = warp * rows_per_warp + lane;  // D row of this lane
    const uint32_t u = r / 2;
    const bool is_im = r & 1;
    const bool valid = lane_ok && u < p.K;
    const uint32_t nl = N / p.sg;
    for (uint32_t ch = 0; ch < (N + 15) / 16; ch++) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + ch * 16, v);
      float w[16];
#pragma unroll
      for (int i = 0; i < 16; i++) w[i] = __shfl_xor_sync(0xffffffffu, v[i], 1);
      if (!valid) continue;
      const int half = is_im ? 1 : 0;  // even lane: columns 0-7, odd: 8-15
      const uint32_t c0 = ch * 16 + half * 8;
      if (c0 >= N) continue;  // N % 16 == 8: the last chunk is half full
      const uint32_t l = c0 / p.sg, sl0 = c0 % p.sg;
      (void)nl;
      const uint32_t s0 = s_base + sl0;
      uint64_t hbits = 0;
      int nbits = 0;
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const float re = is_im ? w[half * 8 + e] : v[half * 8 + e];
        const float im = is_im ? v[half * 8 + e] : w[half * 8 + e];
        const uint32_t s = s0 + e;
        if (s >= p.S) break;
        const float2 x = make_float2(re, im);
        __half lv[8];
        if (p.x) p.x[((uint64_t)(q.l0 + l) * p.K + u) * p.S + s] = x;
        demod(p.Qm, x, lv);
        const uint64_t t0 = (uint64_t)s * p.Qm;
        const uint64_t cb = t0 / p.cb_size;
        if (cb < p.cb_blocks) {
          const uint64_t base = cb * p.cb_stride + p.zeros + t0 % p.cb_size;
          __half *row = reinterpret_cast<__half *>(p.llr) + ((uint64_t)(q.l0 + l) * p.K + u) * p.row_len;
#pragma unroll
          for (int qq = 0; qq < 8; qq++)
            if (qq < (int)p.Qm && base + qq < p.row_len) row[base + qq] = lv[qq];
        }
        if (p.hard) {
          const __half zero = __float2half_rn(0.f);
#pragma unroll
          for (int qq = 0; qq < 8; qq++) {
            if (qq >= (int)p.Qm) break;
            const uint64_t t = t0 + qq;
            uint32_t h = 0;
            if (t < p.n_valid) {
              h = __hlt(lv[qq], zero) ? 1u : 0u;
              if (p.seq) {
                const uint64_t si = t % p.seq_len;
                h ^= (p.seq[(uint64_t)u * p.seq_stride_words + si / 32] >> (si % 32)) & 1u;
              }
            }
            hbits = (hbits << 1) | h;  // first stream bit ends up most significant
            nbits++;
          }
        }
      }
      if (p.hard && nbits) {
        // nbits = 8*Qm unless the group is cut short by S; bytes are whole
        // because sl0 % 8 == 0
        const uint64_t byte0 = (uint64_t)s0 * p.Qm / 8;
        uint8_t *hrow = p.hard + ((uint64_t)(q.l0 + l) * p.K + u) * p.hrow;
        const int nbytes = (nbits + 7) / 8;
        if (nbits % 8) hbits <<= (8 - nbits % 8);
        for (int bI = 0; bI < nbytes; bI++) {
          const uint64_t gb = byte0 + bI;
          if (gb * 8 >= p.n_valid) break;
          hrow[gb] = (uint8_t)(hbits >> (8 * (nbytes - 1 - bI)));
        }
      }
    }
  } else if (tid == 0 && q.err) {
    atomicOr(q.err, tc::kErrTimeout);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, q.tmem_cols);
}

// W [G][M][K] (fp32 complex) -> the per-group A image (see top of file)
__global__ void w_image_kernel(const float2 *W, __nv_bfloat16 *img, uint32_t M, uint32_t K,
                               uint32_t Mp, uint32_t MM, uint32_t nkt) {
  const uint32_t g = blockIdx.x;
  const uint64_t per_group = (uint64_t)nkt * MM * kKT;  // elements
  const float2 *wg = W + (uint64_t)g * M * K;
  __nv_bfloat16 *ig = img + (uint64_t)g * per_group;
  for (uint64_t e = threadIdx.x; e < per_group; e += blockDim.x) {
    // e enumerates the image in memory order: kt, row group, k chunk, row, k
    const uint32_t kin_e = e % 8, rr = (e / 8) % 8, kchunk = (e / 64) % 8;
    const uint32_t rg = (uint32_t)((e / 512) % (MM / 8)), kt = (uint32_t)(e / (512 * (MM / 8)));
    const uint32_t r = rg * 8 + rr, kk = kt * kKT + kchunk * 8 + kin_e;
    const uint32_t plane = kk / Mp, b = kk % Mp, u = r / 2, ri = r & 1;
    float v = 0.f;
    if (u < K && b < M) {
      const float2 w = wg[(uint64_t)b * K + u];
      v = ri == 0 ? (plane == 0 ? w.x : -w.y) : (plane == 0 ? w.y : w.x);
    }
    ig[e] = __float2bfloat16_rn(v);
  }
}

TcShape tc_shape(uint32_t M, uint32_t K) {
  TcShape s;
  s.MM = 2 * K <= 64 ? 64 : 128;
  s.Mp = (M + kKT - 1) / kKT * kKT;
  s.nkt = 2 * s.Mp / kKT;
  s.img_group_bytes = (uint64_t)s.nkt * s.MM * kKT * 2;
  return s;
}

mb_status w_image(const float2 *W, void *img, uint32_t G, uint32_t M, uint32_t K,
                  cudaStream_t st) {
  TcShape s = tc_shape(M, K);
  if (G == 0) return MB_OK;
  w_image_kernel<<<G, 256, 0, st>>>(W, reinterpret_cast<__nv_bfloat16 *>(img), M, K, s.Mp,
                                    s.MM, s.nkt);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

bool equalize_tc_supported(uint32_t K, uint32_t sg, uint32_t nb) {
  const uint32_t N = nb * sg;
  if (K == 0 || K > 64 || sg % 8 != 0) return false;
  const uint32_t MM = 2 * K <= 64 ? 64 : 128;
  if (N == 0 || N > 256 || N % 8 != 0) return false;  // MMA N rule for M = 64
  if (MM == 128 && N % 16 != 0) return false;          // and for M = 128
  return true;
}

mb_status equalize_tc(const EqParams &p, const void *a_img, const void *y_lp, uint32_t S_pad,
                      uint32_t l0, uint32_t nb, int *err, cudaStream_t st) {
  if (!equalize_tc_supported(p.K, p.sg, nb)) return MB_UNSUPPORTED;
  if (S_pad % 8 || S_pad < p.S) return MB_BAD_SHAPE;
  TcShape s = tc_shape(p.M, p.K);
  EqTcParams q;
  q.p = p;
  q.a_img = reinterpret_cast<const uint8_t *>(a_img);
  q.y_lp = reinterpret_cast<const __nv_bfloat16 *>(y_lp);
  q.S_pad = S_pad;
  q.Mp = s.Mp;
  q.nkt = s.nkt;
  q.N = nb * p.sg;
  q.l0 = l0;
  q.err = err;
  q.tmem_cols = 32;
  while (q.tmem_cols < q.N) q.tmem_cols *= 2;
  const size_t smem = (size_t)kStages * (s.MM * kKT * 2 + kKT * q.N * 2);
  const uint32_t G = (p.S + p.sg - 1) / p.sg;
  static std::atomic<uint64_t> configured[2] = {{0}, {0}};
  int dev = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  const int which = s.MM == 64 ? 0 : 1;
  if (!(configured[which].load() & bit)) {
    int maxs = 0;
    MB_CUDA_TRY(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    if (which == 0) {
      MB_CUDA_TRY(cudaFuncGetAttributes(&fa, equalize_tc_kernel<64>));
      MB_CUDA_TRY(cudaFuncSetAttribute(equalize_tc_kernel<64>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       maxs - (int)fa.sharedSizeBytes));
    } else {
      MB_CUDA_TRY(cudaFuncGetAttributes(&fa, equalize_tc_kernel<128>));
      MB_CUDA_TRY(cudaFuncSetAttribute(equalize_tc_kernel<128>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       maxs - (int)fa.sharedSizeBytes));
    }
    configured[which].fetch_or(bit);
  }
  if (s.MM == 64)
    equalize_tc_kernel<64><<<G, 128, smem, st>>>(q);
  else
    equalize_tc_kernel<128><<<G, 128, smem, st>>>(q);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

}  // namespace mb

namespace mb {

__global__ void y_to_lp_kernel(const float2 *y, __nv_bfloat16 *ylp, uint32_t M, uint32_t S,
                               uint32_t S_pad, uint64_t rows) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < rows * S;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t row = e / S, s = e % S;  // row = sym * M + b
    const uint64_t sym = row / M, b = row % M;
    const float2 v = y[e];
    ylp[((sym * 2 + 0) * M + b) * S_pad + s] = __float2bfloat16_rn(v.x);
    ylp[((sym * 2 + 1) * M + b) * S_pad + s] = __float2bfloat16_rn(v.y);
  }
}

mb_status y_to_lp(const float2 *y, void *y_lp, uint32_t nb, uint32_t M, uint32_t S,
                  uint32_t S_pad, cudaStream_t st) {
  const uint64_t rows = (uint64_t)nb * M;
  if (rows == 0) return MB_OK;
  const unsigned blocks = (unsigned)std::min<uint64_t>((rows * S + 255) / 256, 148 * 32);
  y_to_lp_kernel<<<blocks, 256, 0, st>>>(y, reinterpret_cast<__nv_bfloat16 *>(y_lp), M, S,
                                         S_pad, rows);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

}  // namespace mb

using namespace mb;

static uint32_t s_pad_of(uint32_t S) { return (S + 7) / 8 * 8; }

extern "C" mb_status mb_equalize_tc_scratch(uint32_t K, uint32_t M, uint32_t S, uint32_t sg,
                                            uint32_t n_sym, uint64_t *img_bytes,
                                            uint64_t *ylp_bytes) {
  if (!img_bytes || !ylp_bytes) return MB_BAD_ARG;
  if (K == 0 || K > 64 || M == 0 || S == 0 || sg == 0) return MB_BAD_SHAPE;
  const TcShape s = tc_shape(M, K);
  const uint32_t G = (S + sg - 1) / sg;
  *img_bytes = (uint64_t)G * s.img_group_bytes;
  *ylp_bytes = (uint64_t)n_sym * 2 * M * s_pad_of(S) * 2;
  return MB_OK;
}

extern "C" mb_status mb_equalize_tc(const mb_c32 *W, const mb_c32 *y, uint32_t K, uint32_t M,
                                    uint32_t S, uint32_t sg, uint32_t n_sym, uint32_t Qm,
                                    uint64_t cb_size, uint64_t cb_stride, uint64_t zeros,
                                    uint32_t cb_blocks, uint16_t *llr, uint8_t *hard,
                                    const mb_scrambler *scr, mb_c32 *x, void *scratch_img,
                                    void *scratch_ylp, void *stream) {
  EqParams p;
  mb_status s = equalize_prepare(p, W, y, K, M, S, sg, n_sym, Qm, cb_size, cb_stride, zeros,
                                 cb_blocks, llr, hard, scr);
  if (s != MB_OK) return s;
  if (!scratch_img || !scratch_ylp) return MB_BAD_ARG;
  p.x = reinterpret_cast<float2 *>(x);
  if (n_sym == 0) return MB_OK;
  uint32_t nb_max = std::max<uint32_t>(1, 256 / sg);
  while (nb_max > 1 && !equalize_tc_supported(K, sg, nb_max)) nb_max--;
  if (!equalize_tc_supported(K, sg, 1) && !equalize_tc_supported(K, sg, nb_max))
    return MB_UNSUPPORTED;
  const DeviceTables *tab = device_tables();
  if (!tab) return MB_CUDA_ERROR;
  cudaStream_t st = as_stream(stream);
  const uint32_t G = (S + sg - 1) / sg;
  const uint32_t S_pad = s_pad_of(S);
  s = w_image(reinterpret_cast<const float2 *>(W), scratch_img, G, M, K, st);
  if (s != MB_OK) return s;
  s = y_to_lp(reinterpret_cast<const float2 *>(y), scratch_ylp, n_sym, M, S, S_pad, st);
  if (s != MB_OK) return s;
  for (uint32_t l0 = 0; l0 < n_sym;) {
    uint32_t nb = std::min(nb_max, n_sym - l0);
    while (nb > 1 && !equalize_tc_supported(K, sg, nb)) nb--;
    if (!equalize_tc_supported(K, sg, nb)) return MB_UNSUPPORTED;
    const uint8_t *ylp = reinterpret_cast<const uint8_t *>(scratch_ylp) +
                         (uint64_t)l0 * 2 * M * S_pad * 2;
    s = equalize_tc(p, scratch_img, ylp, S_pad, l0, nb, tab->err, st);
    if (s != MB_OK) return s;
    l0 += nb;
  }
  return MB_OK;
}

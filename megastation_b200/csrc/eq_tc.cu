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
#include "eq_common.cuh"
#include "eq_tc.cuh"
#include "sgemv.cuh"
#include "tc.cuh"

namespace mb {

namespace {
constexpr int kStages = 4;
constexpr int kKT = 64;  // reduction elements per k tile (4 MMAs of K=16)

}  // namespace

template <int MM>
__global__ void __launch_bounds__(128, 1)
    equalize_tc_kernel(const EqTcParams q, const __grid_constant__ CUtensorMap ymap) {
  extern __shared__ __align__(1024) uint8_t eq_smem[];
  __shared__ __align__(8) uint64_t full_bar[kStages];
  __shared__ __align__(8) uint64_t empty_bar[kStages];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_base_slot;
  __shared__ int timed_out;

  const EqParams &p = q.p;
  const uint32_t g = blockIdx.x;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  // this CTA's symbols: l_off .. l_off + nbc - 1 of the launch
  const uint32_t l_off = blockIdx.y * q.spc;
  const uint32_t nbc = min(q.spc, q.nb - l_off);
  const uint32_t N = nbc * p.sg;
  const uint32_t a_tile = MM * kKT * 2;           // bytes
  const uint32_t b_tile = kKT * q.spc * p.sg * 2; // stage room: N_max/8 boxes of 8 x 64 BF16
  const uint32_t b_bytes = kKT * N * 2;           // bytes this CTA loads per tile
  const uint32_t s_base = g * p.sg;

  if (tid == 0) {
    for (int s = 0; s < kStages; s++) {
      tc::mbar_init(&full_bar[s], 1);
      tc::mbar_init(&empty_bar[s], 1);
    }
    tc::mbar_init(&done_bar, 1);
    tc::fence_mbar_init();
    timed_out = 0;
    tc::prefetch_tmap(&ymap);
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base_slot, q.tmem_cols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base_slot;

  if (warp == 0 && lane == 0) {
    // ---- producer: detector image tile by bulk copy, y_lp by tensor boxes
    const uint8_t *a_g = q.a_img + (uint64_t)g * q.nkt * a_tile;
    for (uint32_t kt = 0; kt < q.nkt; kt++) {
      const uint32_t s = kt % kStages, use = kt / kStages;
      if (use >= 1 && !tc::mbar_wait(&empty_bar[s], (use - 1) & 1)) {
        timed_out = 1;
        break;
      }
      uint8_t *sa = eq_smem + s * (a_tile + b_tile);
      uint8_t *sb = sa + a_tile;
      tc::mbar_arrive_expect_tx(&full_bar[s], a_tile + b_bytes);
      tc::bulk_g2s(sa, a_g + (uint64_t)kt * a_tile, a_tile, &full_bar[s]);
      const uint32_t kk0 = kt * kKT, plane = kk0 / q.Mp, b0 = kk0 % q.Mp;
      for (uint32_t j = 0; j < N / 8; j++) {
        const uint32_t col0 = j * 8, l = col0 / p.sg, sl = col0 % p.sg;
        const int32_t row = (int32_t)(((l_off + l) * 2 + plane) * p.M + b0);
        tc::tma_load_2d(sb + j * 1024, &ymap, (int32_t)(s_base + sl), row, &full_bar[s]);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    const uint32_t idesc = tc::idesc_bf16(MM, N, false, true);
    bool ok = true;
    for (uint32_t kt = 0; kt < q.nkt; kt++) {
      const uint32_t s = kt % kStages, use = kt / kStages;
      if (!tc::mbar_wait(&full_bar[s], use & 1)) {
        ok = false;
        break;
      }
      tc::fence_after_sync();
      const uint32_t a0 = tc::smem_u32(eq_smem + s * (a_tile + b_tile)), b0 = a0 + a_tile;
#pragma unroll
      for (int ks = 0; ks < kKT / 16; ks++) {
        // A: K-major, K core matrices 128 B apart, 8-row groups 1024 B apart
        const uint64_t ad = tc::smem_desc(a0 + ks * 256, 128, 1024);
        // B: MN-major, 8-antenna K groups 128 B apart, 8-subcarrier MN
        // chunks 1024 B apart (one tensor box each)
        const uint64_t bd = tc::smem_desc(b0 + ks * 256, 128, 1024);
        tc::mma_f16(tmem, ad, bd, idesc, (kt | ks) != 0);
      }
      tc::mma_commit(&empty_bar[s]);
    }
    if (ok) tc::mma_commit(&done_bar);
    else timed_out = 1;
  }
  __syncwarp();
  // everyone: wait for the accumulator (bounded)
  bool ok = tc::mbar_wait(&done_bar, 0);
  if (__syncthreads_or(!ok || timed_out)) {
    if (tid == 0 && q.err) atomicOr(q.err, tc::kErrTimeout);
  } else {
    tc::fence_after_sync();
    // epilogue: warp w reads TMEM lanes 32w..32w+31; rows (2u, 2u+1) are
    // adjacent lanes, exchanged with one shuffle
    const int rows_per_warp = MM == 64 ? 16 : 32;
    const bool lane_ok = lane < rows_per_warp;
    const uint32_t r = warp * rows_per_warp + lane;  // D row of this lane
    const uint32_t u = r / 2;
    const bool is_im = r & 1;
    const bool valid = lane_ok && u < p.K;
    for (uint32_t ch = 0; ch < (N + 15) / 16; ch++) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + ch * 16, v);
      float re8[8], im8[8];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        // even lane keeps columns 0-7, odd lane 8-15
        const float send = is_im ? v[i] : v[8 + i];
        const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
        re8[i] = is_im ? recv : v[i];
        im8[i] = is_im ? v[8 + i] : recv;
      }
      if (!valid) continue;
      const uint32_t c0 = ch * 16 + (is_im ? 8 : 0);
      if (c0 >= N) continue;  // N % 16 == 8: the last chunk is half full
      const uint32_t l = c0 / p.sg, sl0 = c0 % p.sg;
      const uint32_t s0 = s_base + sl0;
      const uint32_t lg = q.l0 + l_off + l;
      __half *llr_row = reinterpret_cast<__half *>(p.llr) + ((uint64_t)lg * p.K + u) * p.row_len;
      uint64_t hbits = 0;
      int nbits = 0;
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const uint32_t s = s0 + e;
        if (s >= p.S) break;
        const float2 x = make_float2(re8[e], im8[e]);
        if (p.x) p.x[((uint64_t)lg * p.K + u) * p.S + s] = x;
        hbits = (hbits << p.Qm) | eq_demap_store(p, llr_row, s, x);
        nbits += p.Qm;
      }
      if (p.hard && nbits) {
        // 8 subcarriers from s0 % 8 == 0 give whole bytes; a group cut short
        // by S pads the last byte with zeros
        const uint32_t byte0 = s0 * p.Qm / 8;
        uint8_t *hrow = p.hard + ((uint64_t)lg * p.K + u) * p.hrow;
        const int nbytes = (nbits + 7) / 8;
        if (nbits % 8) hbits <<= (8 - nbits % 8);
        for (int bI = 0; bI < nbytes; bI++) {
          const uint32_t gb = byte0 + bI;
          if (gb * 8 >= p.n_valid32) break;
          hrow[gb] = (uint8_t)(hbits >> (8 * (nbytes - 1 - bI))) ^ eq_seq_byte(p, u, gb);
        }
      }
    }
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
  // M = 128 needs N % 16: keep every per-CTA symbol chunk legal
  if (MM == 128 && sg % 16 != 0) return false;
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
  // symbols per CTA: about 32 columns, so a launch has several CTAs per
  // group and each CTA's epilogue stays short
  q.spc = std::max<uint32_t>(1, std::min<uint32_t>(nb, 32 / p.sg));
  while (q.spc > 1 && (q.spc * p.sg) % (s.MM == 64 ? 8 : 16)) q.spc--;
  q.nb = nb;
  q.N = q.spc * p.sg;
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
  // tensor map over y_lp rows [nb * 2 * M][S_pad], box 8 subcarriers x 64
  // antennas (one 1 KB group of MN-major core matrices)
  CUtensorMap ymap;
  mb_status tr = make_tmap_2d_bf16(&ymap, y_lp, S_pad, (uint64_t)nb * 2 * p.M, S_pad, 8, kKT);
  if (tr != MB_OK) return tr;
  const dim3 grid(G, (nb + q.spc - 1) / q.spc);
  if (s.MM == 64)
    equalize_tc_kernel<64><<<grid, 128, smem, st>>>(q, ymap);
  else
    equalize_tc_kernel<128><<<grid, 128, smem, st>>>(q, ymap);
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

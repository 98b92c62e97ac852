// eq_tc.cu -- equalize + demodulate on the 5th-generation tensor cores.
//
// The mixed-precision replacement of the reference's SIMT equalizer
// (sgemv/equalize_kernel.cuh:27-481).  A CTA takes one subcarrier group g
// and up to 128 / sg of the launch's symbols, and computes the real-block
// GEMM
//     D (128 x N) = Y (128 x 2*Mp) * A_g^T (2*Mp x N),   N = 2K padded to 16,
// with BF16 operands and FP32 accumulation in tensor memory:
//   Y   = the planar BF16 FFT output y_lp[sym][plane][b][s], one row per
//         (symbol, subcarrier) column of the group, reduction index
//         kk = plane*Mp + b; MN-major in shared memory (each 8 x 16-byte
//         core matrix is 8 antennas x 8 consecutive subcarriers, one tensor
//         box of 8 subcarriers x 64 antennas per 1 KB);
//   A_g = R(W_g^T) with rows interleaved (2u: real part of user u, 2u+1:
//         imaginary part); the ZF kernel writes it into global memory already
//         in the shared-memory image of the K-major no-swizzle canonical
//         layout, one 64-wide k tile at a time, so one bulk copy per tile
//         stages it.
// D row i sits in TMEM lane i: every thread of the epilogue owns one
// (symbol, subcarrier) and reads the complex x of all K users from its own
// lane, demaps each (modulation/demodulation.h:30-67 in FP16), and stores the
// LLRs, so that consecutive lanes write consecutive stretches of each user's
// LLR row.  Hard bits of 8 neighbouring subcarriers are gathered with three
// shuffles into whole descrambled bytes.
//
// Pipeline: kStages shared-memory stages fed by one producer thread (bulk
// copy + tensor boxes); one thread issues the 4 MMAs per tile and commits
// them to the stage's mbarrier.  Every wait is bounded in time and reports a
// timeout through the device error word.
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "eq_common.cuh"
#include "eq_tc.cuh"
#include "eq_tc_epi.cuh"
#include "sgemv.cuh"
#include "tc.cuh"

namespace mb {

namespace {
constexpr int kStages = 3;
constexpr int kKT = 64;     // reduction elements per k tile (4 MMAs of K=16)
constexpr int kCols = 128;  // MMA M: (symbol, subcarrier) columns per CTA
constexpr int kEqThreads = 256;  // 8 warps: warps w and w + 4 read TMEM lane quadrant w
}  // namespace

template <int MM, int QM>
__global__ void __launch_bounds__(kEqThreads, 1)
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
  const uint32_t ncols = nbc * p.sg;                 // valid columns, <= 128
  constexpr uint32_t y_tile = kCols * kKT * 2;       // 16 KB: 128 columns x 64 kk
  constexpr uint32_t a_tile = MM * kKT * 2;          // detector image k tile
  constexpr uint32_t stage_bytes = y_tile + a_tile;
  const uint32_t y_bytes = ncols * kKT * 2;          // bytes this CTA loads per tile
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
    // ---- producer: y columns by tensor boxes, detector image by bulk copy
    const uint8_t *a_g = q.a_img + (uint64_t)g * q.nkt * a_tile;
    for (uint32_t kt = 0; kt < q.nkt; kt++) {
      const uint32_t s = kt % kStages, use = kt / kStages;
      if (use >= 1 && !tc::mbar_wait(&empty_bar[s], (use - 1) & 1)) {
        timed_out = 1;
        break;
      }
      uint8_t *sy = eq_smem + s * stage_bytes;
      uint8_t *sa = sy + y_tile;
      tc::mbar_arrive_expect_tx(&full_bar[s], y_bytes + a_tile);
      tc::bulk_g2s(sa, a_g + (uint64_t)kt * a_tile, a_tile, &full_bar[s]);
      const uint32_t kk0 = kt * kKT, plane = kk0 / q.Mp, b0 = kk0 % q.Mp;
      // boxes of 16 (swizzled, 2 KB) or 8 (1 KB) columns by the 64 k rows
      const uint32_t bw = q.y16 ? 16 : 8;
      for (uint32_t j = 0; j < ncols / bw; j++) {
        const uint32_t col0 = j * bw, l = col0 / p.sg, sl = col0 % p.sg;
        const int32_t row = (int32_t)(((l_off + l) * 2 + plane) * p.M + b0);
        tc::tma_load_2d(sy + j * bw * 128, &ymap, (int32_t)(s_base + sl), row, &full_bar[s]);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer.  Columns ncols..127 of the y stage are never loaded:
    // their D rows are garbage and no thread stores them.
    const uint32_t idesc = tc::idesc_bf16(kCols, q.N, true, false);
    bool ok = true;
    for (uint32_t kt = 0; kt < q.nkt; kt++) {
      const uint32_t s = kt % kStages, use = kt / kStages;
      if (!tc::mbar_wait(&full_bar[s], use & 1)) {
        ok = false;
        break;
      }
      tc::fence_after_sync();
      const uint32_t y0 = tc::smem_u32(eq_smem + s * stage_bytes), a0 = y0 + y_tile;
#pragma unroll
      for (int ks = 0; ks < kKT / 16; ks++) {
        // Y: MN-major.  8-column boxes: 8-antenna K groups 128 B apart,
        // 8-subcarrier MN chunks 1024 B apart (one box each); 16-column
        // swizzled boxes: 32-byte atoms of 16 columns 2048 B apart (one box
        // each), 8-antenna K groups 256 B apart
        const uint64_t yd = q.y16 ? tc::smem_desc_mn_sw32(y0 + ks * 512, 2048, 256)
                                  : tc::smem_desc(y0 + ks * 256, 128, 1024);
        // image: K-major, K core matrices 128 B apart, 8-row groups 1024 B apart
        const uint64_t ad = tc::smem_desc(a0 + ks * 256, 128, 1024);
        tc::mma_f16(tmem, yd, ad, idesc, (kt | ks) != 0);
      }
      tc::mma_commit(&empty_bar[s]);
    }
    if (ok) tc::mma_commit(&done_bar);
    else timed_out = 1;
  }
  __syncwarp();
  // the epilogue's per-thread setup overlaps the load/MMA phase
  EqTcEpilogue<MM, QM> epi;
  epi.prepare(p, s_base, l_off, ncols, q.l0, q.N, warp, lane);
  // everyone: wait for the accumulator (bounded)
  bool ok = tc::mbar_wait(&done_bar, 0);
  if (__syncthreads_or(!ok || timed_out)) {
    if (tid == 0 && q.err) atomicOr(q.err, tc::kErrTimeout);
  } else {
    tc::fence_after_sync();
    epi.run(p, tmem, warp, lane);
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

using EqTcKernel = void (*)(const EqTcParams, const CUtensorMap);

template <int MM>
static EqTcKernel eq_tc_kernel_of(uint32_t Qm) {
  switch (Qm) {
    case 2: return equalize_tc_kernel<MM, 2>;
    case 4: return equalize_tc_kernel<MM, 4>;
    case 6: return equalize_tc_kernel<MM, 6>;
    default: return equalize_tc_kernel<MM, 8>;
  }
}

// raises the dynamic shared memory limit of the (MM, Qm) kernel once per device
static mb_status equalize_tc_configure(uint32_t MM, uint32_t Qm, int dev) {
  static std::atomic<uint64_t> configured[8] = {};
  const int which = (MM == 64 ? 0 : 4) + (Qm == 2 ? 0 : Qm == 4 ? 1 : Qm == 6 ? 2 : 3);
  const uint64_t bit = 1ull << (dev & 63);
  if (configured[which].load() & bit) return MB_OK;
  int maxs = 0;
  MB_CUDA_TRY(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const EqTcKernel k = MM == 64 ? eq_tc_kernel_of<64>(Qm) : eq_tc_kernel_of<128>(Qm);
  cudaFuncAttributes fa;
  MB_CUDA_TRY(cudaFuncGetAttributes(&fa, k));
  MB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   maxs - (int)fa.sharedSizeBytes));
  configured[which].fetch_or(bit);
  return MB_OK;
}

bool equalize_tc_supported(uint32_t K, uint32_t sg, uint32_t nb) {
  // a CTA holds whole symbols of one group in its 128 columns; the MMA's N
  // is 2K rounded up to 16 (at most the image's MM rows)
  if (K == 0 || K > 64 || sg == 0 || sg % 8 != 0 || sg > (uint32_t)kCols) return false;
  return nb >= 1;
}

mb_status equalize_tc(const EqParams &p, const void *a_img, const void *y_lp, uint32_t S_pad,
                      uint32_t l0, uint32_t nb, int *err, cudaStream_t st, uint32_t max_cols) {
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
  // symbols per CTA: as many as fill max_cols (<= 128) columns, spread
  // evenly over the CTAs a group needs
  const uint32_t cols = max_cols ? std::min<uint32_t>(max_cols, kCols) : kCols;
  const uint32_t spc_max = std::max<uint32_t>(1, cols / p.sg);
  const uint32_t ny = (nb + spc_max - 1) / spc_max;
  q.spc = (nb + ny - 1) / ny;
  q.nb = nb;
  q.N = (2 * p.K + 15) / 16 * 16;
  q.l0 = l0;
  q.err = err;
  q.tmem_cols = 32;
  while (q.tmem_cols < q.N) q.tmem_cols *= 2;
  const size_t smem = (size_t)kStages * ((size_t)kCols * kKT * 2 + (size_t)s.MM * kKT * 2);
  const uint32_t G = (p.S + p.sg - 1) / p.sg;
  int dev = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  mb_status cs = equalize_tc_configure(s.MM, p.Qm, dev);
  if (cs != MB_OK) return cs;
  // tensor map over y_lp rows [nb * 2 * M][S_pad], box 16 subcarriers x 64
  // antennas with the 32-byte swizzle (one 2 KB MN-major SW32 atom column:
  // whole 32-byte sectors per antenna row) when groups are whole boxes, else
  // 8 subcarriers x 64 antennas (one 1 KB group of MN-major core matrices)
  q.y16 = p.sg % 16 == 0 ? 1 : 0;
  CUtensorMap ymap;
  mb_status tr = make_tmap_2d_bf16(&ymap, y_lp, S_pad, (uint64_t)nb * 2 * p.M, S_pad, q.y16 ? 16 : 8, kKT,
                                   q.y16 != 0);
  if (tr != MB_OK) return tr;
  const dim3 grid(G, ny);
  (s.MM == 64 ? eq_tc_kernel_of<64>(p.Qm) : eq_tc_kernel_of<128>(p.Qm))<<<grid, kEqThreads, smem, st>>>(q, ymap);
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

// precode_tc.cu -- downlink ZF precoding on the 5th-generation tensor cores.
//
// The mixed-precision replacement of the reference's SIMT precoder
// (sgemv/precode.cu:18-68, precode_kernel.cuh:255-262):
//     z[sym][b][(s + start + N/2) mod N] = sum_u P[g(s)][u][b] s_u[sym][s].
// A CTA takes one subcarrier group g, one half of up to 128 antennas and the
// (symbol, subcarrier) columns of up to 128 / sg symbols, and computes the
// real-block GEMM
//     D (128 x 256) = A (128 x 2Kp) * B_g^T (2Kp x 256)
// with BF16 operands and FP32 accumulation in tensor memory:
//   A   = the user symbols of the CTA's columns, row c = (symbol, subcarrier),
//         reduction index kk = plane*Kp + u (plane 0: Re s_u, 1: Im s_u),
//         built by the threads in the K-major canonical layout;
//   B_g = the real embedding of P_g^T, row n = 2 b + ri (ri 0: Re z_b,
//         1: Im z_b) of the half's 128 antennas, so that each TMEM lane
//         holds (Re z_b, Im z_b) pairs; precoder_image_kernel writes it to
//         global memory already in its shared-memory image (K-major
//         canonical, 64-wide k tiles), staged by one bulk copy per tile.
// Every thread of the epilogue owns one column and stores the FP16 complex
// z of its antennas, consecutive lanes writing consecutive bins of a row.
// The guard bins of z are never written: the caller zeroes them once.
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "precode_tc.cuh"
#include "tc.cuh"

namespace mb {
namespace {

constexpr int kKT = 64;          // reduction elements per k tile
constexpr int kCols = 128;       // MMA M: columns per CTA
constexpr int kAnt = 128;        // antennas per CTA: MMA N = 256
constexpr int kPcThreads = 256;  // warps w and w + 4 read TMEM lane quadrant w
constexpr uint32_t kBTile = 2 * kAnt * kKT * 2;  // 32 KB: 256 rows x 64 kk
constexpr uint32_t kATile = kCols * kKT * 2;     // 16 KB: 128 rows x 64 kk

__host__ __device__ constexpr uint32_t kmaj(uint32_t row, uint32_t kk, uint32_t tile_bytes) {
  // [k tile][row group][k chunk][row][8]: 8-row groups 1024 B apart, k
  // chunks of 8 elements 128 B apart
  return (kk / kKT) * tile_bytes + (row / 8) * 1024 + ((kk % kKT) / 8) * 128 + (row % 8) * 16 + (kk % 8) * 2;
}

struct PcParams {
  const uint8_t *img;   // [G][H][nkt] B tiles
  const float2 *sym;    // [D][K][S]
  __half2 *z;           // [D][M][N] FP16 (re, im)
  uint32_t M, K, Kp, S, sg, N, c, D, H, nkt, spc;
  int *err;
};

__global__ void __launch_bounds__(kPcThreads, 1) precode_tc_kernel(const PcParams q) {
  extern __shared__ __align__(1024) uint8_t pc_smem[];
  __shared__ __align__(8) uint64_t img_bar, done_bar;
  __shared__ uint32_t tmem_slot;
  const uint32_t g = blockIdx.x, h = blockIdx.y;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const uint32_t l_off = blockIdx.z * q.spc, nbc = min(q.spc, q.D - l_off);
  const uint32_t ncols = nbc * q.sg;  // <= 128
  uint8_t *sB = pc_smem, *sA = pc_smem + q.nkt * kBTile;
  if (tid == 0) {
    tc::mbar_init(&img_bar, 1);
    tc::mbar_init(&done_bar, 1);
    tc::fence_mbar_init();
    tc::mbar_arrive_expect_tx(&img_bar, q.nkt * kBTile);
    const uint8_t *src = q.img + ((uint64_t)g * q.H + h) * q.nkt * kBTile;
    for (uint32_t kt = 0; kt < q.nkt; kt++) tc::bulk_g2s(sB + kt * kBTile, src + (uint64_t)kt * kBTile, kBTile, &img_bar);
  }
  if (warp == 0) tc::tmem_alloc(&tmem_slot, 256);
  // A: work item -> (column cc, 8 users u0..u0+7): eight loads of s_u at the
  // column's (symbol, subcarrier) (consecutive threads: consecutive columns,
  // so consecutive subcarriers), then one 16-byte store of the BF16 real
  // parts (plane 0) and one of the imaginary parts (plane 1); columns beyond
  // ncols and users beyond K are zero
  const uint32_t s0 = g * q.sg;
  {
    const uint32_t cc = tid % kCols;
    const uint32_t l = cc / q.sg, s = s0 + cc % q.sg;
    const bool col_ok = cc < ncols && s < q.S;
    const float2 *src = q.sym + (uint64_t)(l_off + l) * q.K * q.S + s;
    for (uint32_t u0 = (tid / kCols) * 8; u0 < q.Kp; u0 += (kPcThreads / kCols) * 8) {
      float2 v[8];
#pragma unroll
      for (int j = 0; j < 8; j++)
        v[j] = col_ok && u0 + j < q.K ? __ldg(src + (uint64_t)(u0 + j) * q.S) : make_float2(0.f, 0.f);
      uint32_t re[4], im[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const __nv_bfloat162 a = __floats2bfloat162_rn(v[2 * j].x, v[2 * j + 1].x);
        const __nv_bfloat162 b = __floats2bfloat162_rn(v[2 * j].y, v[2 * j + 1].y);
        re[j] = *reinterpret_cast<const uint32_t *>(&a);
        im[j] = *reinterpret_cast<const uint32_t *>(&b);
      }
      *reinterpret_cast<uint4 *>(sA + kmaj(cc, u0, kATile)) = make_uint4(re[0], re[1], re[2], re[3]);
      *reinterpret_cast<uint4 *>(sA + kmaj(cc, q.Kp + u0, kATile)) = make_uint4(im[0], im[1], im[2], im[3]);
    }
  }
  tc::fence_proxy_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;
  bool ok = true;
  if (tid == 0) {
    ok = tc::mbar_wait(&img_bar, 0);
    if (ok) {
      tc::fence_after_sync();
      const uint32_t idesc = tc::idesc_bf16(kCols, 2 * kAnt, false, false);
      const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
      for (uint32_t kt = 0; kt < q.nkt; kt++)
#pragma unroll
        for (int ks = 0; ks < kKT / 16; ks++) {
          const uint64_t ad = tc::smem_desc(a0 + kt * kATile + ks * 256, 128, 1024);
          const uint64_t bd = tc::smem_desc(b0 + kt * kBTile + ks * 256, 128, 1024);
          tc::mma_f16(tmem, ad, bd, idesc, (kt | (uint32_t)ks) != 0);
        }
      tc::mma_commit(&done_bar);
    }
  }
  // the column this thread stores, and its bin
  const uint32_t quad = warp % 4, cc = quad * 32 + lane;
  const uint32_t l = cc / q.sg, s = s0 + cc % q.sg;
  const bool valid = cc < ncols && s < q.S;
  const uint32_t bin = (s + q.c) % q.N;
  const bool loaded = __syncthreads_and(ok);
  ok = loaded && tc::mbar_wait(&done_bar, 0);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      if (q.err) atomicOr(q.err, tc::kErrTimeout);
      // the image copies may still be landing: give them a bounded wait
      if (!loaded) tc::mbar_wait(&img_bar, 0, 100000000ull);
    }
  } else {
    tc::fence_after_sync();
    __half2 *zc = q.z + ((uint64_t)(l_off + l) * q.M + h * kAnt) * q.N + bin;
    const uint32_t nb = min((uint32_t)kAnt, q.M - h * kAnt);  // antennas of this half
    // chunk ch: TMEM columns 16 ch .. 16 ch + 15 = antennas 8 ch .. 8 ch + 7
#pragma unroll 1
    for (uint32_t ch = warp / 4; ch < 2 * kAnt / 16; ch += kPcThreads / 128) {
      if (ch * 8 >= nb) break;  // warp-uniform
      float v[16];
      tc::tmem_ld16(tmem + ((quad * 32) << 16) + ch * 16, v);
      if (valid) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const uint32_t b = ch * 8 + j;
          if (b < nb) zc[(uint64_t)b * q.N] = __floats2half2_rn(v[2 * j], v[2 * j + 1]);
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

// P [G][K][M] (the scaled precoder) -> the per-(group, half) B tiles.  A
// work item is one antenna b and 8 users u0..u0+7: eight loads of P[u][b]
// (consecutive threads: consecutive antennas, coalesced), then the four
// 16-byte chunks of rows 2b (Re z) and 2b+1 (Im z) in planes 0 and 1.
__global__ void precoder_image_kernel(const float2 *P, __nv_bfloat16 *img, uint32_t M, uint32_t K,
                                      uint32_t Kp, uint32_t H, uint32_t nkt) {
  const uint32_t g = blockIdx.x, h = blockIdx.y;
  uint8_t *out = reinterpret_cast<uint8_t *>(img) + ((uint64_t)g * H + h) * nkt * kBTile;
  const float2 *Pg = P + (uint64_t)g * K * M;
  const uint32_t items = kAnt * (Kp / 8);
  for (uint32_t e = threadIdx.x; e < items; e += blockDim.x) {
    const uint32_t bl = e % kAnt, u0 = (e / kAnt) * 8, b = h * kAnt + bl;
    float2 p[8];
#pragma unroll
    for (int j = 0; j < 8; j++)
      p[j] = b < M && u0 + j < K ? __ldg(Pg + (uint64_t)(u0 + j) * M + b) : make_float2(0.f, 0.f);
    // Re z = Re P Re s - Im P Im s; Im z = Im P Re s + Re P Im s
    uint32_t w[4][4];  // [ri * 2 + plane][pair]
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const float2 a = p[2 * j], c = p[2 * j + 1];
      const __nv_bfloat162 r0 = __floats2bfloat162_rn(a.x, c.x), r1 = __floats2bfloat162_rn(-a.y, -c.y);
      const __nv_bfloat162 i0 = __floats2bfloat162_rn(a.y, c.y), i1 = __floats2bfloat162_rn(a.x, c.x);
      w[0][j] = *reinterpret_cast<const uint32_t *>(&r0);
      w[1][j] = *reinterpret_cast<const uint32_t *>(&r1);
      w[2][j] = *reinterpret_cast<const uint32_t *>(&i0);
      w[3][j] = *reinterpret_cast<const uint32_t *>(&i1);
    }
#pragma unroll
    for (int ri = 0; ri < 2; ri++)
#pragma unroll
      for (int pl = 0; pl < 2; pl++) {
        const uint32_t *v = w[ri * 2 + pl];
        *reinterpret_cast<uint4 *>(out + kmaj(2 * bl + ri, pl * Kp + u0, kBTile)) = make_uint4(v[0], v[1], v[2], v[3]);
      }
  }
}

}  // namespace

PcShape precode_tc_shape(uint32_t M, uint32_t K) {
  PcShape s;
  s.Kp = (K + 31) / 32 * 32;
  s.H = (M + kAnt - 1) / kAnt;
  s.nkt = 2 * s.Kp / kKT;
  s.img_group_bytes = (uint64_t)s.H * s.nkt * kBTile;
  return s;
}

bool precode_tc_supported(uint32_t K, uint32_t sg) {
  return K >= 1 && K <= 64 && sg >= 1 && sg <= (uint32_t)kCols;
}

mb_status precoder_image(const float2 *P, void *img, uint32_t G, uint32_t M, uint32_t K, cudaStream_t st) {
  if (!precode_tc_supported(K, 1)) return MB_UNSUPPORTED;
  if (G == 0) return MB_OK;
  const PcShape s = precode_tc_shape(M, K);
  precoder_image_kernel<<<dim3(G, s.H), 256, 0, st>>>(P, reinterpret_cast<__nv_bfloat16 *>(img), M, K, s.Kp, s.H,
                                                     s.nkt);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

mb_status precode_tc(const void *img, const float2 *sym, void *z, uint32_t M, uint32_t K, uint32_t S, uint32_t sg,
                     uint32_t N, uint32_t start, uint32_t D, int *err, cudaStream_t st) {
  if (!precode_tc_supported(K, sg)) return MB_UNSUPPORTED;
  if (S > N || M == 0) return MB_BAD_SHAPE;
  if (D == 0 || S == 0) return MB_OK;
  const PcShape s = precode_tc_shape(M, K);
  PcParams q;
  q.img = reinterpret_cast<const uint8_t *>(img);
  q.sym = sym;
  q.z = reinterpret_cast<__half2 *>(z);
  q.M = M;
  q.K = K;
  q.Kp = s.Kp;
  q.S = S;
  q.sg = sg;
  q.N = N;
  q.c = (start + N / 2) % N;
  q.D = D;
  q.H = s.H;
  q.nkt = s.nkt;
  // symbols per CTA: as many as fill the 128 columns, spread evenly
  const uint32_t spc_max = std::max<uint32_t>(1, kCols / sg);
  const uint32_t nz = (D + spc_max - 1) / spc_max;
  q.spc = (D + nz - 1) / nz;
  q.err = err;
  const size_t smem = (size_t)s.nkt * kBTile + (size_t)s.nkt * kATile;
  int dev = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  static std::atomic<uint64_t> configured{0};
  const uint64_t bit = 1ull << (dev & 63);
  if (!(configured.load() & bit)) {
    // up to 2 k tiles of B (64 KB) and A (32 KB)
    MB_CUDA_TRY(cudaFuncSetAttribute(precode_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     2 * (int)(kBTile + kATile)));
    configured.fetch_or(bit);
  }
  const uint32_t G = (S + sg - 1) / sg;
  precode_tc_kernel<<<dim3(G, s.H, nz), kPcThreads, smem, st>>>(q);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

}  // namespace mb

using namespace mb;

extern "C" mb_status mb_precode_tc_scratch(uint32_t M, uint32_t K, uint32_t S, uint32_t sg, uint64_t *img_bytes) {
  if (!img_bytes) return MB_BAD_ARG;
  if (M == 0 || S == 0 || sg == 0) return MB_BAD_SHAPE;
  if (!precode_tc_supported(K, sg)) return MB_UNSUPPORTED;
  *img_bytes = (uint64_t)((S + sg - 1) / sg) * precode_tc_shape(M, K).img_group_bytes;
  return MB_OK;
}

extern "C" mb_status mb_precode_tc(const mb_c32 *P, const mb_c32 *s, uint32_t M, uint32_t K, uint32_t S,
                                   uint32_t sg, uint32_t N, uint32_t start, uint32_t n_sym, void *z,
                                   void *scratch_img, void *stream) {
  if (!P || !s || !z || !scratch_img) return MB_BAD_ARG;
  if (M == 0 || K == 0 || S == 0 || sg == 0 || N < S) return MB_BAD_SHAPE;
  if (!precode_tc_supported(K, sg)) return MB_UNSUPPORTED;
  if ((reinterpret_cast<uintptr_t>(scratch_img) & 15) != 0) return MB_BAD_ARG;
  const DeviceTables *tab = device_tables();
  if (!tab) return MB_CUDA_ERROR;
  cudaStream_t st = as_stream(stream);
  const uint32_t G = (S + sg - 1) / sg;
  mb_status r = precoder_image(reinterpret_cast<const float2 *>(P), scratch_img, G, M, K, st);
  if (r != MB_OK) return r;
  return precode_tc(scratch_img, reinterpret_cast<const float2 *>(s), z, M, K, S, sg, N, start, n_sym, tab->err,
                    st);
}

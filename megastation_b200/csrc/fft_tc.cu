// fft_tc.cu -- 4096-point OFDM FFT with its butterflies on the tensor cores.
//
// Replaces the reference's uplink FFT pipeline for N = 4096 (load kernel ->
// cuFFT C2C -> FFT-shift gather, fft/fft_op.cu:135-143 with
// fft_callback.cuh:20-74) in the mixed-precision slot, where the output goes
// to the tensor-core equalizer as planar BF16 rows.  Cooley-Tukey 64 x 64
// with n = 64 n1 + n2 and bin k = k1 + 64 k2:
//
//   Y[k1][n2]      = sum_n1 x[64 n1 + n2] W64^(n1 k1)     GEMM 1
//   Z[k1][n2]      = Y[k1][n2] W4096^(n2 k1)               CUDA cores
//   X[k1 + 64 k2]  = sum_n2 Z[k1][n2] W64^(n2 k2)          GEMM 2
//
// and bin k is stored as subcarrier (k - start - N/2) mod N when that is
// below S (fft_callback.cuh:43-74).  The complex GEMMs run as real ones on
// the [re; im] embedding (K = 128) with FP16 operands and FP32 accumulation
// in TMEM (tcgen05.mma kind::f16); both multiply by the same 128 x 128 DFT
// operand F.  Each row is scaled by a power of two so that its largest
// component lies in [128, 256): then |Y| and |Z| stay below 2^15.5, inside
// the FP16 range, and the scale is undone exactly before the BF16 store.
//
// One CTA per SM takes every gridDim-th unit of two rows, with 224 KB of
// shared memory (F, one GEMM operand buffer, an output staging buffer and a
// two-unit input ring) and 256 TMEM columns (the two GEMM accumulators).
// Warp 8 is the control warp: one thread streams the units' rows into the
// ring with 128-byte-swizzled TMA boxes (so the conversion reads are free of
// bank conflicts), issues both GEMMs and writes the staged output rows back
// with bulk copies.  Warps 0-7 convert the samples into the GEMM-1 operand,
// twiddle the GEMM-1 result into the GEMM-2 operand (in the same buffer,
// which GEMM 1 no longer needs) and stage the GEMM-2 result as BF16 rows.
// Mbarriers hand each buffer between the roles, so a unit's loads, GEMMs,
// conversion and stores overlap those of its neighbours.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "fft.cuh"
#include "tc.cuh"

namespace mb {

struct FftTcPlan {
  uint8_t *mats;  // F, 128 x 128 FP16 in its shared-memory layout
  float2 *tw;     // W4096^j, j < 4096
  uint32_t c;     // (start + N/2) mod N
};

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kFtCompute = 512;                  // warps 0-15
constexpr int kFtThreads = kFtCompute + 64;      // + the GEMM and copy warps
constexpr uint32_t kFtN = 4096;
constexpr uint32_t kMat = 32768;                 // one 128 x 128 FP16 operand
constexpr uint32_t kStage = 65536;               // raw samples of one unit (c64)
// staged output rows (r, plane) at (2 r + plane) * kStgPitch: 8192 B plus 64,
// so the two planes of a row start on opposite halves of the 32 banks
constexpr uint32_t kStgPitch = 8192 + 64;
constexpr uint32_t kFtSmem = 2 * kMat + 2 * kStage + 4 * kStgPitch;  // F, AZ, ring, staging

// byte offset of element (row, kk) of a 128 x 128 K-major operand: 8-row
// groups 2048 B apart, K core matrices (8 elements, 16 B) 128 B apart
__host__ __device__ constexpr uint32_t kmaj_off(uint32_t row, uint32_t kk) {
  return (row / 8) * 2048 + (kk / 8) * 128 + (row % 8) * 16 + (kk % 8) * 2;
}
// byte offset of element (mn, kk) of a 128 x 128 MN-major operand: 8-row K
// groups 2048 B apart, 8-element MN chunks 128 B apart
__host__ __device__ constexpr uint32_t mnmaj_off(uint32_t mn, uint32_t kk) {
  return (kk / 8) * 2048 + (mn / 8) * 128 + (kk % 8) * 16 + (mn % 8) * 2;
}

struct FtParams {
  uint32_t rows;        // rows of 4096 samples, [symbol][M]
  uint32_t pilot_rows;  // the first pilot_rows are comb-pilot rows (CSI out),
                        // the others uplink rows (planar BF16 out)
  uint32_t M, S, S_pad;
  __nv_bfloat16 *out;   // uplink: [n_sym][re|im][M][S_pad], row (row - pilot_rows)
  float2 *csi;          // pilot: [G][M][K]
  const float2 *pilot;  // pilot: sign of each subcarrier
  uint32_t K, sg, ue_start, tail_rem, G;
  uint32_t sg_magic;    // floor(i / sg) = umulhi(i, sg_magic) for i < 2^13
  const uint8_t *mats;
  const float2 *tw;
  uint32_t c;
  uint32_t units;       // ceil(rows / 2)
  uint32_t upc;         // units per CTA
  int *err;
  // inverse mode (DownlinkIFFT): every row is one [N] spectrum in bin
  // order; the unnormalised inverse FFT is conj(FFT(conj(z))), so the
  // conversion negates the imaginary parts, the GEMMs and twiddles are the
  // forward ones, and the store negates them back, scales by out_scale / N
  // and writes all N samples interleaved (int16 / int8 quantised as
  // ifft_callback.cuh:37-52, or FP16)
  uint32_t inverse;
  int out_dtype;
  float out_scale;      // (max + 1) / N for integer outputs, 1 / N for FP16
  void *tout;           // [rows][N] pairs of out_dtype
};

template <int DT>
struct Fmt {
  static constexpr uint32_t kBytes = DT == MB_IQ_C32 ? 8 : DT == MB_IQ_I8 ? 2 : 4;  // per sample
  static constexpr uint32_t kBoxes = kBytes / 2;      // 128-byte boxes per 64-sample n1 row
  static constexpr uint32_t kPPC = kBytes / 2;        // 16-byte pieces per 8-sample chunk
  static constexpr uint32_t kUnitBytes = 2 * kFtN * kBytes;
};

// integer samples have a known range: a fixed scale instead of the row maximum
template <int DT>
constexpr bool kFixedScale = DT == MB_IQ_I16 || DT == MB_IQ_I8;

// ring offset of the 16-byte piece holding sample n2 (first of its piece)
// of n1 row n1 of unit row r: box (r, n2 / (128 / bytes)) of 64 n1 rows x
// 128 B, swizzled by the TMA
template <int DT>
__device__ __forceinline__ uint32_t ring_off(uint32_t r, uint32_t n1, uint32_t n2) {
  using F = Fmt<DT>;
  const uint32_t byte = n2 * F::kBytes;
  const uint32_t box = r * F::kBoxes + byte / 128;
  return box * 8192 + n1 * 128 + ((((byte % 128) / 16) ^ (n1 & 7)) * 16);
}

template <int DT>
__device__ __forceinline__ float2 chunk_sample(const uint4 *raw, int j) {
  if constexpr (DT == MB_IQ_C32) {
    const uint4 w = raw[j / 2];
    return (j & 1) ? make_float2(__uint_as_float(w.z), __uint_as_float(w.w))
                   : make_float2(__uint_as_float(w.x), __uint_as_float(w.y));
  } else if constexpr (DT == MB_IQ_I16) {
    const uint4 w = raw[j / 4];
    const uint32_t v = (j & 3) == 0 ? w.x : (j & 3) == 1 ? w.y : (j & 3) == 2 ? w.z : w.w;
    return make_float2((float)(int16_t)(v & 0xFFFFu) / 32768.f, (float)(int16_t)(v >> 16) / 32768.f);
  } else if constexpr (DT == MB_IQ_I8) {
    const uint4 w = raw[0];
    const uint32_t v = (j / 2) == 0 ? w.x : (j / 2) == 1 ? w.y : (j / 2) == 2 ? w.z : w.w;
    const uint32_t h = (j & 1) ? v >> 16 : v & 0xFFFFu;
    return make_float2((float)(int8_t)(h & 0xFFu) / 128.f, (float)(int8_t)(h >> 8) / 128.f);
  } else {
    const uint4 w = raw[j / 4];
    const uint32_t v = (j & 3) == 0 ? w.x : (j & 3) == 1 ? w.y : (j & 3) == 2 ? w.z : w.w;
    __half2 h;
    memcpy(&h, &v, 4);
    return __half22float2(h);
  }
}

__device__ __forceinline__ uint32_t h2_bits(float a, float b) {
  const __half2 h = __floats2half2_rn(a, b);
  uint32_t u;
  memcpy(&u, &h, 4);
  return u;
}

__device__ __forceinline__ uint32_t bf2_bits(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  uint32_t u;
  memcpy(&u, &h, 4);
  return u;
}

// Power-of-two scale taking a row maximum with bit pattern mbits (>= 0) to
// [128, 256), and its inverse.
__device__ __forceinline__ void row_scale(uint32_t mbits, float &scale, float &inv) {
  if (mbits == 0) {
    scale = inv = 1.f;
    return;
  }
  int se = 261 - (int)(mbits >> 23);
  se = min(max(se, 1), 253);
  scale = __uint_as_float((uint32_t)se << 23);
  inv = __uint_as_float((uint32_t)(254 - se) << 23);
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}
// named barrier among the compute warps
__device__ __forceinline__ void compute_sync() { asm volatile("bar.sync 1, 512;" ::: "memory"); }

// shared -> global bulk copy (16-byte aligned, size a multiple of 16)
__device__ __forceinline__ void bulk_s2g(void *dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(tc::smem_u32(src)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Bounded wait that also gives up as soon as another thread has failed.
__device__ __forceinline__ bool ft_wait(uint64_t *bar, uint32_t parity, volatile int *fail) {
  // a 20 us suspend hint: waiting warps poll less and leave issue slots to
  // the others (an A/B on one B200: 45.4 -> 44.5 us for the slot launch;
  // within the spread between boxes)
  if (tc::mbar_try_wait_hint(bar, parity, 20000u)) return true;
  const uint64_t t0 = tc::globaltimer();
  while (!tc::mbar_try_wait_hint(bar, parity, 20000u)) {
    if (*fail || tc::globaltimer() - t0 > 1000000000ull) {
      *fail = 1;
      return false;
    }
  }
  return true;
}

template <int DT>
__global__ void __launch_bounds__(kFtThreads, 1)
    fft_tc_kernel(const __grid_constant__ CUtensorMap in_map, const FtParams p) {
  extern __shared__ __align__(1024) uint8_t ft_smem[];
  // F, AZ and the ring start on 1024-byte boundaries (the swizzled TMA boxes
  // need them); the staging rows follow
  uint8_t *sF = ft_smem, *sAZ = ft_smem + kMat, *sRing = ft_smem + 2 * kMat;
  uint8_t *sStg = sRing + 2 * kStage;
  // GEMM operand buffers: integer samples fill at most half of a ring slot,
  // so a second buffer (unit i uses buffer i & 1) sits behind ring slot 0's
  // samples and the conversion of unit i + 1 need not wait for GEMM 2 of
  // unit i to read the first; other sample types keep the one buffer.
  // d2_full[u & 1] completes when GEMM 2 of unit u has finished.
  constexpr bool kAZ2 = Fmt<DT>::kUnitBytes + kMat <= kStage;
  uint8_t *const sAZ1 = kAZ2 ? sRing + Fmt<DT>::kUnitBytes : sAZ;
  // Each barrier completes once per unit.  a_ready comes as a pair per ring
  // slot, waited with parity (i >> 1) & 1: the copy warp may trail the
  // compute warps by two units (while it drains a bulk store), and a plain
  // parity wait would then alias a later phase.  full is per slot anyway;
  // every other barrier's waiters are at most one phase behind.
  __shared__ uint64_t bar_mats, full[2], a_ready[2], z_ready, st_ready, d1_full, d2_full[2], st_done;
  __shared__ uint32_t tmem_slot;
  __shared__ __align__(16) uint32_t s_rmax[16];
  __shared__ volatile int s_fail;
  using F = Fmt<DT>;

  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  // this CTA's units: blockIdx.x, blockIdx.x + gridDim.x, ... (strided, so
  // the pilot rows at the front spread over all CTAs), taken in an order
  // rotated by the CTA index, so that the CTAs reach their pilot units (CSI
  // stores, pilot loads) at different times rather than all at the start
  if (blockIdx.x >= p.units) return;
  const uint32_t n_units = (p.units - blockIdx.x + gridDim.x - 1) / gridDim.x;
  const uint32_t rot = blockIdx.x % n_units;
  auto unit_of = [&](uint32_t i) {
    const uint32_t k = i + rot < n_units ? i + rot : i + rot - n_units;
    return blockIdx.x + k * gridDim.x;
  };

  if (tid == kFtCompute) {
    tc::mbar_init(&bar_mats, 1);
    tc::mbar_init(&full[0], 1);
    tc::mbar_init(&full[1], 1);
    tc::mbar_init(&a_ready[0], kFtCompute / 32);
    tc::mbar_init(&a_ready[1], kFtCompute / 32);
    tc::mbar_init(&z_ready, kFtCompute / 32);
    tc::mbar_init(&st_ready, kFtCompute / 32);
    tc::mbar_init(&d1_full, 1);
    tc::mbar_init(&d2_full[0], 1);
    tc::mbar_init(&d2_full[1], 1);
    tc::mbar_init(&st_done, 1);
    s_fail = 0;
    tc::fence_mbar_init();
    tc::prefetch_tmap(&in_map);
  }
  if (warp == 0) tc::tmem_alloc(&tmem_slot, 256);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;  // D1: columns 0..127, D2: 128..255

  // planar BF16 output row of uplink row lrow (rows counted after the
  // pilot rows), plane pl
  auto out_row = [&](uint32_t lrow, uint32_t pl) {
    const uint32_t sym = lrow / p.M, b = lrow - sym * p.M;
    return p.out + ((uint64_t)(sym * 2 + pl) * p.M + b) * p.S_pad;
  };
  const uint32_t S8 = (p.S + 7) & ~7u;  // columns written by the bulk copies (<= S_pad)

  if (warp == kFtCompute / 32) {
    // ================================================== GEMM warp
    if (lane == 0) {
      const uint32_t fa = tc::smem_u32(sF);
      const uint32_t idesc = tc::idesc_f16(128, 128, true, false);  // A MN-major, B K-major
      // both GEMMs read the unit's operand buffer (MN-major) and F (K-major);
      // k step ks of the operand is 4096 bytes on, i.e. 256 in the
      // descriptor's address field (no carry: addresses stay below 256 KB)
      const uint64_t da_0 = tc::smem_desc(tc::smem_u32(sAZ), 2048, 128);
      const uint64_t da_1 = tc::smem_desc(tc::smem_u32(sAZ1), 2048, 128);
      uint64_t db[8];
#pragma unroll
      for (int ks = 0; ks < 8; ks++) db[ks] = tc::smem_desc(fa + ks * 256, 128, 2048);
      uint32_t n_d1 = 0, n_d2 = 0;
      bool ok = ft_wait(&bar_mats, 0, &s_fail);
      for (uint32_t i = 0; i < n_units && ok; i++) {
        // GEMM 1: D1 (128 (r, n2) x 128 (p', k1)) = A (samples) x F
        if (!ft_wait(&a_ready[i & 1], (i >> 1) & 1, &s_fail)) break;
        tc::fence_after_sync();
        const uint64_t da = (i & 1) ? da_1 : da_0;
#pragma unroll
        for (int ks = 0; ks < 8; ks++) tc::mma_f16(tmem, da + (uint64_t)(ks * 256), db[ks], idesc, ks > 0);
        tc::mma_commit(&d1_full);
        n_d1++;
        // GEMM 2: D2 (128 (r, k1) x 128 (p', k2)) = Z x F
        if (!ft_wait(&z_ready, i & 1, &s_fail)) break;
        tc::fence_after_sync();
#pragma unroll
        for (int ks = 0; ks < 8; ks++) tc::mma_f16(tmem + 128, da + (uint64_t)(ks * 256), db[ks], idesc, ks > 0);
        tc::mma_commit(&d2_full[i & 1]);
        n_d2++;
      }
      if (s_fail) {
        // a wait ran out: let the issued GEMMs drain (bounded)
        if (n_d1) tc::mbar_wait(&d1_full, (n_d1 - 1) & 1, 100000000ull);
        for (uint32_t u = n_d2 >= 2 ? n_d2 - 2 : 0; u < n_d2; u++)
          tc::mbar_wait(&d2_full[u & 1], (u >> 1) & 1, 100000000ull);
      }
    }
  } else if (warp == kFtCompute / 32 + 1) {
    // ================================================== copy warp
    if (lane == 0) {
      uint32_t loads[2] = {0, 0};
      auto issue_load = [&](uint32_t i) {
        if (i >= n_units) return;
        const uint32_t u = unit_of(i);
        loads[i & 1]++;
        uint8_t *slot = sRing + (i & 1) * kStage;
        tc::mbar_arrive_expect_tx(&full[i & 1], F::kUnitBytes);
#pragma unroll
        for (uint32_t r = 0; r < 2; r++)
#pragma unroll
          for (uint32_t bx = 0; bx < F::kBoxes; bx++)
            tc::tma_load_2d(slot + (r * F::kBoxes + bx) * 8192, &in_map, (int32_t)(bx * 128),
                            (int32_t)((2 * u + r) * 64), &full[i & 1]);
      };
      // staged rows hold all 4096 bins in subcarrier order; the first
      // S rounded up to 8 go out by bulk copy (within the row pitch)
      auto issue_stores = [&](uint32_t i) {
        const uint32_t u = unit_of(i);
        if (p.inverse) {
          // each staged row holds the N output samples in time order
          const uint32_t ob = p.out_dtype == MB_IQ_I8 ? 2 : 4;
          for (uint32_t r = 0; r < 2; r++) {
            const uint32_t row = 2 * u + r;
            if (row >= p.rows) break;
            bulk_s2g(reinterpret_cast<uint8_t *>(p.tout) + (uint64_t)row * kFtN * ob, sStg + 2 * r * kStgPitch,
                     kFtN * ob);
          }
          bulk_commit();
          return;
        }
        for (uint32_t r = 0; r < 2; r++) {
          const uint32_t row = 2 * u + r;
          if (row >= p.rows) break;
          if (row < p.pilot_rows) continue;
          for (uint32_t pl = 0; pl < 2; pl++)
            bulk_s2g(out_row(row - p.pilot_rows, pl), sStg + (2 * r + pl) * kStgPitch, S8 * 2);
        }
        bulk_commit();
      };
      tc::mbar_arrive_expect_tx(&bar_mats, kMat);
      tc::bulk_g2s(sF, p.mats, kMat, &bar_mats);
      issue_load(0);
      issue_load(1);
      for (uint32_t i = 0; i < n_units; i++) {
        // the ring slot of unit i takes unit i + 2 once unit i is converted
        if (!ft_wait(&a_ready[i & 1], (i >> 1) & 1, &s_fail)) break;
        issue_load(i + 2);
        if (i > 0) {
          if (!ft_wait(&st_ready, (i - 1) & 1, &s_fail)) break;
          issue_stores(i - 1);
          bulk_wait_read();
          mbar_arrive(&st_done);
        }
      }
      if (!s_fail && ft_wait(&st_ready, (n_units - 1) & 1, &s_fail)) issue_stores(n_units - 1);
      bulk_wait_all();
      if (s_fail) {
        // a wait ran out: record it and let the loads in flight land (bounded)
        if (p.err) atomicOr(p.err, tc::kErrTimeout);
        for (int sl = 0; sl < 2; sl++)
          if (loads[sl]) tc::mbar_wait(&full[sl], (loads[sl] - 1) & 1, 100000000ull);
        tc::mbar_wait(&bar_mats, 0, 100000000ull);
      }
    }
  } else {
    // ================================================== compute warps
    bool ok = true;  // warp-uniform: every compute thread runs the same barriers
    auto wait_ok = [&](uint64_t *bar, uint32_t parity) {
      if (ok) ok = ft_wait(bar, parity, &s_fail);
      ok = __all_sync(0xffffffffu, ok);
    };
    auto wait_d2 = [&](uint32_t u) { wait_ok(&d2_full[u & 1], (u >> 1) & 1); };
    auto arrive = [&](uint64_t *bar) {
      tc::fence_proxy_async_smem();
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar);
    };
    // Conversion: thread -> row rh of the unit, 2 chunks of 8 samples (n1,
    // n2 .. n2 + 7); a warp covers 8 consecutive n1 x 4 chunks, so its
    // 16-byte operand stores fill whole core matrices.  Offsets are the same
    // for every unit.
    const uint32_t rh = tid >> 8, wq = (tid >> 5) & 7;
    uint32_t r_off[2][F::kPPC], a_off[2];
#pragma unroll
    for (int c2 = 0; c2 < 2; c2++) {
      const uint32_t q = wq * 2 + c2, n1 = 8 * (q >> 1) + (lane & 7), n2b = 4 * (q & 1) + (lane >> 3);
#pragma unroll
      for (int w = 0; w < (int)F::kPPC; w++) r_off[c2][w] = ring_off<DT>(rh, n1, 8 * n2b + w * (16 / F::kBytes));
      a_off[c2] = mnmaj_off(64 * rh + 8 * n2b, n1);  // imaginary parts 8 K groups (16 KB) further
    }
    // GEMM-1 epilogue: TMEM lane (r, n2), k1 in [16 part, 16 part + 16)
    const uint32_t quad = warp & 3, part = warp >> 2;
    const uint32_t lane_row = quad * 32 + lane;
    const uint32_t tl = tmem + ((quad * 32) << 16);
    const uint32_t e_n2 = lane_row & 63, e_r = lane_row >> 6;
    // W4096^(n2 k1) for k1 = 16 part + j is tw0 tws^j, formed by recurrence in
    // the twiddle phase (15 FP32 complex products: about 2e-6 relative, far
    // below the FP16 rounding of the result); holding all 16 twiddles for the
    // whole kernel cost 32 registers and made the threads spill
    float2 tw0 = __ldg(p.tw + ((e_n2 * 16 * part) & (kFtN - 1)));
    if constexpr (kFixedScale<DT>) {
      // integer samples: the FFT of q * 2^-8 (int16) or of q (int8) is the
      // FFT of the normalised samples q / 2^15 or q / 2^7 times 2^7; the
      // exact 1/128 rides in the twiddles (GEMM 2 is linear), so the
      // epilogues need no multiply
      tw0.x *= 1.0f / 128.0f;
      tw0.y *= 1.0f / 128.0f;
    }
    const float2 tws = __ldg(p.tw + e_n2);
    const uint32_t z_off = mnmaj_off(64 * e_r + 16 * part, e_n2);
    // GEMM-2 epilogue: TMEM lane (r, k1), k2 in [16 part, 16 part + 16); bin
    // k1 + 64 k2 is subcarrier (k1 + 64 k2 - c) mod N.  With c even the even
    // lane's subcarrier is even: lane pairs swap one packed BF16 pair, then
    // the even lane writes the real pair (sc, sc + 1) and the odd lane the
    // imaginary pair (sc - 1, sc), two 64-byte runs in disjoint banks.
    const uint32_t s_r = lane_row >> 6, s_k1 = lane_row & 63;
    const uint32_t s_base = (s_k1 + kFtN - p.c + 1024 * part) & (kFtN - 1);
    const bool odd = lane & 1, pairs = (p.c & 1) == 0;
    const uint32_t perm = odd ? 0x3276u : 0x5410u;
    uint8_t *stg_mine = sStg + (2 * s_r + (odd ? 1 : 0)) * kStgPitch;
    __nv_bfloat16 *stg_re = reinterpret_cast<__nv_bfloat16 *>(sStg + 2 * s_r * kStgPitch);
    __nv_bfloat16 *stg_im = reinterpret_cast<__nv_bfloat16 *>(sStg + (2 * s_r + 1) * kStgPitch);
    __shared__ float s_inv[2][2];  // [unit parity][row] inverse row scales

    auto store_unit = [&](uint32_t i) {
      // row scale to undo (integer samples: none, the 1/128 is already in
      // the twiddles)
      const float inv = kFixedScale<DT> ? 1.0f : s_inv[i & 1][s_r];
      const uint32_t row = 2 * unit_of(i) + s_r;  // the same for the whole warp
      if (!kFixedScale<DT> && p.inverse) {
        // time sample n = k1 + 64 k2 of row s_r: conj of the forward bin,
        // times the row's inverse scale and out_scale; consecutive lanes
        // write consecutive samples
        uint8_t *srow = sStg + 2 * s_r * kStgPitch;
        const float f = inv * p.out_scale;
        const bool i16 = p.out_dtype == MB_IQ_I16, i8 = p.out_dtype == MB_IQ_I8;
        const float qmax = i16 ? 32767.f : 127.f, qmin = i16 ? -32768.f : -128.f;
#pragma unroll
        for (int jb = 0; jb < 16; jb += 8) {
          float vr[8], vi[8];
          tc::tmem_ld8x2(tl + 128 + 16 * part + jb, vr, tl + 192 + 16 * part + jb, vi);
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const uint32_t n = s_k1 + 64 * (16 * part + jb + j);
            const float re = vr[j] * f, im = -vi[j] * f;
            if (i16 || i8) {
              int qr = __float2int_rn(re), qi = __float2int_rn(im);
              if (re > qmax) qr = (int)qmax; else if (re < qmin) qr = (int)qmin;
              if (im > qmax) qi = (int)qmax; else if (im < qmin) qi = (int)qmin;
              if (i16)
                *reinterpret_cast<short2 *>(srow + 4 * n) = make_short2((short)qr, (short)qi);
              else
                *reinterpret_cast<char2 *>(srow + 2 * n) = make_char2((char)qr, (char)qi);
            } else {
              *reinterpret_cast<__half2 *>(srow + 4 * n) = __floats2half2_rn(re, im);
            }
          }
        }
        arrive(&st_ready);
        return;
      }
      if (row < p.pilot_rows) {
        // LS estimate conj(X) p of subcarrier sc for user u0 + sc % sg into
        // csi[sc / sg][b][u] (fft_callback.cuh:76-108); a user with no pilot
        // in the short last group takes its estimate from group G-2.  Eight
        // bins at a time (half the accumulator registers live at once, which
        // keeps this branch from spilling); their pilot signs are loaded
        // before any branch, so the latencies overlap.
        const uint32_t sym = row / p.M, b = row - sym * p.M, u0 = p.ue_start + sym * p.sg;
#pragma unroll
        for (int jb = 0; jb < 16; jb += 8) {
          float2 ps[8];
#pragma unroll
          for (int j = 0; j < 8; j++) ps[j] = __ldg(p.pilot + min((s_base + 64 * (jb + j)) & (kFtN - 1), p.S - 1));
          float vr[8], vi[8];
          tc::tmem_ld8x2(tl + 128 + 16 * part + jb, vr, tl + 192 + 16 * part + jb, vi);
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const uint32_t sc = (s_base + 64 * (jb + j)) & (kFtN - 1);
            const uint32_t g = __umulhi(sc, p.sg_magic), sl = sc - g * p.sg, uu = u0 + sl;
            const float x = vr[j] * inv, y = vi[j] * inv;
            const float2 e = make_float2(x * ps[j].x + y * ps[j].y, x * ps[j].y - y * ps[j].x);
            if (sc < p.S && uu < p.K) {
              float2 *d = p.csi + ((uint64_t)g * p.M + b) * p.K + uu;
              *d = e;
              if (p.tail_rem && g + 2 == p.G && sl >= p.tail_rem) d[(uint64_t)p.M * p.K] = e;
            }
          }
        }
        arrive(&st_ready);
        return;
      }
      if (pairs) {
#pragma unroll
        for (int jb = 0; jb < 16; jb += 8) {
          float vr[8], vi[8];
          tc::tmem_ld8x2(tl + 128 + 16 * part + jb, vr, tl + 192 + 16 * part + jb, vi);
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const uint32_t own = bf2_bits(vr[j] * inv, vi[j] * inv);
            const uint32_t other = __shfl_xor_sync(0xffffffffu, own, 1);
            const uint32_t s0 = (s_base + 64 * (jb + j)) & (kFtN - 2);
            *reinterpret_cast<uint32_t *>(stg_mine + 2 * s0) = __byte_perm(own, other, perm);
          }
        }
      } else {
        float vr[16], vi[16];
        tc::tmem_ld16(tl + 128 + 16 * part, vr);
        tc::tmem_ld16(tl + 192 + 16 * part, vi);
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const uint32_t sc = (s_base + 64 * j) & (kFtN - 1);
          stg_re[sc] = __float2bfloat16_rn(vr[j] * inv);
          stg_im[sc] = __float2bfloat16_rn(vi[j] * inv);
        }
      }
      arrive(&st_ready);
    };

    for (uint32_t i = 0; i < n_units; i++) {
      const uint8_t *slot = sRing + (i & 1) * kStage;
      // (a) conversion: row maximum, power-of-two scale, FP16 operand A
      wait_ok(&full[i & 1], (i >> 1) & 1);
      uint4 re[2], im[2];
      {
        uint4 raw[2][F::kPPC];
#pragma unroll
        for (int c2 = 0; c2 < 2; c2++)
#pragma unroll
          for (int w = 0; w < (int)F::kPPC; w++) raw[c2][w] = *reinterpret_cast<const uint4 *>(slot + r_off[c2][w]);
        if constexpr (kFixedScale<DT>) {
          // integer samples: |q| <= 2^15 (int16) or 2^7 (int8) converts to
          // FP16 and a fixed power of two takes it below 2^7 (exact), so no
          // row maximum is needed
          const __half2 sc2 = __float2half2_rn(DT == MB_IQ_I16 ? 1.0f / 256.0f : 1.0f);
#pragma unroll
          for (int c2 = 0; c2 < 2; c2++) {
            uint32_t rw[4], iw[4];
#pragma unroll
            for (int t = 0; t < 4; t++) {
              __half2 hr, hi;
              if constexpr (DT == MB_IQ_I16) {
                const uint4 w = raw[c2][t / 2];
                const uint32_t a = (t & 1) ? w.z : w.x, b = (t & 1) ? w.w : w.y;  // samples 2t, 2t+1
                hr = __halves2half2(__short2half_rn((short)(a & 0xFFFFu)), __short2half_rn((short)(b & 0xFFFFu)));
                hi = __halves2half2(__short2half_rn((short)(a >> 16)), __short2half_rn((short)(b >> 16)));
              } else {
                // int8 (re, im, re, im) bytes: with the sign bits flipped a
                // byte is x + 128, and the FP16 bit pattern 0x64XX is
                // 1024 + XX exactly, so one byte permute per half2 and one
                // subtraction of 1152 give x (exact)
                const uint4 w = raw[c2][0];
                const uint32_t v = (t == 0 ? w.x : t == 1 ? w.y : t == 2 ? w.z : w.w) ^ 0x80808080u;
                const uint32_t rb = __byte_perm(v, 0x64646464u, 0x4240u);  // bytes 0, 2 (re)
                const uint32_t ib = __byte_perm(v, 0x64646464u, 0x4341u);  // bytes 1, 3 (im)
                const __half2 bias = __float2half2_rn(1152.0f);
                memcpy(&hr, &rb, 4);
                memcpy(&hi, &ib, 4);
                hr = __hsub2(hr, bias);
                hi = __hsub2(hi, bias);
              }
              if constexpr (DT == MB_IQ_I16) {
                hr = __hmul2(hr, sc2);
                hi = __hmul2(hi, sc2);
              }
              memcpy(&rw[t], &hr, 4);
              memcpy(&iw[t], &hi, 4);
            }
            re[c2] = make_uint4(rw[0], rw[1], rw[2], rw[3]);
            im[c2] = make_uint4(iw[0], iw[1], iw[2], iw[3]);
          }
        } else {
          float m = 0.f;
#pragma unroll
          for (int c2 = 0; c2 < 2; c2++)
#pragma unroll
            for (int j = 0; j < 8; j++) {
              const float2 v = chunk_sample<DT>(raw[c2], j);
              m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
            }
          const uint32_t mb = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
          if (lane == 0) s_rmax[warp] = mb;
          compute_sync();
          const uint4 m0 = *reinterpret_cast<const uint4 *>(&s_rmax[rh * 8]);
          const uint4 m1 = *reinterpret_cast<const uint4 *>(&s_rmax[rh * 8 + 4]);
          const uint32_t rmax = max(max(max(m0.x, m0.y), max(m0.z, m0.w)), max(max(m1.x, m1.y), max(m1.z, m1.w)));
          float scale, inv;
          row_scale(rmax, scale, inv);
          if ((tid & 255) == 0) s_inv[i & 1][rh] = inv;
          const float iscale = p.inverse ? -scale : scale;  // conj(z) for the inverse
#pragma unroll
          for (int c2 = 0; c2 < 2; c2++) {
            float2 v[8];
#pragma unroll
            for (int j = 0; j < 8; j++) v[j] = chunk_sample<DT>(raw[c2], j);
            re[c2] = make_uint4(h2_bits(v[0].x * scale, v[1].x * scale), h2_bits(v[2].x * scale, v[3].x * scale),
                                h2_bits(v[4].x * scale, v[5].x * scale), h2_bits(v[6].x * scale, v[7].x * scale));
            im[c2] = make_uint4(h2_bits(v[0].y * iscale, v[1].y * iscale), h2_bits(v[2].y * iscale, v[3].y * iscale),
                                h2_bits(v[4].y * iscale, v[5].y * iscale), h2_bits(v[6].y * iscale, v[7].y * iscale));
          }
        }
      }
      // the operand buffer holds Z of its previous unit (i - 2 with two
      // buffers, i - 1 with one) until that unit's GEMM 2 has read it
      uint8_t *az = (i & 1) ? sAZ1 : sAZ;
      if (kAZ2 ? i > 1 : i > 0) wait_d2(kAZ2 ? i - 2 : i - 1);
      tc::fence_after_sync();
      if (ok) {
#pragma unroll
        for (int c2 = 0; c2 < 2; c2++) {
          *reinterpret_cast<uint4 *>(az + a_off[c2]) = re[c2];
          *reinterpret_cast<uint4 *>(az + a_off[c2] + 16384) = im[c2];
        }
      }
      arrive(&a_ready[i & 1]);
      // (b) GEMM-2 epilogue of the previous unit into the staging rows,
      // once the bulk copies of the unit before it have read them
      if (i > 0) {
        wait_d2(i - 1);  // D2 of unit i - 1 (already waited with one buffer)
        tc::fence_after_sync();
        if (i > 1) wait_ok(&st_done, (i - 2) & 1);
        if (ok) store_unit(i - 1);
        else arrive(&st_ready);
      }
      // (c) GEMM-1 epilogue: twiddle into the GEMM-2 operand Z
      wait_ok(&d1_full, i & 1);
      tc::fence_after_sync();
      if (ok) {
        float2 w = tw0;
        // eight k1 at a time: half the accumulator registers live at once
#pragma unroll
        for (int g = 0; g < 2; g++) {
          float yr[8], yi[8];
          tc::tmem_ld8x2(tl + 16 * part + 8 * g, yr, tl + 64 + 16 * part + 8 * g, yi);
          float zr[8], zi[8];
#pragma unroll
          for (int b = 0; b < 8; b++) {
            const float xr = yr[b], xi = yi[b];
            zr[b] = xr * w.x - xi * w.y;
            zi[b] = xr * w.y + xi * w.x;
            w = make_float2(w.x * tws.x - w.y * tws.y, w.x * tws.y + w.y * tws.x);
          }
          *reinterpret_cast<uint4 *>(az + z_off + g * 128) =
              make_uint4(h2_bits(zr[0], zr[1]), h2_bits(zr[2], zr[3]), h2_bits(zr[4], zr[5]), h2_bits(zr[6], zr[7]));
          *reinterpret_cast<uint4 *>(az + z_off + g * 128 + 16384) =
              make_uint4(h2_bits(zi[0], zi[1]), h2_bits(zi[2], zi[3]), h2_bits(zi[4], zi[5]), h2_bits(zi[6], zi[7]));
        }
      }
      arrive(&z_ready);
    }
    // the last unit's inverse scales were written after the last barrier
    if constexpr (!kFixedScale<DT>) compute_sync();
    wait_d2(n_units - 1);
    tc::fence_after_sync();
    if (n_units > 1) wait_ok(&st_done, (n_units - 2) & 1);
    if (ok) store_unit(n_units - 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

using FtKernel = void (*)(const CUtensorMap, const FtParams);
FtKernel fft_tc_kernel_of(int dt) {
  switch (dt) {
    case MB_IQ_C32: return fft_tc_kernel<MB_IQ_C32>;
    case MB_IQ_I16: return fft_tc_kernel<MB_IQ_I16>;
    case MB_IQ_I8: return fft_tc_kernel<MB_IQ_I8>;
    default: return fft_tc_kernel<MB_IQ_F16>;
  }
}

// raises the dynamic shared memory limit of a sample type's kernel once per
// device, and returns the device's SM count
mb_status fft_tc_configure(int dt, int dev, int *sms) {
  static std::atomic<uint64_t> configured[4] = {};
  static std::atomic<int> sm_count[64] = {};
  const int which = dt == MB_IQ_C32 ? 0 : dt == MB_IQ_I16 ? 1 : dt == MB_IQ_I8 ? 2 : 3;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(configured[which].load() & bit)) {
    MB_CUDA_TRY(cudaFuncSetAttribute(fft_tc_kernel_of(dt), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kFtSmem));
    int n = 0;
    MB_CUDA_TRY(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    sm_count[dev & 63].store(n);
    configured[which].fetch_or(bit);
  }
  *sms = sm_count[dev & 63].load();
  return MB_OK;
}

// one wave: units spread evenly over at most one CTA per SM
mb_status fft_tc_launch(const FftTcPlan *pl, const void *iq, int iq_dtype, FtParams &p, cudaStream_t st,
                        uint32_t upc) {
  int dev = 0, sms = 0;
  MB_CUDA_TRY(cudaGetDevice(&dev));
  mb_status r = fft_tc_configure(iq_dtype, dev, &sms);
  if (r != MB_OK) return r;
  const uint32_t bytes = iq_dtype == MB_IQ_C32 ? 8 : iq_dtype == MB_IQ_I8 ? 2 : 4;
  // the rows as 64-sample n1 rows of 64 * bytes bytes, read in 128-byte boxes
  CUtensorMap map;
  r = make_tmap_2d_u8_sw128(&map, iq, 64ull * bytes, (uint64_t)p.rows * 64, 64ull * bytes, 64);
  if (r != MB_OK) return r;
  p.mats = pl->mats;
  p.tw = pl->tw;
  p.c = pl->c;
  p.units = (p.rows + 1) / 2;
  p.upc = upc ? upc : (p.units + (uint32_t)max(sms, 1) - 1) / (uint32_t)max(sms, 1);
  const uint32_t grid = (p.units + p.upc - 1) / p.upc;
  fft_tc_kernel_of(iq_dtype)<<<grid, kFtThreads, kFtSmem, st>>>(map, p);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

}  // namespace

FftTcPlan *fft_tc_plan_create(uint32_t N, uint32_t start) {
  if (N != kFtN) return nullptr;
  const uint32_t c = (start + N / 2) % N;
  // F[(p', k)][(p, n)]: real embedding of W64^(n k).  Row (p', k) weighs the
  // (re, im) inputs by (Re W, -Im W) for the real output p' = 0 and by
  // (Im W, Re W) for p' = 1.
  std::vector<uint16_t> mats(kMat / 2, 0);
  for (uint32_t k = 0; k < 64; k++)
    for (uint32_t n = 0; n < 64; n++) {
      const double ang = 2.0 * kPi * (double)((n * k) % 64) / 64.0;
      const float wr = (float)std::cos(ang), wi = (float)-std::sin(ang);
      const float v[2][2] = {{wr, -wi}, {wi, wr}};  // [p'][p]
      for (int pp = 0; pp < 2; pp++)
        for (int pi = 0; pi < 2; pi++) {
          const __half h = __float2half_rn(v[pp][pi]);
          uint16_t bits;
          memcpy(&bits, &h, 2);
          mats[kmaj_off(64 * pp + k, 64 * pi + n) / 2] = bits;
        }
    }
  std::vector<float2> tw(kFtN);
  for (uint32_t j = 0; j < kFtN; j++) {
    const double ang = 2.0 * kPi * (double)j / (double)kFtN;
    tw[j] = make_float2((float)std::cos(ang), (float)-std::sin(ang));
  }
  FftTcPlan *pl = new FftTcPlan{nullptr, nullptr, c};
  cudaError_t e = cudaMalloc(&pl->mats, kMat);
  if (e == cudaSuccess) e = cudaMalloc(&pl->tw, sizeof(float2) * kFtN);
  if (e == cudaSuccess) e = cudaMemcpy(pl->mats, mats.data(), kMat, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(pl->tw, tw.data(), sizeof(float2) * kFtN, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    record_error(e);
    fft_tc_plan_destroy(pl);
    return nullptr;
  }
  return pl;
}

void fft_tc_plan_destroy(FftTcPlan *pl) {
  if (!pl) return;
  cudaFree(pl->mats);
  cudaFree(pl->tw);
  delete pl;
}

bool fft_tc_lp_supported(const FftTcPlan *pl, const void *iq, uint32_t S_pad, const void *y_lp) {
  return pl && S_pad % 8 == 0 && (reinterpret_cast<uintptr_t>(iq) & 15) == 0 &&
         (reinterpret_cast<uintptr_t>(y_lp) & 15) == 0;
}

mb_status fft_tc_uplink_lp(const FftTcPlan *pl, const void *iq, int iq_dtype, uint32_t rows, uint32_t M,
                           uint32_t S, void *y_lp, uint32_t S_pad, int *err, cudaStream_t st,
                           uint32_t upc) {
  if (!fft_tc_lp_supported(pl, iq, S_pad, y_lp) || S > kFtN || S > S_pad) return MB_BAD_ARG;
  if (rows == 0) return MB_OK;
  FtParams p{};
  p.rows = rows;
  p.M = M;
  p.S = S;
  p.S_pad = S_pad;
  p.out = reinterpret_cast<__nv_bfloat16 *>(y_lp);
  p.err = err;
  p.pilot_rows = 0;
  return fft_tc_launch(pl, iq, iq_dtype, p, st, upc);
}

bool fft_tc_inverse_supported(const FftTcPlan *pl, const void *in, int in_dtype, const void *out, int out_dtype) {
  return pl && (in_dtype == MB_IQ_C32 || in_dtype == MB_IQ_F16) &&
         (out_dtype == MB_IQ_I16 || out_dtype == MB_IQ_I8 || out_dtype == MB_IQ_F16) &&
         (reinterpret_cast<uintptr_t>(in) & 15) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
}

mb_status fft_tc_inverse(const FftTcPlan *pl, const void *in, int in_dtype, uint32_t rows, void *out, int out_dtype,
                         int *err, cudaStream_t st) {
  if (!fft_tc_inverse_supported(pl, in, in_dtype, out, out_dtype)) return MB_BAD_ARG;
  if (rows == 0) return MB_OK;
  FtParams p{};
  p.rows = rows;
  p.pilot_rows = 0;
  p.M = 1;
  p.inverse = 1;
  p.out_dtype = out_dtype;
  p.out_scale = out_dtype == MB_IQ_I16 ? 32768.f / kFtN : out_dtype == MB_IQ_I8 ? 128.f / kFtN : 1.f / kFtN;
  p.tout = out;
  p.err = err;
  return fft_tc_launch(pl, in, in_dtype, p, st, 0);
}

bool fft_tc_pilot_supported(const FftTcPlan *pl, const void *iq) {
  return pl && (reinterpret_cast<uintptr_t>(iq) & 15) == 0;
}

mb_status fft_tc_pilot(const FftTcPlan *pl, const void *iq, int iq_dtype, uint32_t n_sym, uint32_t M, uint32_t S,
                       uint32_t K, uint32_t sg, uint32_t ue_start, uint32_t tail_rem, const float2 *pilot,
                       float2 *csi, int *err, cudaStream_t st, uint32_t upc) {
  if (!fft_tc_pilot_supported(pl, iq) || S > kFtN || sg == 0 || sg >= kFtN || !pilot || !csi) return MB_BAD_ARG;
  if (n_sym == 0 || M == 0) return MB_OK;
  FtParams p{};
  p.rows = n_sym * M;
  p.M = M;
  p.S = S;
  p.csi = csi;
  p.pilot = pilot;
  p.K = K;
  p.sg = sg;
  p.ue_start = ue_start;
  p.tail_rem = tail_rem;
  p.G = (S + sg - 1) / sg;
  p.sg_magic = (uint32_t)((0x100000000ull + sg - 1) / sg);
  p.err = err;
  p.pilot_rows = p.rows;
  return fft_tc_launch(pl, iq, iq_dtype, p, st, upc);
}

mb_status fft_tc_slot(const FftTcPlan *pl, const void *iq, int iq_dtype, uint32_t P, uint32_t U, uint32_t M,
                      uint32_t S, uint32_t K, uint32_t sg, uint32_t tail_rem, const float2 *pilot, float2 *csi,
                      void *y_lp, uint32_t S_pad, int *err, cudaStream_t st, uint32_t upc) {
  if (!fft_tc_lp_supported(pl, iq, S_pad, y_lp) || S > kFtN || S > S_pad || sg == 0 || sg >= kFtN || !pilot ||
      !csi)
    return MB_BAD_ARG;
  FtParams p{};
  p.rows = (P + U) * M;
  p.pilot_rows = P * M;
  if (p.rows == 0) return MB_OK;
  p.M = M;
  p.S = S;
  p.S_pad = S_pad;
  p.out = reinterpret_cast<__nv_bfloat16 *>(y_lp);
  p.csi = csi;
  p.pilot = pilot;
  p.K = K;
  p.sg = sg;
  p.ue_start = 0;
  p.tail_rem = tail_rem;
  p.G = (S + sg - 1) / sg;
  p.sg_magic = (uint32_t)((0x100000000ull + sg - 1) / sg);
  p.err = err;
  return fft_tc_launch(pl, iq, iq_dtype, p, st, upc);
}

}  // namespace mb

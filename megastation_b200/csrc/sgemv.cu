// sgemv.cu -- fused equalize+demodulate+descramble and precode (FP32 SIMT).
//
// Equalize replaces EqualizeKernel (sgemv/equalize_kernel.cuh:27-481, one
// GEMV per subcarrier, one launch per symbol) with a batched complex GEMM
// per subcarrier group: X (K x L*sg) = W_g^T (K x M) * Y (M x L*sg) over L
// symbols at once, so the detector W_g is read once per L symbols instead
// of once per symbol.  The epilogue applies the reference demapper in FP16
// (modulation/demodulation.h:30-67), places the LLRs in the code-block
// layout (equalize_kernel.cuh:272-287) and packs descrambled hard bits.
//
// Precode replaces PrecodeKernel (sgemv/precode_kernel.cuh:25-387) the same
// way: Z (M x L*sg) = P_g^T (M x K) * S (K x L*sg), scattered into the
// FFT-shifted N-point rows, with the guard bins written as zero.
#include <algorithm>

#include "common.cuh"
#include "eq_common.cuh"
#include "sgemv.cuh"

namespace mb {

// SIMT epilogue: demap, store LLRs, OR the Qm hard bits into the CTA's
// word buffer hw (per (l_local, u) row of hw_words words, bit offsets
// relative to the group's first stream bit, MSB-first bytes).
__device__ __forceinline__ void equalize_store(const EqParams &p, uint32_t l,
                                               uint32_t l_local, uint32_t u,
                                               uint32_t s, uint32_t s_local,
                                               float2 x, uint32_t *hw) {
  if (p.x) p.x[((uint64_t)l * p.K + u) * p.S + s] = x;
  __half *row = reinterpret_cast<__half *>(p.llr) + ((uint64_t)l * p.K + u) * p.row_len;
  const uint32_t hb = eq_demap_store(p, row, s, x);
  if (hw && hb) {
    uint32_t *w = hw + ((uint64_t)l_local * p.K + u) * p.hw_words;
    for (uint32_t q = 0; q < p.Qm; q++) {
      if (!((hb >> (p.Qm - 1 - q)) & 1u)) continue;
      const uint32_t rel = s_local * p.Qm + q;  // bit within the group
      const uint32_t byte = rel >> 3, bit = 7 - (rel & 7);
      atomicOr(w + byte / 4, 1u << (8 * (byte % 4) + bit));
    }
  }
}

// Writes the CTA's hard-bit bytes: group g covers stream bits starting at
// g*sg*Qm, which is byte aligned because sg*Qm % 8 == 0.
__device__ __forceinline__ void equalize_flush_hard(const EqParams &p,
                                                    uint32_t g, uint32_t l0,
                                                    uint32_t nl,
                                                    const uint32_t *hw) {
  const uint64_t byte0 = (uint64_t)g * p.sg * p.Qm / 8;
  const uint32_t nbytes = p.sg * p.Qm / 8;
  const uint32_t total = nl * p.K * nbytes;
  for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
    uint32_t rb = e % nbytes, lu = e / nbytes;
    uint64_t gb = byte0 + rb;
    if (gb * 8 >= p.n_valid) continue;
    uint32_t word = hw[(uint64_t)lu * p.hw_words + rb / 4];
    uint8_t v = (uint8_t)(word >> (8 * (rb % 4)));
    uint32_t l = l0 + lu / p.K, u = lu % p.K;
    p.hard[((uint64_t)l * p.K + u) * p.hrow + gb] = v ^ eq_seq_byte(p, u, (uint32_t)gb);
  }
}

constexpr int kEqKB = 16;  // antennas per shared-memory k tile

template <int TU, int TC>
__global__ void __launch_bounds__(256) equalize_fp32_kernel(const EqParams p) {
  constexpr int CT = 32, UT = 8;
  __shared__ float2 Ws[kEqKB][8 * TU];
  __shared__ float2 Ys[kEqKB][CT * TC];
  extern __shared__ uint32_t eq_hw[];
  const uint32_t g = blockIdx.x;
  const uint32_t l0 = blockIdx.y * p.L;
  const uint32_t nl = min(p.L, p.n_sym - l0);
  const uint32_t s_begin = g * p.sg;
  const uint32_t ns = min(p.sg, p.S - s_begin);
  const uint32_t ncols = nl * p.sg;
  const int tid = threadIdx.x, tc = tid % CT, tu = tid / CT;
  uint32_t *hw = p.hard ? eq_hw : nullptr;
  if (hw)
    for (uint32_t e = tid; e < nl * p.K * p.hw_words; e += blockDim.x) hw[e] = 0;

  float2 acc[TU][TC];
#pragma unroll
  for (int i = 0; i < TU; i++)
#pragma unroll
    for (int j = 0; j < TC; j++) acc[i][j] = make_float2(0.f, 0.f);

  const float2 *Wg = p.W + (uint64_t)g * p.M * p.K;
  for (uint32_t b0 = 0; b0 < p.M; b0 += kEqKB) {
    for (uint32_t e = tid; e < kEqKB * 8 * TU; e += blockDim.x) {
      uint32_t b = e / (8 * TU), u = e % (8 * TU);
      float2 v = make_float2(0.f, 0.f);
      if (b0 + b < p.M && u < p.K) v = __ldg(Wg + (uint64_t)(b0 + b) * p.K + u);
      Ws[b][u] = v;
    }
    for (uint32_t e = tid; e < kEqKB * CT * TC; e += blockDim.x) {
      uint32_t b = e / (CT * TC), c = e % (CT * TC);
      float2 v = make_float2(0.f, 0.f);
      uint32_t ll = c / p.sg, sl = c % p.sg;
      if (b0 + b < p.M && c < ncols && sl < ns)
        v = __ldg(p.y + ((uint64_t)(l0 + ll) * p.M + b0 + b) * p.S + s_begin + sl);
      Ys[b][c] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int b = 0; b < kEqKB; b++) {
      float2 w[TU], yv[TC];
#pragma unroll
      for (int i = 0; i < TU; i++) w[i] = Ws[b][tu + i * UT];
#pragma unroll
      for (int j = 0; j < TC; j++) yv[j] = Ys[b][tc + j * CT];
#pragma unroll
      for (int i = 0; i < TU; i++)
#pragma unroll
        for (int j = 0; j < TC; j++) cfma(acc[i][j], w[i], yv[j]);
    }
    __syncthreads();
  }

#pragma unroll
  for (int i = 0; i < TU; i++)
#pragma unroll
    for (int j = 0; j < TC; j++) {
      const uint32_t u = tu + i * UT, c = tc + j * CT;
      if (u >= p.K || c >= ncols) continue;
      const uint32_t ll = c / p.sg, sl = c % p.sg;
      if (sl >= ns) continue;
      equalize_store(p, l0 + ll, ll, u, s_begin + sl, sl, acc[i][j], hw);
    }
  if (hw) {
    __syncthreads();
    equalize_flush_hard(p, g, l0, nl, hw);
  }
}

template <int TU, int TC>
static mb_status launch_eq(const EqParams &p, uint32_t G, cudaStream_t st) {
  dim3 grid(G, (p.n_sym + p.L - 1) / p.L);
  size_t smem = p.hard ? sizeof(uint32_t) * p.L * p.K * p.hw_words : 0;
  equalize_fp32_kernel<TU, TC><<<grid, 256, smem, st>>>(p);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

mb_status equalize_fp32(EqParams p, cudaStream_t st) {
  const uint32_t G = (p.S + p.sg - 1) / p.sg;
  int tu = p.K <= 8 ? 1 : p.K <= 16 ? 2 : p.K <= 32 ? 4 : 8;
  uint32_t L = std::max<uint32_t>(1, 64 / p.sg);
  L = std::min(L, p.n_sym);
  uint32_t ncols = L * p.sg;
  int tc = ncols <= 32 ? 1 : ncols <= 64 ? 2 : 4;
  if (ncols > 128) return MB_UNSUPPORTED;
  p.L = L;
#define EQ_CASE(a, b) \
  if (tu == a && tc == b) return launch_eq<a, b>(p, G, st);
  EQ_CASE(1, 1) EQ_CASE(1, 2) EQ_CASE(1, 4)
  EQ_CASE(2, 1) EQ_CASE(2, 2) EQ_CASE(2, 4)
  EQ_CASE(4, 1) EQ_CASE(4, 2) EQ_CASE(4, 4)
  EQ_CASE(8, 1) EQ_CASE(8, 2) EQ_CASE(8, 4)
#undef EQ_CASE
  return MB_UNSUPPORTED;
}

// ---- precode ------------------------------------------------------------
struct PcParams {
  const float2 *P;  // [G][K][M]
  const float2 *s;  // [n_sym][K][S]
  float2 *out;      // [n_sym][M][N]
  uint32_t M, K, S, sg, N, start, n_sym, L;
};

constexpr int kPcUB = 16;  // users per shared-memory k tile

template <int TB, int TC>
__global__ void __launch_bounds__(256) precode_kernel(const PcParams p) {
  constexpr int CT = 32, BT = 8;
  __shared__ float2 Ps[kPcUB][BT * TB];
  __shared__ float2 Ss[kPcUB][CT * TC];
  const uint32_t G = (p.S + p.sg - 1) / p.sg;
  const uint32_t g = blockIdx.x;
  const uint32_t l0 = blockIdx.y * p.L;
  const uint32_t nl = min(p.L, p.n_sym - l0);
  const uint32_t b_base = blockIdx.z * BT * TB;
  const int tid = threadIdx.x, tc = tid % CT, tb = tid / CT;
  if (g == G) {
    // guard bins: subcarrier indices i in [S, N) map to the bins
    // (i + start + N/2) % N, one run of N - S bins per row that may wrap
    // around N: zero the runs of this CTA's rows, a warp per row
    const uint32_t nb = min((uint32_t)(BT * TB), p.M - b_base);
    const uint32_t ng = p.N - p.S;
    const uint32_t k0 = (p.S + p.start + p.N / 2) % p.N;
    const uint32_t n1 = min(ng, p.N - k0);  // bins k0 .. k0 + n1 - 1, then 0 .. ng - n1 - 1
    const int warp = tid / 32, lane = tid % 32;
    for (uint32_t r = warp; r < nl * nb; r += blockDim.x / 32) {
      const uint32_t b = b_base + r % nb, l = l0 + r / nb;
      float2 *row = p.out + ((uint64_t)l * p.M + b) * p.N;
      for (uint32_t e = lane; e < n1; e += 32) row[k0 + e] = make_float2(0.f, 0.f);
      for (uint32_t e = lane; e < ng - n1; e += 32) row[e] = make_float2(0.f, 0.f);
    }
    return;
  }
  const uint32_t s_begin = g * p.sg;
  const uint32_t ns = min(p.sg, p.S - s_begin);
  const uint32_t ncols = nl * p.sg;
  float2 acc[TB][TC];
#pragma unroll
  for (int i = 0; i < TB; i++)
#pragma unroll
    for (int j = 0; j < TC; j++) acc[i][j] = make_float2(0.f, 0.f);
  const float2 *Pg = p.P + (uint64_t)g * p.K * p.M;
  for (uint32_t u0 = 0; u0 < p.K; u0 += kPcUB) {
    for (uint32_t e = tid; e < kPcUB * BT * TB; e += blockDim.x) {
      uint32_t u = e / (BT * TB), b = e % (BT * TB);
      float2 v = make_float2(0.f, 0.f);
      if (u0 + u < p.K && b_base + b < p.M)
        v = __ldg(Pg + (uint64_t)(u0 + u) * p.M + b_base + b);
      Ps[u][b] = v;
    }
    for (uint32_t e = tid; e < kPcUB * CT * TC; e += blockDim.x) {
      uint32_t u = e / (CT * TC), c = e % (CT * TC);
      float2 v = make_float2(0.f, 0.f);
      uint32_t ll = c / p.sg, sl = c % p.sg;
      if (u0 + u < p.K && c < ncols && sl < ns)
        v = __ldg(p.s + ((uint64_t)(l0 + ll) * p.K + u0 + u) * p.S + s_begin + sl);
      Ss[u][c] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int u = 0; u < kPcUB; u++) {
      float2 w[TB], sv[TC];
#pragma unroll
      for (int i = 0; i < TB; i++) w[i] = Ps[u][tb + i * BT];
#pragma unroll
      for (int j = 0; j < TC; j++) sv[j] = Ss[u][tc + j * CT];
#pragma unroll
      for (int i = 0; i < TB; i++)
#pragma unroll
        for (int j = 0; j < TC; j++) cfma(acc[i][j], w[i], sv[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < TB; i++)
#pragma unroll
    for (int j = 0; j < TC; j++) {
      const uint32_t b = b_base + tb + i * BT, c = tc + j * CT;
      if (b >= p.M || c >= ncols) continue;
      const uint32_t ll = c / p.sg, sl = c % p.sg;
      if (sl >= ns) continue;
      const uint32_t k = (s_begin + sl + p.start + p.N / 2) % p.N;
      p.out[((uint64_t)(l0 + ll) * p.M + b) * p.N + k] = acc[i][j];
    }
}

mb_status precode_fp32(const float2 *P, const float2 *s, float2 *out,
                       uint32_t M, uint32_t K, uint32_t S, uint32_t sg,
                       uint32_t N, uint32_t start, uint32_t n_sym,
                       cudaStream_t st) {
  PcParams p{P, s, out, M, K, S, sg, N, start, n_sym, 0};
  uint32_t L = std::max<uint32_t>(1, 64 / sg);
  L = std::min(L, n_sym);
  p.L = L;
  const uint32_t ncols = L * sg;
  const uint32_t G = (S + sg - 1) / sg;
  constexpr int TB = 4;
  dim3 grid(G + 1, (n_sym + L - 1) / L, (M + 8 * TB - 1) / (8 * TB));
  if (ncols <= 32)
    precode_kernel<TB, 1><<<grid, 256, 0, st>>>(p);
  else if (ncols <= 64)
    precode_kernel<TB, 2><<<grid, 256, 0, st>>>(p);
  else if (ncols <= 128)
    precode_kernel<TB, 4><<<grid, 256, 0, st>>>(p);
  else
    return MB_UNSUPPORTED;
  MB_LAUNCH_CHECK();
  return MB_OK;
}

}  // namespace mb

using namespace mb;

// The descrambling sequence is stored expanded into MSB-first bytes (bit t
// of the stream is bit 7 - t % 8 of byte t / 8, the byte order of
// scrambler_kernel.cuh:43-50), so descrambling packed hard bits is one XOR
// per byte.
struct mb_scrambler {
  uint8_t *bytes;       // device
  uint64_t nbits;       // bits available per user
  uint64_t row_bytes;   // byte stride between users (0: shared by all users)
  uint32_t num_ue;
};

const uint8_t *mb::scrambler_bytes(const mb_scrambler *s, uint64_t *nbits,
                                   uint64_t *row_bytes) {
  *nbits = s->nbits;
  *row_bytes = s->row_bytes;
  return s->bytes;
}

extern "C" mb_status mb_scrambler_create(int mode, uint32_t c_init,
                                         uint32_t num_ue, uint64_t num_bits,
                                         mb_scrambler **out) {
  if (!out) return MB_BAD_ARG;
  *out = nullptr;
  if (!device_tables()) return MB_CUDA_ERROR;
  std::vector<uint8_t> h;
  uint64_t nbits = 0, row_bytes = 0;
  if (mode == MB_SCR_LFSR127) {
    // scrambler/scrambler.cu:22-31: period 127, the same for every user;
    // expanded over the largest stream a symbol can carry (8192 x 8 bits)
    nbits = std::max<uint64_t>(num_bits, 65536);
    uint8_t seq[127];
    uint8_t st = 0x5D;
    for (int i = 0; i < 127; i++) {
      const uint8_t fb = (st ^ (st >> 3)) & 1;
      seq[i] = fb;
      st = (uint8_t)((st >> 1) | (fb << 6));
    }
    h.assign((nbits + 7) / 8, 0);
    for (uint64_t t = 0; t < nbits; t++)
      if (seq[t % 127]) h[t / 8] |= (uint8_t)(0x80u >> (t % 8));
  } else if (mode == MB_SCR_GOLD) {
    if (num_ue == 0 || num_bits == 0) return MB_BAD_SHAPE;
    // TS 38.211 5.2.1, c_init(u) = c_init + u
    nbits = num_bits;
    row_bytes = (num_bits + 7) / 8;
    h.assign(row_bytes * num_ue, 0);
    const uint64_t Nc = 1600;
    for (uint32_t u = 0; u < num_ue; u++) {
      uint32_t x1 = 1, x2 = (c_init + u) & 0x7fffffffu;  // 31-bit registers
      for (uint64_t n = 0; n < Nc + num_bits; n++) {
        if (n >= Nc && ((x1 ^ x2) & 1u)) {
          const uint64_t t = n - Nc;
          h[u * row_bytes + t / 8] |= (uint8_t)(0x80u >> (t % 8));
        }
        const uint32_t f1 = ((x1 >> 3) ^ x1) & 1u;
        const uint32_t f2 = ((x2 >> 3) ^ (x2 >> 2) ^ (x2 >> 1) ^ x2) & 1u;
        x1 = (x1 >> 1) | (f1 << 30);
        x2 = (x2 >> 1) | (f2 << 30);
      }
    }
  } else {
    return MB_BAD_ARG;
  }
  mb_scrambler *s = new mb_scrambler();
  s->nbits = nbits;
  s->row_bytes = row_bytes;
  s->num_ue = num_ue;
  cudaError_t e = cudaMalloc(&s->bytes, h.size());
  if (e == cudaSuccess) e = cudaMemcpy(s->bytes, h.data(), h.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(s->bytes);
    delete s;
    return record_error(e);
  }
  *out = s;
  return MB_OK;
}

extern "C" mb_status mb_scrambler_destroy(mb_scrambler *s) {
  if (!s) return MB_BAD_ARG;
  cudaFree(s->bytes);
  delete s;
  return MB_OK;
}

mb_status mb::equalize_prepare(EqParams &p, const mb_c32 *W, const mb_c32 *y,
                               uint32_t K, uint32_t M, uint32_t S, uint32_t sg,
                               uint32_t n_sym, uint32_t Qm, uint64_t cb_size,
                               uint64_t cb_stride, uint64_t zeros,
                               uint32_t cb_blocks, uint16_t *llr,
                               uint8_t *hard, const mb_scrambler *scr) {
  if (!W || !y || !llr) return MB_BAD_ARG;
  if (K == 0 || K > 64 || M == 0 || S == 0 || sg == 0 || sg > 128) return MB_BAD_SHAPE;
  if (Qm != 2 && Qm != 4 && Qm != 6 && Qm != 8) return MB_BAD_ARG;
  if (cb_size == 0 || cb_blocks == 0 || cb_stride < zeros + cb_size) return MB_BAD_SHAPE;
  if (hard && (sg * Qm) % 8 != 0) return MB_UNSUPPORTED;
  p = EqParams{};
  p.W = reinterpret_cast<const float2 *>(W);
  p.y = reinterpret_cast<const float2 *>(y);
  p.llr = llr;
  p.hard = hard;
  p.K = K;
  p.M = M;
  p.S = S;
  p.sg = sg;
  p.n_sym = n_sym;
  p.Qm = Qm;
  p.cb_size = cb_size;
  p.cb_stride = cb_stride;
  p.zeros = zeros;
  p.cb_blocks = cb_blocks;
  p.row_len = cb_stride * cb_blocks;
  p.n_valid = std::min<uint64_t>((uint64_t)S * Qm, cb_size * cb_blocks);
  p.hrow = (p.n_valid + 7) / 8;
  p.hw_words = (sg * Qm / 8 + 3) / 4;
  if (p.row_len >= (1ull << 31) || (uint64_t)S * Qm >= (1ull << 31)) return MB_BAD_SHAPE;
  p.cb_size32 = (uint32_t)cb_size;
  p.cb_stride32 = (uint32_t)cb_stride;
  p.zeros32 = (uint32_t)zeros;
  p.row_len32 = (uint32_t)p.row_len;
  p.n_valid32 = (uint32_t)p.n_valid;
  if (scr && hard) {
    uint64_t nbits = 0;
    p.seqb = scrambler_bytes(scr, &nbits, &p.seq_row_bytes);
    if (p.seq_row_bytes && scr->num_ue < K) return MB_BAD_SHAPE;
    if (nbits < p.n_valid) return MB_BAD_SHAPE;  // sequence shorter than the stream
  }
  return MB_OK;
}

extern "C" mb_status mb_equalize(const mb_c32 *W, const mb_c32 *y, uint32_t K,
                                 uint32_t M, uint32_t S, uint32_t sg,
                                 uint32_t n_sym, uint32_t Qm, uint64_t cb_size,
                                 uint64_t cb_stride, uint64_t zeros,
                                 uint32_t cb_blocks, uint16_t *llr,
                                 uint8_t *hard, const mb_scrambler *scr,
                                 mb_c32 *x, void *stream) {
  EqParams p;
  mb_status s = equalize_prepare(p, W, y, K, M, S, sg, n_sym, Qm, cb_size,
                                 cb_stride, zeros, cb_blocks, llr, hard, scr);
  if (s != MB_OK) return s;
  p.x = reinterpret_cast<float2 *>(x);
  if (n_sym == 0) return MB_OK;
  return equalize_fp32(p, as_stream(stream));
}

extern "C" mb_status mb_precode(const mb_c32 *P, const mb_c32 *s, uint32_t M,
                                uint32_t K, uint32_t S, uint32_t sg,
                                uint32_t N, uint32_t start, uint32_t n_sym,
                                mb_c32 *out, void *stream) {
  if (!P || !s || !out) return MB_BAD_ARG;
  if (M == 0 || K == 0 || S == 0 || sg == 0 || sg > 128 || N < S) return MB_BAD_SHAPE;
  if (n_sym == 0) return MB_OK;
  return precode_fp32(reinterpret_cast<const float2 *>(P),
                      reinterpret_cast<const float2 *>(s),
                      reinterpret_cast<float2 *>(out), M, K, S, sg, N, start,
                      n_sym, as_stream(stream));
}

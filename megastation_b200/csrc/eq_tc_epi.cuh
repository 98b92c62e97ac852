// eq_tc_epi.cuh -- the tensor-core equalizer's epilogue, shared by the
// equalizer (eq_tc.cu) and the fused ZF + equalize kernel (zf_mixed.cu).
//
// D row i sits in TMEM lane i: every thread of the 256-thread epilogue owns
// one (symbol, subcarrier) column (lane 32 (warp % 4) + lane) and reads the
// complex x of all K users from its own lane, warps w and w + 4 taking
// alternate chunks of 8 users.  It demaps each x
// (modulation/demodulation.h:30-67 in FP16, demod2 on (Re, Im) pairs), stores
// the LLRs at the placement of equalize_kernel.cuh:272-287 (consecutive
// lanes write consecutive stretches of each user's LLR row), and gathers the
// hard bits of 8 neighbouring subcarriers with independent shuffles into
// whole descrambled bytes.  Everything the epilogue needs besides the
// accumulator, the descrambling bytes included, is computed in prepare(),
// which the caller runs before it waits for the MMAs, so its latency hides
// under them.
#pragma once
#include "demod.cuh"
#include "sgemv.cuh"
#include "tc.cuh"

namespace mb {

template <int MM, int QM>
struct EqTcEpilogue {
  static constexpr int kThreads = 256;
  static constexpr uint32_t NSUB = QM == 6 ? 2 : 8 / QM;
  static constexpr int kMaxCh = MM / 32;  // N <= MM columns: at most MM / 32 chunks per warp
  uint32_t quad, s, lg, base, nvm, sa, boff, gb, nch;
  bool valid, llr_on, pair, byte_on;
  uint32_t sqw[kMaxCh][2];

  // s_base: the group's first subcarrier; column c = l sg + sl < ncols is
  // (symbol l_off + l, subcarrier s_base + sl), its outputs at symbol
  // l0 + l_off + l; N = 2K padded to 16
  __device__ __forceinline__ void prepare(const EqParams &p, uint32_t s_base, uint32_t l_off, uint32_t ncols,
                                          uint32_t l0, uint32_t N, int warp, int lane) {
    quad = warp % 4;
    const uint32_t c = quad * 32 + lane;
    const uint32_t l = c / p.sg, sl = c % p.sg;
    s = s_base + sl;
    valid = c < ncols && s < p.S;
    lg = l0 + l_off + l;
    // LLR placement of subcarrier s (equalize_kernel.cuh:272-287), the same
    // for every user: code block cb, offset base in the (symbol, user) row
    const uint32_t t0 = s * QM;
    const uint32_t cb = t0 / p.cb_size32;
    base = cb * p.cb_stride32 + p.zeros32 + (t0 - cb * p.cb_size32);
    llr_on = valid && cb < p.cb_blocks;
    pair = base + QM <= p.row_len32 && ((p.row_len32 | base) & 1) == 0 &&
           (reinterpret_cast<uintptr_t>(p.llr) & 3) == 0;
    // hard bits: stream positions < n_valid only, first bit most significant
    nvm = 0;
#pragma unroll
    for (int qb = 0; qb < QM; qb++)
      if (t0 + qb < p.n_valid32) nvm |= 1u << (QM - 1 - qb);
    if (!valid) nvm = 0;
    // 8-lane groups hold 8 consecutive subcarriers of one symbol (sg % 8 ==
    // 0), i.e. QM whole bytes of the hard-bit row.  Lane gl < QM writes byte
    // gl; its 8 bits come from the NSUB subcarriers from sa on, fetched with
    // independent shuffles (a group cut short by S pads with zeros).
    const uint32_t gl = lane & 7;
    sa = gl < (uint32_t)QM ? 8 * gl / QM : 0;
    boff = 8 * gl - QM * sa;  // first bit of the byte within sa's bits
    const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
    const uint32_t nvalid = __popc((vmask >> (lane & ~7u)) & 0xFFu);
    gb = (s - gl) * QM / 8 + gl;
    byte_on = p.hard && gl < (nvalid * QM + 7) / 8 && gb * 8 < p.n_valid32;
    const uint32_t end = p.n_valid32 - gb * 8;
    const uint32_t seq_mask = byte_on && end < 8 ? (0xFF00u >> end) & 0xFFu : 0xFFu;
    nch = N / 16;
    // descrambling bytes of this warp's chunks ch = warp / 4 + 2 cc, four to
    // a word: byte j of chunk cc (user 8 ch + j) in sqw[cc][j / 4].  A
    // sequence shared by every user (seq_row_bytes 0: the reference's LFSR
    // scrambler) is one load per thread, else one per user.
    const bool shared_seq = p.seq_row_bytes == 0;
    const uint32_t sb = p.seqb && byte_on && shared_seq ? (uint32_t)__ldg(p.seqb + gb) & seq_mask : 0u;
#pragma unroll
    for (int cc = 0; cc < kMaxCh; cc++) {
      const uint32_t ch = warp / 4 + 2 * cc;
      const uint8_t *spu = p.seqb ? p.seqb + (uint64_t)(ch * 8) * p.seq_row_bytes + gb : nullptr;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        uint32_t w = 0;
#pragma unroll
        for (int b = 0; b < 4; b++) {
          const uint32_t j = 4 * h + b;
          if (spu && byte_on && ch < nch && ch * 8 + j < p.K)
            w |= (shared_seq ? sb : (uint32_t)__ldg(spu + j * p.seq_row_bytes) & seq_mask) << (8 * b);
        }
        sqw[cc][h] = w;
      }
    }
  }

  // the accumulator (tmem: lane 0, column 0 of D) has landed: demap and store
  __device__ __forceinline__ void run(const EqParams &p, uint32_t tmem, int warp, int lane) {
    // chunk loop not unrolled: the chunk's bytes are always in sqw[0], the
    // array rotating by one chunk per pass
#pragma unroll 1
    for (uint32_t ch = warp / 4; ch < nch; ch += kThreads / 128) {
      float v[16];
      tc::tmem_ld16(tmem + (quad * 32 << 16) + ch * 16, v);
      const uint64_t row = (uint64_t)lg * p.K + ch * 8;  // (symbol, first user of the chunk)
      __half *lpu = reinterpret_cast<__half *>(p.llr) + row * p.row_len + base;
      uint8_t *hpu = p.hard ? p.hard + row * p.hrow + gb : nullptr;
      float2 *xpu = p.x ? p.x + row * p.S + s : nullptr;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        if (ch * 8 + j >= p.K) break;
        const float2 x = make_float2(v[2 * j], v[2 * j + 1]);
        __half2 lv[QM / 2];  // (Re, Im) pairs, bit-identical to demod()
        demod2<QM>(x, lv);
        if (llr_on) {
          if (pair) {
#pragma unroll
            for (int h = 0; h < QM / 2; h++) reinterpret_cast<__half2 *>(lpu)[h] = lv[h];
          } else {
#pragma unroll
            for (int h = 0; h < QM / 2; h++) {
              if (base + 2 * h < p.row_len32) lpu[2 * h] = __low2half(lv[h]);
              if (base + 2 * h + 1 < p.row_len32) lpu[2 * h + 1] = __high2half(lv[h]);
            }
          }
        }
        if (hpu) {
          const uint32_t hb = hard2<QM>(lv) & nvm;
          uint32_t win = 0;
#pragma unroll
          for (uint32_t k = 0; k < NSUB; k++)
            win = (win << QM) | __shfl_sync(0xffffffffu, hb, (lane & ~7) + sa + k);
          const uint32_t sq = (sqw[0][j / 4] >> (8 * (j % 4))) & 0xFFu;
          if (byte_on) *hpu = (uint8_t)((win >> (NSUB * QM - boff - 8)) ^ sq);
          hpu += p.hrow;
        }
        if (xpu) {
          if (valid) *xpu = x;
          xpu += p.S;
        }
        lpu += p.row_len;
      }
#pragma unroll
      for (int cc = 0; cc + 1 < kMaxCh; cc++) {
        sqw[cc][0] = sqw[cc + 1][0];
        sqw[cc][1] = sqw[cc + 1][1];
      }
    }
  }
};

}  // namespace mb

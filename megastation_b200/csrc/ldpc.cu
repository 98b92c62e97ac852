// ldpc.cu -- NR LDPC encode and layered min-sum decode over a caller-supplied
// base graph (the reference's LDPCEncoder / LDPCDecoder, operators/ldpc/
// encoder.h:48-75 and decoder.h:28-87, take both from cuPHY).
//
// Graph structure (TS 38.212 5.3.2, both NR base graphs): block rows 0..3
// ("core") span the kb information columns and the four core parity columns
// kb..kb+3; every later row i has one more column, kb + i, as an identity
// block.  Block (i, j) with shift s is the Z x Z identity with its columns
// cyclically shifted right by s: row r has its one in column (r + s) mod Z.
// With the first mb rows of the graph (mb = parity nodes, the code rate):
//
// Encode (one CTA per code block): lambda_i = sum_j P^s_ij s_j over the core
// rows' information entries, the core parity p = B^-1 lambda (B the 4Z x 4Z
// core block, inverted over GF(2) on the host once, rows as bit words: one
// AND + popc per 32 bits), then each extension row's parity from the
// information and core parity columns.  Out: the (kb - 2 + mb) Z bits after
// the 2Z punctured systematic ones (cuPHY's puncture option, nrLDPCEncode).
//
// Decode (one CTA per pair of code blocks, thread z = check node z of the
// current layer, both blocks in the two halves of FP16 pairs): LLRs (FP16,
// positive = bit 0) into a __half2 array in shared memory with the graph's
// entries; the rows in order as layers; per check node and block:
// q_e = app - r_e (r_e the node's previous message to entry e, rebuilt from
// its compressed state), min1 (first index), min2 and the parity of the
// sign bits of q, then app = q_e + r'_e, r'_e = +-min(0.75 min, 256).  Rows
// of up to 20 entries keep q in registers (ldpc_node, variants for 4, 6, 10
// and 20 entries).  FP16 is the reference decoder's precision (cuPHY), and
// the pairs halve the instructions per block; channel LLRs clamped to
// +-1024 and messages to +-256 keep every value finite for up to 32 passes.
// Within a layer the Z check nodes touch disjoint variables (a circulant is
// a permutation), so a layer needs one barrier.  The compressed state (min1,
// min2, index, sign bits) per (layer, check node) lives in global memory,
// loaded two layers ahead.  Every step is one IEEE FP16 operation, so the
// results equal the float16 restatement bit for bit.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "ldpc.cuh"

namespace mb {
namespace {

constexpr uint32_t kMaxZ = 384;
constexpr uint32_t kMaxDeg = 27;   // sign bits per check node and block in its state
constexpr float kAlpha = 0.75f;    // min-sum normalisation
// FP16 range: channel LLRs are clamped to +-kLlrMax once and every message
// to +-kMsgMax; q and app stay exact sums (app = llr + the messages of the
// variable's rows, up to rounding), below 1024 + 46 * 256 = 12800 with at
// most 46 rows, and the rounding of two operations a row visit (at most 32
// each below 65504) adds at most 46 * 32 * 32 in kMaxIter passes: nothing
// overflows.  (Clamping q or app instead breaks that sum: a later row then
// removes more of its old message than app still holds, and signs flip.)
constexpr float kLlrMax = 1024.f;
constexpr float kMsgMax = 256.f;
constexpr uint32_t kMaxIter = 32;

__global__ void ldpc_encode_kernel(mb_ldpc h, const uint8_t *info, uint64_t info_stride, uint8_t *cw,
                                   uint64_t cw_stride) {
  extern __shared__ uint8_t enc_smem[];
  const uint32_t Z = h.Z, kb = h.kb, mb = h.mb, tid = threadIdx.x, nt = blockDim.x;
  uint8_t *x = enc_smem;                                      // [(kb + mb) Z] bits, one per byte
  uint32_t *lamw = reinterpret_cast<uint32_t *>(enc_smem + ((kb + mb) * Z + 3) / 4 * 4);  // [words]
  uint8_t *lam = reinterpret_cast<uint8_t *>(lamw + h.words);  // [4Z]
  const uint8_t *in = info + (uint64_t)blockIdx.x * info_stride;
  for (uint32_t v = tid; v < kb * Z; v += nt) x[v] = (in[v / 8] >> (7 - v % 8)) & 1u;
  __syncthreads();
  // lambda: the core rows over the information columns
  for (uint32_t t = tid; t < 4 * Z; t += nt) {
    const uint32_t i = t / Z, z = t % Z;
    uint32_t acc = 0;
    for (uint32_t e = h.row_ptr[i]; e < h.row_ptr[i + 1]; e++) {
      const uint32_t c = h.col[e];
      if (c < kb) acc ^= x[c * Z + (z + h.sh[e]) % Z];
    }
    lam[t] = (uint8_t)acc;
  }
  __syncthreads();
  for (uint32_t w = tid; w < h.words; w += nt) {
    uint32_t v = 0;
    for (uint32_t b = 0; b < 32 && 32 * w + b < 4 * Z; b++) v |= (uint32_t)lam[32 * w + b] << b;
    lamw[w] = v;
  }
  __syncthreads();
  // core parity p = B^-1 lambda
  for (uint32_t t = tid; t < 4 * Z; t += nt) {
    const uint32_t *row = h.binv + (uint64_t)t * h.words;
    uint32_t par = 0;
    for (uint32_t w = 0; w < h.words; w++) par ^= __popc(__ldg(row + w) & lamw[w]);
    x[kb * Z + t] = (uint8_t)(par & 1u);
  }
  __syncthreads();
  // extension rows: one parity block each, from the information and core
  // parity columns
  for (uint32_t t = tid; t < (mb - 4) * Z; t += nt) {
    const uint32_t i = 4 + t / Z, z = t % Z;
    uint32_t acc = 0;
    for (uint32_t e = h.row_ptr[i]; e < h.row_ptr[i + 1]; e++) {
      const uint32_t c = h.col[e];
      if (c < kb + 4) acc ^= x[c * Z + (z + h.sh[e]) % Z];
    }
    x[(kb + i) * Z + z] = (uint8_t)acc;
  }
  __syncthreads();
  // the encoded bits after the 2Z punctured ones, MSB first
  uint8_t *out = cw + (uint64_t)blockIdx.x * cw_stride;
  const uint32_t n_out = (kb - 2 + mb) * Z;
  for (uint32_t b = tid; b < (n_out + 7) / 8; b += nt) {
    uint32_t v = 0;
    for (uint32_t k = 0; k < 8; k++) {
      const uint32_t bit = 8 * b + k;
      v = (v << 1) | (bit < n_out ? x[2 * Z + bit] : 0u);
    }
    out[b] = (uint8_t)v;
  }
}

// Packed pairs: a CTA decodes two code blocks at once, lane 0 (the low half
// of every __half2) the pair's first block and lane 1 its second.
__device__ __forceinline__ uint32_t h2u(__half2 v) {
  uint32_t u;
  memcpy(&u, &v, 4);
  return u;
}
__device__ __forceinline__ __half2 u2h(uint32_t u) {
  __half2 v;
  memcpy(&v, &u, 4);
  return v;
}
__device__ __forceinline__ __half2 llr_clamp(__half2 v) {
  return __hmax2(__hmin2(v, __float2half2_rn(kLlrMax)), __float2half2_rn(-kLlrMax));
}

// A check node's state for the pair (one uint4 per layer and node):
//   x, y  min1, min2 (__half2: |q| of each block)
//   z     signs of q for entries 0..15: bit e block 0, bit 16 + e block 1
//   w     signs for entries 16..26 in bits 0..10 / 16..26, and the index of
//         min1 of block 0 in bits 11..15, of block 1 in bits 27..31
// The interleaving puts both blocks' bits for entry e at the same distance
// from bits 15 and 31, so one shift lines them up with the FP16 sign bits.
// The node's messages rebuilt from the state:
struct PairMsg {
  uint32_t m1, m2;    // min(0.75 min1, kMsgMax), min(0.75 min2, kMsgMax) (__half2 bits)
  uint32_t sgl, sgh;  // z / w with each block's sign parity applied: the message signs
  uint32_t ohl, ohh;  // min1's index one-hot in the same interleaved layout
};
__device__ __forceinline__ PairMsg pair_msg(const uint4 &st) {
  PairMsg m;
  const __half2 a = __float2half2_rn(kAlpha);  // 0.75, exact in FP16
  const __half2 cap = __float2half2_rn(kMsgMax);
  m.m1 = h2u(__hmin2(__hmul2(a, u2h(st.x)), cap));
  m.m2 = h2u(__hmin2(__hmul2(a, u2h(st.y)), cap));
  const uint32_t par0 = (__popc(st.z & 0xFFFFu) + __popc(st.w & 0x7FFu)) & 1u;
  const uint32_t par1 = (__popc(st.z >> 16) + __popc(st.w & 0x07FF0000u)) & 1u;
  const uint32_t flip = (par0 ? 0x0000FFFFu : 0u) | (par1 ? 0xFFFF0000u : 0u);
  m.sgl = st.z ^ flip;
  m.sgh = st.w ^ flip;  // only bits 0..10 and 16..26 are read
  const uint32_t p0 = (st.w >> 11) & 31u, p1 = st.w >> 27;
  m.ohl = (p0 < 16 ? 1u << p0 : 0u) | (p1 < 16 ? 1u << (16 + p1) : 0u);
  m.ohh = (p0 >= 16 ? 1u << (p0 - 16) : 0u) | (p1 >= 16 ? 1u << p1 : 0u);
  return m;
}
// the message to entry j: the (capped) 0.75 min2 at min1's index, 0.75
// min1 elsewhere, with the sign of q_j times the parity of all signs
__device__ __forceinline__ __half2 pair_r(const PairMsg &m, uint32_t j) {
  const uint32_t sh = j < 16 ? 15 - j : 31 - j;
  const uint32_t oh = (j < 16 ? m.ohl : m.ohh) << sh;
  const uint32_t sg = (j < 16 ? m.sgl : m.sgh) << sh;
  // bits 15 / 31 of oh spread over their halves (byte permute with the
  // selector's sign-replicate bit: bytes 1 and 3's top bits)
  uint32_t sel;
  asm("prmt.b32 %0, %1, %2, 0xBB99;" : "=r"(sel) : "r"(oh), "r"(0u));
  const uint32_t mag = (m.m1 & ~sel) | (m.m2 & sel);
  return u2h(mag ^ (sg & 0x80008000u));
}
// min tracking of entry j's |q| (blocks apart): the first index of min1 and
// the least of the others, as a sequential scan in entry order keeps them;
// the signs of q go into nl / nh
__device__ __forceinline__ void pair_track(__half2 q, uint32_t j, __half2 &min1, __half2 &min2, uint32_t &pos,
                                           uint32_t &nl, uint32_t &nh) {
  const uint32_t qb = h2u(q);
  const __half2 mag = u2h(qb & 0x7FFF7FFFu);
  const uint32_t lt = __hlt2_mask(mag, min1);
  pos = (pos & ~lt) | ((j * 0x00010001u) & lt);
  min2 = __hmin2(min2, __hmax2(min1, mag));
  min1 = __hmin2(min1, mag);
  if (j < 16)
    nl |= (qb >> (15 - j)) & (0x00010001u << j);
  else
    nh |= (qb >> (31 - j)) & (0x00010001u << (j - 16));
}
__device__ __forceinline__ uint4 pair_state(__half2 min1, __half2 min2, uint32_t pos, uint32_t nl, uint32_t nh,
                                            uint32_t deg) {
  if (deg == 1) min2 = min1;
  return make_uint4(h2u(min1), h2u(min2), nl, nh | ((pos & 31u) << 11) | ((pos >> 16) << 27));
}

// One check node's update for the pair over a row of at most D entries, all
// in registers: every app load issued before any store (a row holds one
// circulant per column block, so the node's D slots are distinct), then
// q_e = app - r_e (r_e rebuilt from the node's previous state) with the min
// tracking, then app = q_e + r'_e.  Returns the new state.
template <int D>
__device__ __forceinline__ uint4 ldpc_node(__half2 *app, const uint2 *ent, uint32_t deg, uint32_t tid, uint32_t Z,
                                           const uint4 &st) {
  // rows of more than 10 entries recompute the slot indices for the stores
  // rather than hold them (register pressure)
  constexpr bool kKeepIdx = D <= 10;
  auto slot = [&](int j) {
    const uint2 en = ent[j];
    return en.x + tid - (tid >= en.y ? Z : 0u);
  };
  const PairMsg mo = pair_msg(st);
  uint32_t idx[kKeepIdx ? D : 1];
  __half2 q[D];
#pragma unroll
  for (int j = 0; j < D; j++) {
    if (j < (int)deg) {
      const uint32_t ix = slot(j);
      if constexpr (kKeepIdx) idx[j] = ix;
      q[j] = app[ix];
    }
  }
  __half2 min1 = __float2half2_rn(INFINITY), min2 = min1;
  uint32_t pos = 0, nl = 0, nh = 0;
#pragma unroll
  for (int j = 0; j < D; j++) {
    if (j < (int)deg) {
      q[j] = __hsub2(q[j], pair_r(mo, j));
      pair_track(q[j], j, min1, min2, pos, nl, nh);
    }
  }
  const uint4 ns = pair_state(min1, min2, pos, nl, nh, deg);
  const PairMsg mn = pair_msg(ns);
#pragma unroll
  for (int j = 0; j < D; j++) {
    if (j < (int)deg) {
      uint32_t ix;
      if constexpr (kKeepIdx) ix = idx[j];
      else ix = slot(j);
      app[ix] = __hadd2(q[j], pair_r(mn, j));
    }
  }
  return ns;
}

// The same update for rows of any degree (up to kMaxDeg): q_e is stored in
// place of app between the two passes.
__device__ __forceinline__ uint4 ldpc_node_any(__half2 *app, const uint2 *ent, uint32_t deg, uint32_t tid,
                                               uint32_t Z, const uint4 &st) {
  const PairMsg mo = pair_msg(st);
  __half2 min1 = __float2half2_rn(INFINITY), min2 = min1;
  uint32_t pos = 0, nl = 0, nh = 0;
  for (uint32_t e = 0; e < deg; e++) {
    const uint2 en = ent[e];
    __half2 *a = app + en.x + tid - (tid >= en.y ? Z : 0u);
    const __half2 qe = __hsub2(*a, pair_r(mo, e));
    *a = qe;
    pair_track(qe, e, min1, min2, pos, nl, nh);
  }
  const uint4 ns = pair_state(min1, min2, pos, nl, nh, deg);
  const PairMsg mn = pair_msg(ns);
  for (uint32_t e = 0; e < deg; e++) {
    const uint2 en = ent[e];
    __half2 *a = app + en.x + tid - (tid >= en.y ? Z : 0u);
    *a = __hadd2(*a, pair_r(mn, e));
  }
  return ns;
}

// CTA p decodes code blocks b0 + 2p and b0 + 2p + 1 (the second only when
// 2p + 1 < nb; otherwise its lane repeats the first and is not written)
__global__ void __launch_bounds__(kMaxZ, 2) ldpc_decode_kernel(mb_ldpc h, const __half *llr, uint64_t llr_stride,
                                                               uint8_t *out, uint64_t out_stride, uint32_t max_iter,
                                                               uint32_t b0, uint32_t nb) {
  // the pair's a-posteriori LLRs [(kb + mb) Z] (__half2), then the entries
  // {col * Z, shift} and the row pointers
  extern __shared__ uint32_t dec_smem[];
  const uint32_t Z = h.Z, kb = h.kb, mb = h.mb, N = (kb + mb) * Z, tid = threadIdx.x, nt = blockDim.x;
  __half2 *app = reinterpret_cast<__half2 *>(dec_smem);
  uint2 *ent = reinterpret_cast<uint2 *>(dec_smem + (N + 1) / 2 * 2);  // [nnz]
  uint32_t *r_ptr = reinterpret_cast<uint32_t *>(ent + h.nnz);         // [mb + 1]
  const uint32_t cb = b0 + 2 * blockIdx.x;
  const bool two = 2 * blockIdx.x + 1 < nb;
  const __half *in0 = llr + (uint64_t)cb * llr_stride;
  const __half *in1 = two ? in0 + llr_stride : in0;
  for (uint32_t v = tid; v < N; v += nt) app[v] = llr_clamp(__halves2half2(in0[v], in1[v]));
  // entry e as {col * Z + shift, Z - shift}: check node z meets variable
  // col * Z + (z + shift) mod Z, i.e. x + z, less Z once z >= y
  for (uint32_t e = tid; e < h.nnz; e += nt) ent[e] = make_uint2((uint32_t)h.col[e] * Z + h.sh[e], Z - h.sh[e]);
  for (uint32_t i = tid; i <= mb; i += nt) r_ptr[i] = h.row_ptr[i];
  __syncthreads();
  // Thread z only ever reads and writes check node z's state, so its loads
  // run two layers ahead of their use (a row's state is rewritten mb >= 4
  // layers before it is read again); the first pass starts from zero
  // messages without reading.
  uint4 *state = h.state + (uint64_t)blockIdx.x * mb * Z;
  // the state of row r in pass it: none in the first pass nor past the last
  auto load_state = [&](uint32_t it, uint32_t r) {
    return (it == 0 || it >= max_iter || tid >= Z) ? make_uint4(0u, 0u, 0u, 0u) : state[r * Z + tid];
  };
  uint4 st_a = load_state(0, 0), st_b = load_state(0, 1);
  for (uint32_t it = 0; it < max_iter; it++) {
    for (uint32_t i = 0; i < mb; i++) {
      const uint4 st = st_a;
      st_a = st_b;
      // row i + 2, in this pass or the next (mb >= 4)
      st_b = i + 2 < mb ? load_state(it, i + 2) : load_state(it + 1, i + 2 - mb);
      if (tid < Z) {
        const uint32_t e0 = r_ptr[i], deg = r_ptr[i + 1] - e0;
        // every thread of the layer takes the same branch
        uint4 ns;
        if (deg <= 4)
          ns = ldpc_node<4>(app, ent + e0, deg, tid, Z, st);
        else if (deg <= 6)
          ns = ldpc_node<6>(app, ent + e0, deg, tid, Z, st);
        else if (deg <= 10)
          ns = ldpc_node<10>(app, ent + e0, deg, tid, Z, st);
        else if (deg <= 20)
          ns = ldpc_node<20>(app, ent + e0, deg, tid, Z, st);
        else
          ns = ldpc_node_any(app, ent + e0, deg, tid, Z, st);
        state[i * Z + tid] = ns;
      }
      __syncthreads();
    }
  }
  // hard decisions of the information bits, MSB first, both blocks
  uint8_t *o0 = out + (uint64_t)cb * out_stride, *o1 = o0 + out_stride;
  for (uint32_t b = tid; b < (kb * Z + 7) / 8; b += nt) {
    uint32_t v0 = 0, v1 = 0;
    for (uint32_t k = 0; k < 8; k++) {
      const uint32_t bit = 8 * b + k;
      const uint32_t ng = bit < kb * Z ? __hlt2_mask(app[bit], __float2half2_rn(0.f)) : 0u;
      v0 = (v0 << 1) | (ng & 1u);
      v1 = (v1 << 1) | (ng >> 31);
    }
    o0[b] = (uint8_t)v0;
    if (two) o1[b] = (uint8_t)v1;
  }
}

// B^-1 over GF(2) of the 4Z x 4Z core block, rows as 64-bit words; false
// when B is singular
bool core_inverse(const std::vector<std::vector<std::pair<uint32_t, uint32_t>>> &rows, uint32_t kb, uint32_t Z,
                  std::vector<uint64_t> &inv, uint32_t &w64) {
  const uint32_t n = 4 * Z;
  w64 = (n + 63) / 64;
  std::vector<uint64_t> a((size_t)n * w64, 0), b((size_t)n * w64, 0);
  for (uint32_t i = 0; i < 4; i++)
    for (auto &cs : rows[i])
      if (cs.first >= kb && cs.first < kb + 4)
        for (uint32_t r = 0; r < Z; r++) {
          const uint32_t c = (cs.first - kb) * Z + (r + cs.second) % Z;
          a[(size_t)(i * Z + r) * w64 + c / 64] ^= 1ull << (c % 64);
        }
  for (uint32_t r = 0; r < n; r++) b[(size_t)r * w64 + r / 64] = 1ull << (r % 64);
  for (uint32_t c = 0; c < n; c++) {
    uint32_t p = c;
    while (p < n && !((a[(size_t)p * w64 + c / 64] >> (c % 64)) & 1ull)) p++;
    if (p == n) return false;
    if (p != c)
      for (uint32_t w = 0; w < w64; w++) {
        std::swap(a[(size_t)p * w64 + w], a[(size_t)c * w64 + w]);
        std::swap(b[(size_t)p * w64 + w], b[(size_t)c * w64 + w]);
      }
    for (uint32_t r = 0; r < n; r++)
      if (r != c && ((a[(size_t)r * w64 + c / 64] >> (c % 64)) & 1ull))
        for (uint32_t w = 0; w < w64; w++) {
          a[(size_t)r * w64 + w] ^= a[(size_t)c * w64 + w];
          b[(size_t)r * w64 + w] ^= b[(size_t)c * w64 + w];
        }
  }
  inv.swap(b);
  return true;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" mb_status mb_ldpc_destroy(mb_ldpc *h) {
  if (!h) return MB_BAD_ARG;
  cudaFree(h->row_ptr);
  cudaFree(h->col);
  cudaFree(h->sh);
  cudaFree(h->binv);
  cudaFree(h->state);
  delete h;
  return MB_OK;
}

extern "C" mb_status mb_ldpc_create(const mb_ldpc_graph *g, uint32_t Z, uint32_t parity_nodes,
                                    uint32_t max_batch, mb_ldpc **out) {
  if (!g || !out || !g->row || !g->col || !g->shift) return MB_BAD_ARG;
  *out = nullptr;
  const uint32_t kb = g->kb, mbr = parity_nodes;
  if (Z == 0 || Z > kMaxZ || kb < 3 || mbr < 4 || mbr > g->rows || max_batch == 0) return MB_BAD_SHAPE;
  // rows < mb, entries by (row, col), shifts reduced mod Z (TS 38.212:
  // P = V mod Z); the NR block structure checked
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> rows(mbr);
  for (uint32_t k = 0; k < g->nnz; k++) {
    const uint32_t r = g->row[k], c = g->col[k];
    if (r >= g->rows || c >= kb + g->rows) return MB_BAD_ARG;
    if (r >= mbr) continue;
    const bool ext = c >= kb + 4;
    if (ext && (r < 4 || c != kb + r || g->shift[k] % Z != 0)) return MB_BAD_ARG;
    rows[r].push_back({c, (uint32_t)(g->shift[k] % Z)});
  }
  uint32_t nnz = 0;
  std::vector<uint32_t> row_ptr(mbr + 1, 0);
  std::vector<uint16_t> col, sh;
  for (uint32_t r = 0; r < mbr; r++) {
    std::sort(rows[r].begin(), rows[r].end());
    for (size_t k = 1; k < rows[r].size(); k++)
      if (rows[r][k].first == rows[r][k - 1].first) return MB_BAD_ARG;  // one circulant per block
    if (rows[r].empty() || rows[r].size() > kMaxDeg) return MB_BAD_ARG;
    if (r >= 4) {
      bool own = false;
      for (auto &cs : rows[r]) own |= cs.first == kb + r;
      if (!own) return MB_BAD_ARG;
    }
    for (auto &cs : rows[r]) {
      col.push_back((uint16_t)cs.first);
      sh.push_back((uint16_t)cs.second);
    }
    nnz += (uint32_t)rows[r].size();
    row_ptr[r + 1] = nnz;
  }
  std::vector<uint64_t> inv64;
  uint32_t w64 = 0;
  if (!core_inverse(rows, kb, Z, inv64, w64)) return MB_BAD_ARG;
  const uint32_t n = 4 * Z, words = (n + 31) / 32;
  std::vector<uint32_t> inv32((size_t)n * words);
  for (uint32_t r = 0; r < n; r++)
    for (uint32_t w = 0; w < words; w++)
      inv32[(size_t)r * words + w] = (uint32_t)(inv64[(size_t)r * w64 + w / 2] >> (32 * (w % 2)));
  mb_ldpc *h = new mb_ldpc();
  h->kb = kb;
  h->Z = Z;
  h->mb = mbr;
  h->nnz = nnz;
  h->max_batch = max_batch;
  h->words = words;
  MB_CUDA_TRY(cudaGetDevice(&h->dev));
  mb_status st = MB_OK;
  auto alloc_copy = [&](void **p, const void *src, size_t bytes) {
    if (st != MB_OK) return;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess && src) e = cudaMemcpy(*p, src, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) st = record_error(e);
  };
  alloc_copy((void **)&h->row_ptr, row_ptr.data(), row_ptr.size() * sizeof(uint32_t));
  alloc_copy((void **)&h->col, col.data(), col.size() * sizeof(uint16_t));
  alloc_copy((void **)&h->sh, sh.data(), sh.size() * sizeof(uint16_t));
  alloc_copy((void **)&h->binv, inv32.data(), inv32.size() * sizeof(uint32_t));
  alloc_copy((void **)&h->state, nullptr, (size_t)((max_batch + 1) / 2) * mbr * Z * sizeof(uint4));
  if (st != MB_OK) {
    mb_ldpc_destroy(h);
    return st;
  }
  *out = h;
  return MB_OK;
}

extern "C" mb_status mb_ldpc_encode(mb_ldpc *h, const uint8_t *info, uint64_t info_stride, uint8_t *cw,
                                    uint64_t cw_stride, uint32_t batch, void *stream) {
  if (!h || !info || !cw) return MB_BAD_ARG;
  if (info_stride < ((uint64_t)h->kb * h->Z + 7) / 8 ||
      cw_stride < ((uint64_t)(h->kb - 2 + h->mb) * h->Z + 7) / 8)
    return MB_BAD_SHAPE;
  if (batch == 0) return MB_OK;
  const size_t smem = ((size_t)(h->kb + h->mb) * h->Z + 3) / 4 * 4 + h->words * 4 + 4 * h->Z;
  ldpc_encode_kernel<<<batch, 256, smem, as_stream(stream)>>>(*h, info, info_stride, cw, cw_stride);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" mb_status mb_ldpc_decode(mb_ldpc *h, const uint16_t *llr, uint64_t llr_stride, uint8_t *out,
                                    uint64_t out_stride, uint32_t batch, uint32_t max_iter, void *stream) {
  if (!h || !llr || !out) return MB_BAD_ARG;
  if (llr_stride < (uint64_t)(h->kb + h->mb) * h->Z || out_stride < ((uint64_t)h->kb * h->Z + 7) / 8)
    return MB_BAD_SHAPE;
  if (max_iter > kMaxIter) return MB_BAD_ARG;  // the FP16 range argument above
  if (batch == 0) return MB_OK;
  const size_t smem = ((size_t)(h->kb + h->mb) * h->Z + 1) / 2 * 8 + 8 * (size_t)h->nnz + 4 * ((size_t)h->mb + 1);
  static_assert(kMaxZ <= 1024, "one thread per check node");
  int maxs = 0;
  MB_CUDA_TRY(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->dev));
  if (smem > (size_t)maxs) return MB_UNSUPPORTED;
  MB_CUDA_TRY(cudaFuncSetAttribute(ldpc_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const uint32_t threads = (h->Z + 31) / 32 * 32;
  // at most max_batch code blocks at a time, in pairs: each pair keeps its
  // check-node state
  for (uint32_t b0 = 0; b0 < batch; b0 += h->max_batch) {
    const uint32_t nb = std::min(h->max_batch, batch - b0);
    ldpc_decode_kernel<<<(nb + 1) / 2, threads, smem, as_stream(stream)>>>(
        *h, reinterpret_cast<const __half *>(llr), llr_stride, out, out_stride, max_iter, b0, nb);
    MB_LAUNCH_CHECK();
  }
  return MB_OK;
}

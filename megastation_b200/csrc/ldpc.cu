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
// Decode (one CTA per code block, thread z = check node z of the current
// layer): LLRs (FP16, positive = bit 0) into a float array in shared memory
// with the graph's entries; the rows in order as layers; per check node:
// q_e = app - r_e (r_e the node's previous message to entry e, rebuilt from
// its compressed state), min1 (first index), min2 and the sign parity of
// q < 0, then app = q_e + r'_e, r'_e = +-(0.75 min); rows of up to 20
// entries keep q in registers (ldpc_node).  Within a layer
// the Z check nodes touch disjoint variables (a circulant is a permutation),
// so a layer needs one barrier.  The compressed state (min1, min2, index,
// sign bits) per (layer, check node) lives in global memory, loaded two
// layers ahead.  Every
// floating-point step is an explicitly rounded single operation, so the
// results equal the float32 restatement bit for bit.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "ldpc.cuh"

namespace mb {
namespace {

constexpr uint32_t kMaxZ = 384;
constexpr uint32_t kMaxDeg = 32;   // sign bits per check node state
constexpr float kAlpha = 0.75f;    // min-sum normalisation

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

// One check node's update over a row of at most D entries, all in registers:
// every app load issued before any store (a row holds one circulant per
// column block, so the node's D slots are distinct), then q_e = app - r_e
// (r_e rebuilt from the node's previous state st) with min1 (first index),
// min2 and the signs of q, then app = q_e + r'_e.  Returns the new state.
template <int D>
__device__ __forceinline__ uint4 ldpc_node(float *app, const uint2 *ent, uint32_t deg, uint32_t tid, uint32_t Z,
                                           const uint4 &st) {
  uint32_t idx[D];
  float q[D];
#pragma unroll
  for (int j = 0; j < D; j++) {
    if (j < (int)deg) {
      const uint2 en = ent[j];
      uint32_t z = tid + en.y;
      if (z >= Z) z -= Z;
      idx[j] = en.x + z;
    }
  }
#pragma unroll
  for (int j = 0; j < D; j++)
    if (j < (int)deg) q[j] = app[idx[j]];
  const float m1o = __fmul_rn(kAlpha, __uint_as_float(st.x));
  const float m2o = __fmul_rn(kAlpha, __uint_as_float(st.y));
  const uint32_t sgn_o = st.w ^ ((__popc(st.w) & 1u) ? ~0u : 0u);
  float min1 = INFINITY, min2 = INFINITY;
  uint32_t pos = 0, neg = 0;
#pragma unroll
  for (int j = 0; j < D; j++) {
    if (j < (int)deg) {
      const float r = __uint_as_float(__float_as_uint((uint32_t)j == st.z ? m2o : m1o) ^ (((sgn_o >> j) & 1u) << 31));
      q[j] = __fsub_rn(q[j], r);
      const float aq = fabsf(q[j]);
      neg |= (q[j] < 0.f ? 1u : 0u) << j;
      if (aq < min1) {
        min2 = min1;
        min1 = aq;
        pos = j;
      } else if (aq < min2) {
        min2 = aq;
      }
    }
  }
  if (deg == 1) min2 = min1;
  const float m1 = __fmul_rn(kAlpha, min1), m2 = __fmul_rn(kAlpha, min2);
  const uint32_t sgn = neg ^ ((__popc(neg) & 1u) ? ~0u : 0u);
#pragma unroll
  for (int j = 0; j < D; j++)
    if (j < (int)deg)
      app[idx[j]] = __fadd_rn(q[j], __uint_as_float(__float_as_uint((uint32_t)j == pos ? m2 : m1) ^ (((sgn >> j) & 1u) << 31)));
  return make_uint4(__float_as_uint(min1), __float_as_uint(min2), pos, neg);
}

// The same update for rows of any degree (up to 32): q_e is stored in place
// of app between the two passes.
__device__ __forceinline__ uint4 ldpc_node_any(float *app, const uint2 *ent, uint32_t deg, uint32_t tid,
                                               uint32_t Z, const uint4 &st) {
  const float m1o = __fmul_rn(kAlpha, __uint_as_float(st.x));
  const float m2o = __fmul_rn(kAlpha, __uint_as_float(st.y));
  const uint32_t sgn_o = st.w ^ ((__popc(st.w) & 1u) ? ~0u : 0u);
  float min1 = INFINITY, min2 = INFINITY;
  uint32_t pos = 0, neg = 0;
  for (uint32_t e = 0; e < deg; e++) {
    const uint2 en = ent[e];
    uint32_t z = tid + en.y;
    if (z >= Z) z -= Z;
    float *a = app + en.x + z;
    const float r = __uint_as_float(__float_as_uint(e == st.z ? m2o : m1o) ^ (((sgn_o >> e) & 1u) << 31));
    const float qe = __fsub_rn(*a, r);
    *a = qe;
    const float aq = fabsf(qe);
    neg |= (qe < 0.f ? 1u : 0u) << e;
    if (aq < min1) {
      min2 = min1;
      min1 = aq;
      pos = e;
    } else if (aq < min2) {
      min2 = aq;
    }
  }
  if (deg == 1) min2 = min1;
  const float m1 = __fmul_rn(kAlpha, min1), m2 = __fmul_rn(kAlpha, min2);
  const uint32_t sgn = neg ^ ((__popc(neg) & 1u) ? ~0u : 0u);
  for (uint32_t e = 0; e < deg; e++) {
    const uint2 en = ent[e];
    uint32_t z = tid + en.y;
    if (z >= Z) z -= Z;
    float *a = app + en.x + z;
    *a = __fadd_rn(*a, __uint_as_float(__float_as_uint(e == pos ? m2 : m1) ^ (((sgn >> e) & 1u) << 31)));
  }
  return make_uint4(__float_as_uint(min1), __float_as_uint(min2), pos, neg);
}

__global__ void __launch_bounds__(kMaxZ, 2) ldpc_decode_kernel(mb_ldpc h, const __half *llr, uint64_t llr_stride,
                                                            uint8_t *out, uint64_t out_stride, uint32_t max_iter,
                                                            uint32_t b0) {
  extern __shared__ float app[];  // [(kb + mb) Z], then the entries {col * Z, shift} and the row pointers
  const uint32_t Z = h.Z, kb = h.kb, mb = h.mb, N = (kb + mb) * Z, tid = threadIdx.x, nt = blockDim.x;
  uint2 *ent = reinterpret_cast<uint2 *>(app + (N + 1) / 2 * 2);  // [nnz]
  uint32_t *r_ptr = reinterpret_cast<uint32_t *>(ent + h.nnz);    // [mb + 1]
  const uint32_t cb = b0 + blockIdx.x;
  const __half *in = llr + (uint64_t)cb * llr_stride;
  for (uint32_t v = tid; v < N; v += nt) app[v] = __half2float(in[v]);
  for (uint32_t e = tid; e < h.nnz; e += nt) ent[e] = make_uint2((uint32_t)h.col[e] * Z, h.sh[e]);
  for (uint32_t i = tid; i <= mb; i += nt) r_ptr[i] = h.row_ptr[i];
  __syncthreads();
  // Thread z only ever reads and writes check node z's state, so its loads
  // run two layers ahead of their use (a row's state is rewritten mb >= 4
  // layers before it is read again); the first pass starts from zero
  // messages without reading.
  uint4 *state = h.state + (uint64_t)blockIdx.x * mb * Z;
  const uint32_t layers = max_iter * mb;
  auto load_state = [&](uint32_t L) {
    return (L < mb || L >= layers || tid >= Z) ? make_uint4(0u, 0u, 0u, 0u) : state[(L % mb) * Z + tid];
  };
  uint4 st_a = load_state(0), st_b = load_state(1);
  for (uint32_t it = 0; it < max_iter; it++) {
    for (uint32_t i = 0; i < mb; i++) {
      const uint32_t L = it * mb + i;
      const uint4 st = st_a;
      st_a = st_b;
      st_b = load_state(L + 2);
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
  // hard decisions of the information bits, MSB first
  uint8_t *o = out + (uint64_t)cb * out_stride;
  for (uint32_t b = tid; b < (kb * Z + 7) / 8; b += nt) {
    uint32_t v = 0;
    for (uint32_t k = 0; k < 8; k++) {
      const uint32_t bit = 8 * b + k;
      v = (v << 1) | (bit < kb * Z && app[bit] < 0.f ? 1u : 0u);
    }
    o[b] = (uint8_t)v;
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
  alloc_copy((void **)&h->state, nullptr, (size_t)max_batch * mbr * Z * sizeof(uint4));
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
  if (batch == 0) return MB_OK;
  const size_t smem = ((size_t)(h->kb + h->mb) * h->Z + 1) / 2 * 8 + 8 * (size_t)h->nnz + 4 * ((size_t)h->mb + 1);
  static_assert(kMaxZ <= 1024, "one thread per check node");
  int maxs = 0;
  MB_CUDA_TRY(cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->dev));
  if (smem > (size_t)maxs) return MB_UNSUPPORTED;
  MB_CUDA_TRY(cudaFuncSetAttribute(ldpc_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const uint32_t threads = (h->Z + 31) / 32 * 32;
  // at most max_batch code blocks at a time: each keeps its check-node state
  for (uint32_t b0 = 0; b0 < batch; b0 += h->max_batch) {
    const uint32_t nb = std::min(h->max_batch, batch - b0);
    ldpc_decode_kernel<<<nb, threads, smem, as_stream(stream)>>>(*h, reinterpret_cast<const __half *>(llr),
                                                                 llr_stride, out, out_stride, max_iter, b0);
    MB_LAUNCH_CHECK();
  }
  return MB_OK;
}

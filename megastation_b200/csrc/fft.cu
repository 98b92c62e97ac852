// fft.cu -- fused OFDM FFT operators for sm_100a.
//
// Replaces the reference's three-launch pipelines (load kernel -> cuFFT ->
// store kernel, fft/fft_op.cu:135-174) with ONE kernel per call: the first
// radix pass loads and converts the IQ samples straight from HBM
// (fft_callback.cuh:20-41), the middle passes run in shared memory, and the
// last pass applies the operator's epilogue straight from registers: the
// FFT-shift gather of the uplink (fft_callback.cuh:43-74), the LS pilot
// estimate scattered into the CSI layout (fft_callback.cuh:76-108), or the
// IFFT quantiser (ifft_callback.cuh:21-59).  The samples therefore cross
// HBM once in and once out.
//
// Algorithm: Stockham autosort FFT (Govindaraju et al., "High performance
// discrete Fourier transforms on graphics processors", SC'08), radix 16
// passes plus one radix 2/4/8 pass for N = 2^n, n in [4, 13].  Each thread
// owns 16 complex values; a row of N points uses N/16 threads, and a CTA
// holds max(1, 256/(N/16)) rows.  Twiddles come from per-device tables
// computed in double at init and laid out per pass as [r][k], so a warp's
// twiddle loads are coalesced; a radix-16 pass loads the entries of r = 1
// and 4 and forms the other powers by at most three complex products.
#include <cuda_bf16.h>

#include <atomic>

#include "common.cuh"
#include "fft.cuh"

namespace mb {

enum FftMode { kUplink = 0, kPilot = 1, kIfft = 2, kUplinkLP = 3 };

struct FftParams {
  const void *in;
  void *out;
  const float2 *tw;      // Stockham twiddle table of N
  const float2 *pilot;   // pilot sign (kPilot), device
  uint64_t rows;         // n_sym * M
  uint32_t M, S, start, K, sg, ue_start;
  uint32_t S_pad;        // kUplinkLP row pitch (elements)
  uint32_t tail_rem;     // kPilot: S % sg when the short last group is filled (0: off)
  int in_dtype, out_dtype;
};

// ---- in-register DFTs (natural order in and out) ------------------------
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {  // a * W4 (= -i fwd)
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2 &x0, float2 &x1, float2 &x2,
                                     float2 &x3) {
  float2 a0 = cadd(x0, x2), a1 = csub(x0, x2);
  float2 a2 = cadd(x1, x3), a3 = mul_mi<INV>(csub(x1, x3));
  x0 = cadd(a0, a2);
  x2 = csub(a0, a2);
  x1 = cadd(a1, a3);
  x3 = csub(a1, a3);
}

// W16^m, m in [0, 15] (constant-folded once m is a compile-time constant)
template <bool INV>
__device__ __forceinline__ float2 w16(int m) {
  const float c1 = 0.92387953251128674f, s1 = 0.38268343236508978f,
              c2 = 0.70710678118654752f;
  float2 w;
  switch (m & 15) {
    case 0: w = make_float2(1.f, 0.f); break;
    case 1: w = make_float2(c1, -s1); break;
    case 2: w = make_float2(c2, -c2); break;
    case 3: w = make_float2(s1, -c1); break;
    case 4: w = make_float2(0.f, -1.f); break;
    case 5: w = make_float2(-s1, -c1); break;
    case 6: w = make_float2(-c2, -c2); break;
    case 7: w = make_float2(-c1, -s1); break;
    case 8: w = make_float2(-1.f, 0.f); break;
    case 9: w = make_float2(-c1, s1); break;
    case 10: w = make_float2(-c2, c2); break;
    case 11: w = make_float2(-s1, c1); break;
    case 12: w = make_float2(0.f, 1.f); break;
    case 13: w = make_float2(s1, c1); break;
    case 14: w = make_float2(c2, c2); break;
    default: w = make_float2(c1, s1); break;
  }
  if (INV) w.y = -w.y;
  return w;
}

template <bool INV>
__device__ __forceinline__ float2 mul_w16(float2 a, int m) {
  m &= 15;
  if (m == 0) return a;
  if (m == 4) return mul_mi<INV>(a);
  if (m == 8) return make_float2(-a.x, -a.y);
  if (m == 12) return mul_mi<!INV>(a);
  return cmul(a, w16<INV>(m));
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2 *v) {
  if constexpr (R == 2) {
    float2 a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  } else if constexpr (R == 4) {
    dft4<INV>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    // n = 2 n1 + n2, k = k1 + 4 k2
    float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    dft4<INV>(e[0], e[1], e[2], e[3]);
    dft4<INV>(o[0], o[1], o[2], o[3]);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
      float2 t = mul_w16<INV>(o[k1], 2 * k1);
      v[k1] = cadd(e[k1], t);
      v[k1 + 4] = csub(e[k1], t);
    }
  } else {
    static_assert(R == 16, "radix");
    // n = 4 n1 + n2, k = k1 + 4 k2
    float2 a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
      a[n2][0] = v[n2];
      a[n2][1] = v[4 + n2];
      a[n2][2] = v[8 + n2];
      a[n2][3] = v[12 + n2];
      dft4<INV>(a[n2][0], a[n2][1], a[n2][2], a[n2][3]);
#pragma unroll
      for (int k1 = 0; k1 < 4; k1++) a[n2][k1] = mul_w16<INV>(a[n2][k1], n2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
      float2 b0 = a[0][k1], b1 = a[1][k1], b2 = a[2][k1], b3 = a[3][k1];
      dft4<INV>(b0, b1, b2, b3);
      v[k1] = b0;
      v[k1 + 4] = b1;
      v[k1 + 8] = b2;
      v[k1 + 12] = b3;
    }
  }
}

// ---- plan -------------------------------------------------------------
template <int LOGN>
struct Plan {
  static constexpr int N = 1 << LOGN;
  static constexpr int T = N / 16;                 // threads per row
  static constexpr int ROWS = T >= 256 ? 1 : 256 / T;
  static constexpr int THREADS = T * ROWS;
  // resident CTAs per SM the register budget must allow (64 regs/thread at
  // 256 threads x 4): keeps 32 warps per SM in flight for the HBM stream
  static constexpr int MIN_BLOCKS = THREADS >= 512 ? 2 : 4;
  static constexpr int P16 = LOGN / 4;             // radix-16 passes
  static constexpr int RLAST = 1 << (LOGN % 4);    // trailing radix (1: none)
  static constexpr int PASSES = P16 + (RLAST > 1 ? 1 : 0);
  static constexpr int PADN = N + N / 16;          // padded smem row
  static __host__ __device__ __forceinline__ constexpr int radix(int p) {
    return p < P16 ? 16 : RLAST;
  }
  // product of the radices before pass p
  static __host__ __device__ __forceinline__ constexpr int ns(int p) {
    return p == 0 ? 1 : ns(p - 1) * radix(p - 1);
  }
  // offset of pass p's [r][k] block in the twiddle table
  static __host__ __device__ __forceinline__ constexpr int tw_off(int p) {
    return p <= 1 ? 0 : tw_off(p - 1) + radix(p - 1) * ns(p - 1);
  }
};

__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

// ---- loads and epilogues ------------------------------------------------
__device__ __forceinline__ float2 load_iq(const FftParams &p, uint64_t e) {
  switch (p.in_dtype) {
    case MB_IQ_C32:
      return __ldg(reinterpret_cast<const float2 *>(p.in) + e);
    case MB_IQ_I16: {
      short2 s = __ldg(reinterpret_cast<const short2 *>(p.in) + e);
      return make_float2((float)s.x / 32768.f, (float)s.y / 32768.f);
    }
    case MB_IQ_I8: {
      char2 s = reinterpret_cast<const char2 *>(p.in)[e];
      return make_float2((float)s.x / 128.f, (float)s.y / 128.f);
    }
    default: {
      __half2 h = reinterpret_cast<const __half2 *>(p.in)[e];
      return __half22float2(h);
    }
  }
}

// Per-row output context, computed once per thread so that the per-element
// epilogue needs no 64-bit division.
struct RowCtx {
  void *o0;       // row base of the output (LP: real plane)
  void *o1;       // LP: imaginary plane row
  uint32_t u0;    // pilot: first user of this symbol's comb
  uint32_t b;     // pilot: antenna
};

template <int MODE, int N>
__device__ __forceinline__ RowCtx row_ctx(const FftParams &p, uint64_t row) {
  RowCtx c{};
  const uint32_t sym = (uint32_t)(row / p.M), b = (uint32_t)(row - (uint64_t)sym * p.M);
  if constexpr (MODE == kUplink) {
    c.o0 = reinterpret_cast<float2 *>(p.out) + row * p.S;
  } else if constexpr (MODE == kUplinkLP) {
    __nv_bfloat16 *o = reinterpret_cast<__nv_bfloat16 *>(p.out);
    c.o0 = o + ((uint64_t)(sym * 2 + 0) * p.M + b) * p.S_pad;
    c.o1 = o + ((uint64_t)(sym * 2 + 1) * p.M + b) * p.S_pad;
  } else if constexpr (MODE == kPilot) {
    c.u0 = p.ue_start + sym * p.sg;
    c.b = b;
  } else {
    c.o0 = reinterpret_cast<char *>(p.out) + row * N * (p.out_dtype == MB_IQ_C32 ? 8 : p.out_dtype == MB_IQ_I8 ? 2 : 4);
  }
  return c;
}

template <int MODE, int N>
__device__ __forceinline__ void epilogue(const FftParams &p, const RowCtx &c, uint32_t k,
                                         float2 v) {
  if constexpr (MODE == kUplink) {
    const uint32_t i = (k - p.start - N / 2) & (N - 1);
    if (i < p.S) reinterpret_cast<float2 *>(c.o0)[i] = v;
  } else if constexpr (MODE == kUplinkLP) {
    // planar BF16 rows for the tensor-core equalizer: [sym][re|im][M][S_pad]
    const uint32_t i = (k - p.start - N / 2) & (N - 1);
    if (i < p.S) {
      reinterpret_cast<__nv_bfloat16 *>(c.o0)[i] = __float2bfloat16_rn(v.x);
      reinterpret_cast<__nv_bfloat16 *>(c.o1)[i] = __float2bfloat16_rn(v.y);
    }
  } else if constexpr (MODE == kPilot) {
    const uint32_t i = (k - p.start - N / 2) & (N - 1);
    if (i < p.S) {
      const uint32_t g = i / p.sg;
      const uint32_t u = c.u0 + (i - g * p.sg);
      if (u < p.K) {
        const float2 ps = __ldg(p.pilot + i);
        const float2 e = make_float2(v.x * ps.x + v.y * ps.y, v.x * ps.y - v.y * ps.x);
        reinterpret_cast<float2 *>(p.out)[((uint64_t)g * p.M + c.b) * p.K + u] = e;
        // a user with no pilot in the short last group takes its estimate
        // from group G-2 (the slot's tail rule)
        if (p.tail_rem && g + 2 == (p.S + p.sg - 1) / p.sg && i - g * p.sg >= p.tail_rem)
          reinterpret_cast<float2 *>(p.out)[((uint64_t)(g + 1) * p.M + c.b) * p.K + u] = e;
      }
    }
  } else {
    if (p.out_dtype == MB_IQ_I16 || p.out_dtype == MB_IQ_I8) {
      const bool i16 = p.out_dtype == MB_IQ_I16;
      const float qmax = i16 ? 32767.f : 127.f, qmin = i16 ? -32768.f : -128.f;
      const float sc = (qmax + 1.f) / (float)N;
      float re = v.x * sc, im = v.y * sc;
      int qr = __float2int_rn(re), qi = __float2int_rn(im);
      if (re > qmax) qr = (int)qmax; else if (re < qmin) qr = (int)qmin;
      if (im > qmax) qi = (int)qmax; else if (im < qmin) qi = (int)qmin;
      if (i16)
        reinterpret_cast<short2 *>(c.o0)[k] = make_short2((short)qr, (short)qi);
      else
        reinterpret_cast<char2 *>(c.o0)[k] = make_char2((char)qr, (char)qi);
    } else if (p.out_dtype == MB_IQ_F16) {
      const float sc = 1.f / (float)N;
      reinterpret_cast<__half2 *>(c.o0)[k] = __floats2half2_rn(v.x * sc, v.y * sc);
    } else {
      const float sc = 1.f / (float)N;
      reinterpret_cast<float2 *>(c.o0)[k] = make_float2(v.x * sc, v.y * sc);
    }
  }
}

template <int LOGN, int MODE>
__global__ void __launch_bounds__(Plan<LOGN>::THREADS, Plan<LOGN>::MIN_BLOCKS)
    fft_kernel(const FftParams p) {
  using PL = Plan<LOGN>;
  constexpr int N = PL::N, T = PL::T;
  constexpr bool INV = MODE == kIfft;
  extern __shared__ float2 smem_fft[];

  const int lrow = threadIdx.x / T;      // row within CTA
  const int t = threadIdx.x % T;         // thread within row
  const uint64_t row = (uint64_t)blockIdx.x * PL::ROWS + lrow;
  const bool active = row < p.rows;
  float2 *sm = smem_fft + lrow * PL::PADN;

  float2 v[16];
  int Ns = 1;
#pragma unroll
  for (int pass = 0; pass < PL::PASSES; pass++) {
    const int R = PL::radix(pass);
    const int BPT = 16 / R;  // butterflies per thread
    // ---- gather inputs
    if (pass == 0) {
      if (active) {
        const uint64_t base = row * N;
#pragma unroll
        for (int bi = 0; bi < 16; bi++) {
          // element j + r*N/R for butterfly j = t + (bi / R) * T, r = bi % R
          const int j = t + (bi / R) * T, r = bi % R;
          v[bi] = load_iq(p, base + j + r * (N / R));
        }
      } else {
#pragma unroll
        for (int bi = 0; bi < 16; bi++) v[bi] = make_float2(0.f, 0.f);
      }
    } else {
#pragma unroll
      for (int bi = 0; bi < 16; bi++) {
        const int j = t + (bi / R) * T, r = bi % R;
        v[bi] = sm[pad(j + r * (N / R))];
      }
      __syncthreads();  // every thread has read before anyone overwrites
      if (R == 16) {
        // W^(r jm), r = 1..15, from the exact table entries of r = 1 and 4
        // (at most three products from an exact entry): two loads instead
        // of fifteen
        const int jm = t % Ns;
        float2 w[16];
        w[1] = __ldg(p.tw + PL::tw_off(pass) + Ns + jm);
        w[4] = __ldg(p.tw + PL::tw_off(pass) + 4 * Ns + jm);
        if (INV) {
          w[1].y = -w[1].y;
          w[4].y = -w[4].y;
        }
        w[2] = cmul(w[1], w[1]);
        w[3] = cmul(w[2], w[1]);
        w[5] = cmul(w[4], w[1]);
        w[6] = cmul(w[4], w[2]);
        w[7] = cmul(w[4], w[3]);
        w[8] = cmul(w[4], w[4]);
#pragma unroll
        for (int r = 9; r < 16; r++) w[r] = cmul(w[8], w[r - 8]);
#pragma unroll
        for (int r = 1; r < 16; r++) v[r] = cmul(v[r], w[r]);
      } else {
#pragma unroll
        for (int bi = 0; bi < 16; bi++) {
          const int j = t + (bi / R) * T, r = bi % R;
          if (r) {
            const int m = PL::tw_off(pass) + r * Ns + (j % Ns);
            float2 w = __ldg(p.tw + m);
            if (INV) w.y = -w.y;
            v[bi] = cmul(v[bi], w);
          }
        }
      }
    }
    // ---- butterflies
    (void)BPT;
    if (R == 16) {
      dft<16, INV>(v);
    } else if (R == 8) {
      dft<8, INV>(v);
      dft<8, INV>(v + 8);
    } else if (R == 4) {
#pragma unroll
      for (int b = 0; b < 4; b++) dft<4, INV>(v + 4 * b);
    } else {
#pragma unroll
      for (int b = 0; b < 8; b++) dft<2, INV>(v + 2 * b);
    }
    // ---- scatter outputs
    if (pass + 1 < PL::PASSES) {
#pragma unroll
      for (int bi = 0; bi < 16; bi++) {
        const int j = t + (bi / R) * T, r = bi % R;
        const int idxD = (j / Ns) * Ns * R + (j % Ns);
        sm[pad(idxD + r * Ns)] = v[bi];
      }
      __syncthreads();
    } else if (active) {
      const RowCtx ctx = row_ctx<MODE, N>(p, row);
#pragma unroll
      for (int bi = 0; bi < 16; bi++) {
        const int j = t + (bi / R) * T, r = bi % R;
        // last pass: Ns = N / R, so idxD = j
        epilogue<MODE, N>(p, ctx, (uint32_t)(j + r * Ns), v[bi]);
      }
    }
    Ns *= R;
  }
}

template <int LOGN, int MODE>
static mb_status launch_one(const FftParams &p, cudaStream_t st) {
  using PL = Plan<LOGN>;
  const size_t smem = PL::PASSES > 1 ? sizeof(float2) * PL::PADN * PL::ROWS : 0;
  if (smem > 48 * 1024) {
    static std::atomic<uint64_t> configured{0};
    int dev = 0;
    MB_CUDA_TRY(cudaGetDevice(&dev));
    const uint64_t bit = 1ull << (dev & 63);
    if (!(configured.load() & bit)) {
      MB_CUDA_TRY(cudaFuncSetAttribute(fft_kernel<LOGN, MODE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
      configured.fetch_or(bit);
    }
  }
  const uint64_t blocks = (p.rows + PL::ROWS - 1) / PL::ROWS;
  if (blocks == 0) return MB_OK;
  if (blocks > 0x7fffffffull) return MB_BAD_SHAPE;
  fft_kernel<LOGN, MODE><<<(unsigned)blocks, PL::THREADS, smem, st>>>(p);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

template <int MODE>
static mb_status launch_fft(int logn, const FftParams &p, cudaStream_t st) {
  switch (logn) {
    case 4: return launch_one<4, MODE>(p, st);
    case 5: return launch_one<5, MODE>(p, st);
    case 6: return launch_one<6, MODE>(p, st);
    case 7: return launch_one<7, MODE>(p, st);
    case 8: return launch_one<8, MODE>(p, st);
    case 9: return launch_one<9, MODE>(p, st);
    case 10: return launch_one<10, MODE>(p, st);
    case 11: return launch_one<11, MODE>(p, st);
    case 12: return launch_one<12, MODE>(p, st);
    case 13: return launch_one<13, MODE>(p, st);
  }
  return MB_BAD_SHAPE;
}

}  // namespace mb

using namespace mb;

struct mb_fft {
  mb_fft_desc d;
  int logn;
  int device;
  const float2 *tw;
  float2 *pilot;  // device pilot sign table (S entries)
  FftTcPlan *tc;  // tensor-core FFT operands (N = 4096), else null
};

extern "C" mb_status mb_fft_create(const mb_fft_desc *desc, mb_fft **out) {
  if (!desc || !out) return MB_BAD_ARG;
  *out = nullptr;
  const mb_fft_desc &d = *desc;
  if (!is_pow2(d.ofdm_ca) || d.ofdm_ca < 16 || d.ofdm_ca > 8192) return MB_BAD_SHAPE;
  if (d.ofdm_num == 0 || d.ofdm_num > d.ofdm_ca || d.bs_num == 0) return MB_BAD_SHAPE;
  const DeviceTables *tab = device_tables();
  if (!tab) return MB_CUDA_ERROR;
  mb_fft *f = new mb_fft();
  f->d = d;
  f->logn = ilog2(d.ofdm_ca);
  cudaGetDevice(&f->device);
  f->tw = tab->twiddle[f->logn];
  f->pilot = nullptr;
  f->tc = fft_tc_plan_create(d.ofdm_ca, d.ofdm_start);
  if (d.ue_num > 0 && d.sc_group > 0) {
    mb_c32 *h = new mb_c32[d.ofdm_num];
    mb_pilot_sign(d.ofdm_num, h);
    cudaError_t e = cudaMalloc(&f->pilot, sizeof(float2) * d.ofdm_num);
    if (e == cudaSuccess)
      e = cudaMemcpy(f->pilot, h, sizeof(float2) * d.ofdm_num, cudaMemcpyHostToDevice);
    delete[] h;
    if (e != cudaSuccess) {
      if (f->pilot) cudaFree(f->pilot);
      fft_tc_plan_destroy(f->tc);
      delete f;
      return record_error(e);
    }
  }
  *out = f;
  return MB_OK;
}

extern "C" mb_status mb_fft_destroy(mb_fft *f) {
  if (!f) return MB_BAD_ARG;
  if (f->pilot) cudaFree(f->pilot);
  fft_tc_plan_destroy(f->tc);
  delete f;
  return MB_OK;
}

static bool dtype_ok(int dt) { return dt >= MB_IQ_C32 && dt <= MB_IQ_F16; }

extern "C" mb_status mb_fft_uplink(mb_fft *f, const void *iq, int iq_dtype,
                                   uint32_t n_sym, mb_c32 *out, void *stream) {
  if (!f || !iq || !out || !dtype_ok(iq_dtype)) return MB_BAD_ARG;
  FftParams p{};
  p.in = iq;
  p.out = out;
  p.tw = f->tw;
  p.rows = (uint64_t)n_sym * f->d.bs_num;
  p.M = f->d.bs_num;
  p.S = f->d.ofdm_num;
  p.start = f->d.ofdm_start;
  p.in_dtype = iq_dtype;
  return launch_fft<kUplink>(f->logn, p, as_stream(stream));
}

extern "C" mb_status mb_fft_uplink_bf16(mb_fft *f, const void *iq, int iq_dtype, uint32_t n_sym,
                                        void *out, uint32_t row_pitch, void *stream) {
  return fft_uplink_lp(f, iq, iq_dtype, n_sym, out, row_pitch, as_stream(stream));
}

mb_status mb::fft_uplink_lp(mb_fft *f, const void *iq, int iq_dtype, uint32_t n_sym,
                            void *y_lp, uint32_t S_pad, cudaStream_t st, uint32_t max_ctas) {
  if (!f || !iq || !y_lp || !dtype_ok(iq_dtype) || S_pad < f->d.ofdm_num) return MB_BAD_ARG;
  if (fft_tc_lp_supported(f->tc, iq, S_pad, y_lp)) {
    const DeviceTables *tab = device_tables();
    const uint32_t rows = n_sym * f->d.bs_num;
    return fft_tc_uplink_lp(f->tc, iq, iq_dtype, rows, f->d.bs_num, f->d.ofdm_num, y_lp, S_pad,
                            tab ? tab->err : nullptr, st, fft_tc_upc(rows, max_ctas));
  }
  FftParams p{};
  p.in = iq;
  p.out = y_lp;
  p.tw = f->tw;
  p.rows = (uint64_t)n_sym * f->d.bs_num;
  p.M = f->d.bs_num;
  p.S = f->d.ofdm_num;
  p.start = f->d.ofdm_start;
  p.S_pad = S_pad;
  p.in_dtype = iq_dtype;
  return launch_fft<kUplinkLP>(f->logn, p, st);
}

extern "C" mb_status mb_fft_pilot(mb_fft *f, const void *iq, int iq_dtype,
                                  uint32_t n_sym, uint32_t ue_start,
                                  mb_c32 *csi, void *stream) {
  if (!f || !iq || !csi || !dtype_ok(iq_dtype)) return MB_BAD_ARG;
  if (!f->pilot) return MB_BAD_SHAPE;  // created without ue_num / sc_group
  FftParams p{};
  p.in = iq;
  p.out = csi;
  p.tw = f->tw;
  p.pilot = f->pilot;
  p.rows = (uint64_t)n_sym * f->d.bs_num;
  p.M = f->d.bs_num;
  p.S = f->d.ofdm_num;
  p.start = f->d.ofdm_start;
  p.K = f->d.ue_num;
  p.sg = f->d.sc_group;
  p.ue_start = ue_start;
  p.in_dtype = iq_dtype;
  return launch_fft<kPilot>(f->logn, p, as_stream(stream));
}

bool mb::fft_slot_tc_ok(mb_fft *f, const void *iq, uint32_t S_pad, const void *y_lp) {
  return f && f->pilot && fft_tc_lp_supported(f->tc, iq, S_pad, y_lp);
}

mb_status mb::fft_slot_tc(mb_fft *f, const void *iq, int iq_dtype, uint32_t P, uint32_t U, mb_c32 *csi,
                          void *y_lp, uint32_t S_pad, cudaStream_t st, uint32_t max_ctas) {
  if (!fft_slot_tc_ok(f, iq, S_pad, y_lp) || !dtype_ok(iq_dtype) || !csi) return MB_BAD_ARG;
  const uint32_t S = f->d.ofdm_num, sg = f->d.sc_group, G = (S + sg - 1) / sg;
  const DeviceTables *tab = device_tables();
  return fft_tc_slot(f->tc, iq, iq_dtype, P, U, f->d.bs_num, S, f->d.ue_num, sg, G >= 2 ? S % sg : 0, f->pilot,
                     reinterpret_cast<float2 *>(csi), y_lp, S_pad, tab ? tab->err : nullptr, st,
                     fft_tc_upc((uint64_t)(P + U) * f->d.bs_num, max_ctas));
}

extern "C" mb_status mb_fft_pilot_mixed(mb_fft *f, const void *iq, int iq_dtype, uint32_t n_sym,
                                        uint32_t ue_start, mb_c32 *csi, void *stream) {
  if (!f || !iq || !csi || !dtype_ok(iq_dtype)) return MB_BAD_ARG;
  if (!f->pilot) return MB_BAD_SHAPE;
  if (!fft_tc_pilot_supported(f->tc, iq)) return mb_fft_pilot(f, iq, iq_dtype, n_sym, ue_start, csi, stream);
  const DeviceTables *tab = device_tables();
  return fft_tc_pilot(f->tc, iq, iq_dtype, n_sym, f->d.bs_num, f->d.ofdm_num, f->d.ue_num, f->d.sc_group,
                      ue_start, 0, f->pilot, reinterpret_cast<float2 *>(csi), tab ? tab->err : nullptr,
                      as_stream(stream));
}

mb_status mb::fft_pilot_fill(mb_fft *f, const void *iq, int iq_dtype, uint32_t n_sym, mb_c32 *csi,
                             cudaStream_t st, bool tensor) {
  if (!f || !iq || !csi || !dtype_ok(iq_dtype)) return MB_BAD_ARG;
  if (!f->pilot) return MB_BAD_SHAPE;
  if (tensor && fft_tc_pilot_supported(f->tc, iq)) {
    const uint32_t S = f->d.ofdm_num, sg = f->d.sc_group, G = (S + sg - 1) / sg;
    const DeviceTables *tab = device_tables();
    return fft_tc_pilot(f->tc, iq, iq_dtype, n_sym, f->d.bs_num, S, f->d.ue_num, sg, 0, G >= 2 ? S % sg : 0,
                        f->pilot, reinterpret_cast<float2 *>(csi), tab ? tab->err : nullptr, st);
  }
  FftParams p{};
  p.in = iq;
  p.out = csi;
  p.tw = f->tw;
  p.pilot = f->pilot;
  p.rows = (uint64_t)n_sym * f->d.bs_num;
  p.M = f->d.bs_num;
  p.S = f->d.ofdm_num;
  p.start = f->d.ofdm_start;
  p.K = f->d.ue_num;
  p.sg = f->d.sc_group;
  p.ue_start = 0;
  const uint32_t G = (p.S + p.sg - 1) / p.sg;
  p.tail_rem = G >= 2 ? p.S % p.sg : 0;
  p.in_dtype = iq_dtype;
  return launch_fft<kPilot>(f->logn, p, st);
}

bool mb::fft_ifft_tc_ok(mb_fft *f, const void *in, int in_dtype, const void *out, int out_dtype) {
  return f && fft_tc_inverse_supported(f->tc, in, in_dtype, out, out_dtype);
}

mb_status mb::fft_tc_inverse_slot(mb_fft *f, const void *in, uint32_t n_sym, void *out, int out_dtype,
                                  cudaStream_t st) {
  if (!fft_ifft_tc_ok(f, in, MB_IQ_F16, out, out_dtype)) return MB_BAD_ARG;
  const DeviceTables *tab = device_tables();
  return fft_tc_inverse(f->tc, in, MB_IQ_F16, n_sym * f->d.bs_num, out, out_dtype, tab ? tab->err : nullptr, st);
}

extern "C" mb_status mb_ifft_downlink_mixed(mb_fft *f, const void *in, int in_dtype, uint32_t n_sym, void *out,
                                            int out_dtype, void *stream) {
  if (!f || !in || !out || !dtype_ok(in_dtype) || !dtype_ok(out_dtype)) return MB_BAD_ARG;
  if (fft_tc_inverse_supported(f->tc, in, in_dtype, out, out_dtype)) {
    const DeviceTables *tab = device_tables();
    return fft_tc_inverse(f->tc, in, in_dtype, n_sym * f->d.bs_num, out, out_dtype, tab ? tab->err : nullptr,
                          as_stream(stream));
  }
  if (in_dtype != MB_IQ_C32) return MB_UNSUPPORTED;
  return mb_ifft_downlink(f, reinterpret_cast<const mb_c32 *>(in), n_sym, out, out_dtype, stream);
}

extern "C" mb_status mb_ifft_downlink(mb_fft *f, const mb_c32 *in,
                                      uint32_t n_sym, void *out, int out_dtype,
                                      void *stream) {
  if (!f || !in || !out || !dtype_ok(out_dtype)) return MB_BAD_ARG;
  FftParams p{};
  p.in = in;
  p.out = out;
  p.tw = f->tw;
  p.rows = (uint64_t)n_sym * f->d.bs_num;
  p.M = f->d.bs_num;
  p.in_dtype = MB_IQ_C32;
  p.out_dtype = out_dtype;
  return launch_fft<kIfft>(f->logn, p, as_stream(stream));
}

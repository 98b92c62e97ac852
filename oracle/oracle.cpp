/*
 * oracle.cpp -- CPU restatement of the MegaStation per-slot baseband
 * operators.  TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for the
 * CUDA path and the timed host baseline, never linked into the product.
 *
 * Reference paths are relative to the MegaStation source tree.
 */
#include "oracle.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;
typedef std::complex<float> cf;

/* ------------------------------------------------------------------ half */
uint16_t orc_f2h(float f) {
  _Float16 h = (_Float16)f;
  uint16_t u;
  memcpy(&u, &h, 2);
  return u;
}

float orc_h2f(uint16_t u) {
  _Float16 h;
  memcpy(&h, &u, 2);
  return (float)h;
}

static inline _Float16 hval(float f) { return (_Float16)f; }
static inline _Float16 habs(_Float16 h) { return h < (_Float16)0 ? -h : h; }
static inline uint16_t hbits(_Float16 h) {
  uint16_t u;
  memcpy(&u, &h, 2);
  return u;
}

/* ------------------------------------------------------------- sequences */
/* primes up to 2039, as the reference table kPrimeArray (utils.h:27-52) */
static uint32_t zc_length(uint64_t seq_len) {
  uint32_t best = 0;
  for (uint32_t p = 2; p <= 2039; p++) {
    bool prime = true;
    for (uint32_t d = 2; d * d <= p; d++)
      if (p % d == 0) {
        prime = false;
        break;
      }
    if (!prime) continue;
    if (p <= seq_len) best = p;
  }
  /* utils.h:56-62: the largest table prime <= seq_len, else the table's
   * last entry (2039) when seq_len exceeds it or nothing matches. */
  if (best == 0 || seq_len >= 2039) best = 2039;
  return best;
}

/* utils.h:54-75.  The phase is formed in double and handed to sincosf,
 * i.e. rounded to float first; sin/cos of that float are taken here in
 * double and rounded, which agrees with glibc sincosf to within 1 ulp. */
void orc_zadoff_chu(uint64_t seq_len, float *out) {
  uint32_t len = zc_length(seq_len);
  double root = floor(len * 2.0 / 31.0 + 0.5);
  for (uint64_t i = 0; i < seq_len; i++) {
    uint16_t m = (uint16_t)(i % len);
    double th = -M_PI * root * m * (m + 1) / len;
    float thf = (float)th;
    out[2 * i] = (float)cos((double)thf);
    out[2 * i + 1] = (float)sin((double)thf);
  }
}

/* utils.h:77-95: c = e^{j alpha i} with the product alpha*i in float. */
void orc_cyclic_shift(const float *in, float *out, uint64_t len, float alpha) {
  for (uint64_t i = 0; i < len; i++) {
    float a = alpha * (float)i;
    float cr = (float)cos((double)a), ci = (float)sin((double)a);
    float re = in[2 * i], im = in[2 * i + 1];
    out[2 * i] = re * cr - im * ci;
    out[2 * i + 1] = re * ci + im * cr;
  }
}

/* fft_op.cu:176-192: zc(S) shifted by pi/4, divided by its power. */
void orc_pilot_sign(uint64_t S, float *out) {
  orc_zadoff_chu(S, out);
  orc_cyclic_shift(out, out, S, (float)(M_PI / 4));
  for (uint64_t i = 0; i < S; i++) {
    float p2 = out[2 * i] * out[2 * i] + out[2 * i + 1] * out[2 * i + 1];
    out[2 * i] /= p2;
    out[2 * i + 1] /= p2;
  }
}

/* modulation.cu:82-86: user u gets zc(S) shifted by u*pi/6. */
void orc_dmrs_table(uint64_t S, uint64_t K, float *out) {
  std::vector<float> zc(2 * S);
  orc_zadoff_chu(S, zc.data());
  for (uint64_t u = 0; u < K; u++)
    orc_cyclic_shift(zc.data(), out + 2 * u * S, S, (float)(u * M_PI / 6));
}

/* ------------------------------------------------------------- scrambler */
/* scrambler.cu:22-31: 7-bit LFSR x^7+x^4+1 from state 0x5D, 127 bits. */
void orc_scrambler_seq127(uint8_t *seq) {
  uint8_t s = 0x5D;
  for (int i = 0; i < 127; i++) {
    uint8_t fb = (s ^ (s >> 3)) & 1;
    seq[i] = fb;
    s >>= 1;
    s |= fb << 6;
  }
}

/* scrambler_kernel.cuh:36-56: byte j XOR bits seq[(8j+k) % 127], k = 0
 * landing in the most significant bit. */
void orc_scramble_bytes(uint8_t *out, const uint8_t *in, uint64_t num_bytes,
                        uint64_t batch) {
  uint8_t seq[127];
  orc_scrambler_seq127(seq);
  for (uint64_t b = 0; b < batch; b++)
    for (uint64_t j = 0; j < num_bytes; j++) {
      uint32_t idx = (uint32_t)((j * 8) % 127);
      uint8_t sb = 0;
      for (int k = 0; k < 8; k++) {
        sb = (uint8_t)((sb << 1) | seq[idx]);
        idx = (idx + 1) % 127;
      }
      out[b * num_bytes + j] = sb ^ in[b * num_bytes + j];
    }
}

/* TS 38.211 5.2.1: c(n) = x1(n+Nc) ^ x2(n+Nc), Nc = 1600,
 * x1(n+31) = x1(n+3) ^ x1(n), x2(n+31) = x2(n+3)^x2(n+2)^x2(n+1)^x2(n),
 * x1 starts 1,0,0,...; x2 starts with the bits of c_init. */
void orc_gold_seq(uint32_t c_init, uint64_t n_bits, uint8_t *bits) {
  const uint64_t Nc = 1600;
  uint64_t total = n_bits + Nc + 31;
  std::vector<uint8_t> x1(total), x2(total);
  for (int i = 0; i < 31; i++) {
    x1[i] = (i == 0);
    x2[i] = (c_init >> i) & 1;
  }
  for (uint64_t n = 0; n + 31 < total; n++) {
    x1[n + 31] = x1[n + 3] ^ x1[n];
    x2[n + 31] = x2[n + 3] ^ x2[n + 2] ^ x2[n + 1] ^ x2[n];
  }
  for (uint64_t n = 0; n < n_bits; n++) bits[n] = x1[n + Nc] ^ x2[n + Nc];
}

/* ------------------------------------------------------------ modulation */
/* modulation.cu:22-72: Gray tables, first stream bit = index MSB. */
void orc_mod_table(int Qm, float *t) {
  int M = 1 << Qm;
  if (Qm == 2) {
    float s = (float)(1 / sqrt(2));
    float v[2] = {-s, s};
    for (int i = 0; i < 4; i++) {
      t[2 * i] = v[i / 2];
      t[2 * i + 1] = v[i % 2];
    }
  } else if (Qm == 4) {
    float s = (float)(1 / sqrt(10));
    float v[4] = {1 * s, 3 * s, -1 * s, -3 * s};
    for (int i = 0; i < M; i++) {
      int im = (((i >> 2) & 1) << 1) + (i & 1);
      int re = (((i >> 3) & 1) << 1) + ((i >> 1) & 1);
      t[2 * i] = v[re];
      t[2 * i + 1] = v[im];
    }
  } else if (Qm == 6) {
    float s = (float)(1 / sqrt(42));
    float v[8] = {3 * s, 1 * s, 5 * s, 7 * s, -3 * s, -1 * s, -5 * s, -7 * s};
    for (int i = 0; i < M; i++) {
      int im = (((i >> 4) & 1) << 2) + (((i >> 2) & 1) << 1) + (i & 1);
      int re = (((i >> 5) & 1) << 2) + (((i >> 3) & 1) << 1) + ((i >> 1) & 1);
      t[2 * i] = v[re];
      t[2 * i + 1] = v[im];
    }
  } else if (Qm == 8) {
    float s = (float)(1 / sqrt(170));
    float v[16] = {-15 * s, -13 * s, -9 * s, -11 * s, -1 * s, -3 * s,
                   -7 * s,  -5 * s,  15 * s, 13 * s,  9 * s,  11 * s,
                   1 * s,   3 * s,   7 * s,  5 * s};
    for (int i = 0; i < M; i++) {
      int im = ((i & 0x40) >> 3) + ((i & 0x10) >> 2) + ((i & 0x4) >> 1) +
               (i & 0x1);
      int re = ((i & 0x80) >> 4) + ((i & 0x20) >> 3) + ((i & 0x8) >> 2) +
               ((i & 0x2) >> 1);
      t[2 * i] = v[re];
      t[2 * i + 1] = v[im];
    }
  }
}

/* modulation_kernel.cuh:37-68 */
void orc_modulate(const uint8_t *in, float *out, uint64_t in_bytes,
                  uint64_t num_carriers, uint64_t num_ues, int Qm,
                  uint32_t pilot_spacing, const float *pilot_table) {
  float table[512];
  orc_mod_table(Qm, table);
  for (uint64_t u = 0; u < num_ues; u++)
    for (uint64_t c = 0; c < num_carriers; c++) {
      uint64_t shrink =
          pilot_spacing ? c - ((c / pilot_spacing) + 1) : c;
      const uint8_t *src = in + u * in_bytes;
      uint32_t mb = 0;
      uint64_t idx = shrink * Qm;
      for (int i = 0; i < Qm && (idx / 8) < in_bytes; i++, idx++)
        mb = ((src[idx / 8] >> (idx % 8)) & 1) | (mb << 1);
      float *o = out + 2 * (u * num_carriers + c);
      if (pilot_spacing && (c % pilot_spacing) == 0) {
        o[0] = pilot_table[2 * (u * num_carriers + c)];
        o[1] = pilot_table[2 * (u * num_carriers + c) + 1];
      } else {
        o[0] = table[2 * (mb & ((1u << Qm) - 1))];
        o[1] = table[2 * (mb & ((1u << Qm) - 1)) + 1];
      }
    }
}

/* demodulation.h:30-67 in half arithmetic (each t - |l| rounds once). */
void orc_demod(int Qm, float re, float im, uint16_t *llr) {
  _Float16 l[8];
  if (Qm == 2) {
    l[0] = hval(re * -20.0f * sqrtf(2.f));
    l[1] = hval(im * -20.0f * sqrtf(2.f));
  } else if (Qm == 4) {
    _Float16 t = hval(2 * 100 / sqrtf(10.f));
    l[0] = hval(100 * re);
    l[1] = hval(100 * im);
    l[2] = (_Float16)((float)t - (float)habs(l[0]));
    l[3] = (_Float16)((float)t - (float)habs(l[1]));
  } else if (Qm == 6) {
    _Float16 t1 = hval(4 * 100 / sqrtf(42.f));
    _Float16 t2 = hval(2 * 100 / sqrtf(42.f));
    l[0] = hval(100 * re);
    l[1] = hval(100 * im);
    l[2] = (_Float16)((float)t1 - (float)habs(l[0]));
    l[3] = (_Float16)((float)t1 - (float)habs(l[1]));
    l[4] = (_Float16)((float)t2 - (float)habs(l[2]));
    l[5] = (_Float16)((float)t2 - (float)habs(l[3]));
  } else if (Qm == 8) {
    _Float16 t1 = hval(8 * 100 / sqrtf(170.f));
    _Float16 t2 = hval(4 * 100 / sqrtf(170.f));
    _Float16 t3 = hval(2 * 100 / sqrtf(170.f));
    l[0] = hval(100 * re);
    l[1] = hval(100 * im);
    l[2] = (_Float16)((float)t1 - (float)habs(l[0]));
    l[3] = (_Float16)((float)t1 - (float)habs(l[1]));
    l[4] = (_Float16)((float)t2 - (float)habs(l[2]));
    l[5] = (_Float16)((float)t2 - (float)habs(l[3]));
    l[6] = (_Float16)((float)t3 - (float)habs(l[4]));
    l[7] = (_Float16)((float)t3 - (float)habs(l[5]));
  } else {
    return;
  }
  for (int q = 0; q < Qm; q++) llr[q] = hbits(l[q]);
}

/* ------------------------------------------------------------------- FFT */
template <typename T>
static void fft_inplace(std::complex<T> *x, uint32_t n, int inverse,
                        const std::complex<T> *tw /* n/2 entries */) {
  /* iterative radix-2 decimation in time, unnormalised (cuFFT convention:
   * forward e^{-j2pi kn/N}, inverse e^{+j2pi kn/N}) */
  for (uint32_t i = 1, j = 0; i < n; i++) {
    uint32_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(x[i], x[j]);
  }
  for (uint32_t len = 2; len <= n; len <<= 1) {
    uint32_t step = n / len;
    for (uint32_t i = 0; i < n; i += len)
      for (uint32_t k = 0; k < len / 2; k++) {
        std::complex<T> w = tw[k * step];
        if (inverse) w = std::conj(w);
        std::complex<T> u = x[i + k], v = x[i + k + len / 2] * w;
        x[i + k] = u + v;
        x[i + k + len / 2] = u - v;
      }
  }
}

template <typename T>
static std::vector<std::complex<T>> twiddles(uint32_t n) {
  std::vector<std::complex<T>> tw(n / 2 + 1);
  for (uint32_t k = 0; k < n / 2 + 1; k++) {
    double a = -2.0 * M_PI * (double)k / (double)n;
    tw[k] = std::complex<T>((T)cos(a), (T)sin(a));
  }
  return tw;
}

void orc_fft_d(double *x, uint32_t n, int inverse) {
  auto tw = twiddles<double>(n);
  fft_inplace<double>(reinterpret_cast<cd *>(x), n, inverse, tw.data());
}

/* fft_callback.cuh:20-41 + fft_utils.h:19-22: ints scale by 1/(max+1). */
template <typename T>
static inline std::complex<T> load_iq(const void *in, int dtype, uint64_t i) {
  switch (dtype) {
    case 0: {
      const float *p = (const float *)in;
      return std::complex<T>(p[2 * i], p[2 * i + 1]);
    }
    case 1: {
      const int16_t *p = (const int16_t *)in;
      return std::complex<T>((float)p[2 * i] / 32768.f,
                             (float)p[2 * i + 1] / 32768.f);
    }
    case 2: {
      const int8_t *p = (const int8_t *)in;
      return std::complex<T>((float)p[2 * i] / 128.f,
                             (float)p[2 * i + 1] / 128.f);
    }
    case 3: {
      const uint16_t *p = (const uint16_t *)in;
      return std::complex<T>(orc_h2f(p[2 * i]), orc_h2f(p[2 * i + 1]));
    }
  }
  return std::complex<T>(0, 0);
}

/* fft_op.cu:135-143 + fft_callback.cuh:43-74:
 * out[b][i] = FFT(row b)[(i + start + N/2) % N], i < S. */
void orc_uplink_fft(const void *in, int dtype, uint32_t M, uint32_t N,
                    uint32_t S, uint32_t start, float *out) {
  auto tw = twiddles<double>(N);
  std::vector<cd> row(N);
  for (uint32_t b = 0; b < M; b++) {
    for (uint32_t k = 0; k < N; k++)
      row[k] = load_iq<double>(in, dtype, (uint64_t)b * N + k);
    fft_inplace<double>(row.data(), N, 0, tw.data());
    for (uint32_t i = 0; i < S; i++) {
      cd v = row[(i + start + N / 2) % N];
      out[2 * ((uint64_t)b * S + i)] = (float)v.real();
      out[2 * ((uint64_t)b * S + i) + 1] = (float)v.imag();
    }
  }
}

/* fft_op.cu:145-165 + fft_callback.cuh:76-108: the least-squares pilot
 * estimate conj(X)*p/|p|^2 of subcarrier i goes to CSI[g][b][u] with
 * g = i / sg and u = ue_start + i % sg (dropped when u >= K). */
void orc_pilot_fft(const void *in, int dtype, uint32_t M, uint32_t N,
                   uint32_t S, uint32_t start, uint32_t K, uint32_t sg,
                   uint32_t ue_start, const float *ps, float *csi) {
  auto tw = twiddles<double>(N);
  std::vector<cd> row(N);
  for (uint32_t b = 0; b < M; b++) {
    for (uint32_t k = 0; k < N; k++)
      row[k] = load_iq<double>(in, dtype, (uint64_t)b * N + k);
    fft_inplace<double>(row.data(), N, 0, tw.data());
    for (uint32_t i = 0; i < S; i++) {
      cd x = row[(i + start + N / 2) % N];
      cd p(ps[2 * i], ps[2 * i + 1]);
      cd e = std::conj(x) * p;
      uint64_t g = i / sg, u = ue_start + i % sg;
      if (u >= K) continue;
      uint64_t o = g * (uint64_t)M * K + (uint64_t)b * K + u;
      csi[2 * o] = (float)e.real();
      csi[2 * o + 1] = (float)e.imag();
    }
  }
}

/* fft_op.cu:167-174 + ifft_callback.cuh:21-59: unnormalised inverse FFT,
 * then q = sat(rint(x * (max+1)/N)) for int outputs.  out_dtype 0 (complex
 * float32) and 3 (complex fp16) store x/N. */
void orc_ifft_downlink(const float *in, uint32_t M, uint32_t N, int out_dtype,
                       void *out) {
  auto tw = twiddles<double>(N);
  std::vector<cd> row(N);
  for (uint32_t b = 0; b < M; b++) {
    for (uint32_t k = 0; k < N; k++)
      row[k] = cd(in[2 * ((uint64_t)b * N + k)], in[2 * ((uint64_t)b * N + k) + 1]);
    fft_inplace<double>(row.data(), N, 1, tw.data());
    for (uint32_t k = 0; k < N; k++) {
      uint64_t o = (uint64_t)b * N + k;
      float re = (float)row[k].real(), im = (float)row[k].imag();
      if (out_dtype == 1 || out_dtype == 2) {
        float qmax = out_dtype == 1 ? 32767.f : 127.f;
        float qmin = out_dtype == 1 ? -32768.f : -128.f;
        float sc = (qmax + 1.0f) / (float)N;
        float v[2] = {re * sc, im * sc};
        int q[2];
        for (int c = 0; c < 2; c++) {
          q[c] = (int)nearbyintf(v[c]);
          if (v[c] > qmax) q[c] = (int)qmax;
          else if (v[c] < qmin) q[c] = (int)qmin;
        }
        if (out_dtype == 1) {
          ((int16_t *)out)[2 * o] = (int16_t)q[0];
          ((int16_t *)out)[2 * o + 1] = (int16_t)q[1];
        } else {
          ((int8_t *)out)[2 * o] = (int8_t)q[0];
          ((int8_t *)out)[2 * o + 1] = (int8_t)q[1];
        }
      } else if (out_dtype == 3) {
        float sc = 1.0f / (float)N;
        ((uint16_t *)out)[2 * o] = orc_f2h(re * sc);
        ((uint16_t *)out)[2 * o + 1] = orc_f2h(im * sc);
      } else {
        float sc = 1.0f / (float)N;
        ((float *)out)[2 * o] = re * sc;
        ((float *)out)[2 * o + 1] = im * sc;
      }
    }
  }
}

/* ------------------------------------------------------------ zero forcing */
/* Source group of user u in group g: the last group of a band whose S is not
 * a multiple of sg has only S - (G-1)*sg pilot subcarriers, so users whose
 * comb position (u % sg) lies past them borrow group g-1's estimate.  The
 * reference sizes CSI for S/sg groups and drops the tail
 * (baseband/buffers.cc:73-78); this is the documented deviation. */
static inline uint32_t src_group(uint32_t g, uint32_t u, uint32_t G,
                                 uint32_t S, uint32_t sg) {
  if (g + 1 == G && g > 0) {
    uint32_t rem = S - g * sg;
    if (rem < sg && (u % sg) >= rem) return g - 1;
  }
  return g;
}

/* Hermitian power iteration: largest eigenvalue of A (K x K, row-major). */
static double herm_lmax(const std::vector<cd> &A, uint32_t K) {
  std::vector<cd> v(K, cd(1.0, 0.0)), w(K);
  double lam = 0;
  for (int it = 0; it < 200; it++) {
    double nrm = 0;
    for (uint32_t i = 0; i < K; i++) {
      cd s = 0;
      for (uint32_t j = 0; j < K; j++) s += A[i * K + j] * v[j];
      w[i] = s;
      nrm += std::norm(s);
    }
    nrm = sqrt(nrm);
    if (nrm == 0) return 0;
    for (uint32_t i = 0; i < K; i++) v[i] = w[i] / nrm;
    if (fabs(nrm - lam) <= 1e-13 * nrm) {
      lam = nrm;
      break;
    }
    lam = nrm;
  }
  return lam;
}

/* beamform.cu:74-122: per group, Gram A = C C^H with C = CSI[g] viewed as a
 * K x M column-major matrix (C[u][b] = csi[g][b][u]), Cholesky A = L L^H,
 * W = A^{-1} C written in the CSI layout.  FP64.  cond[g] = 2-norm condition
 * number of A (power iteration on A and A^{-1}).  Returns the number of
 * groups whose Gram is not positive definite (their W is zero). */
int orc_zf(const float *csi, uint32_t G, uint32_t M, uint32_t K, uint32_t S,
           uint32_t sg, float *W, double *cond) {
  int bad = 0;
  for (uint32_t g = 0; g < G; g++) {
    std::vector<cd> C((size_t)K * M), A((size_t)K * K), L((size_t)K * K);
    for (uint32_t u = 0; u < K; u++) {
      uint32_t gs = src_group(g, u, G, S, sg);
      for (uint32_t b = 0; b < M; b++) {
        uint64_t o = (uint64_t)gs * M * K + (uint64_t)b * K + u;
        C[(size_t)u * M + b] = cd(csi[2 * o], csi[2 * o + 1]);
      }
    }
    for (uint32_t i = 0; i < K; i++)
      for (uint32_t j = 0; j < K; j++) {
        cd s = 0;
        for (uint32_t b = 0; b < M; b++)
          s += C[(size_t)i * M + b] * std::conj(C[(size_t)j * M + b]);
        A[i * K + j] = s;
      }
    bool ok = true;
    for (uint32_t j = 0; j < K && ok; j++) {
      double d = A[j * K + j].real();
      for (uint32_t k = 0; k < j; k++) d -= std::norm(L[j * K + k]);
      if (!(d > 0)) {
        ok = false;
        break;
      }
      double ljj = sqrt(d);
      L[j * K + j] = ljj;
      for (uint32_t i = j + 1; i < K; i++) {
        cd s = A[i * K + j];
        for (uint32_t k = 0; k < j; k++) s -= L[i * K + k] * std::conj(L[j * K + k]);
        L[i * K + j] = s / ljj;
      }
    }
    if (cond) {
      if (!ok) {
        cond[g] = INFINITY;
      } else {
        /* explicit inverse via the Cholesky factor */
        std::vector<cd> Ai((size_t)K * K);
        for (uint32_t c = 0; c < K; c++) {
          std::vector<cd> z(K);
          for (uint32_t i = 0; i < K; i++) {
            cd s = (i == c) ? cd(1, 0) : cd(0, 0);
            for (uint32_t k = 0; k < i; k++) s -= L[i * K + k] * z[k];
            z[i] = s / L[i * K + i];
          }
          for (int i = (int)K - 1; i >= 0; i--) {
            cd s = z[i];
            for (uint32_t k = i + 1; k < K; k++) s -= std::conj(L[k * K + i]) * z[k];
            z[i] = s / L[i * K + i];
          }
          for (uint32_t i = 0; i < K; i++) Ai[i * K + c] = z[i];
        }
        cond[g] = herm_lmax(A, K) * herm_lmax(Ai, K);
      }
    }
    for (uint32_t b = 0; b < M; b++) {
      std::vector<cd> z(K);
      if (ok) {
        for (uint32_t i = 0; i < K; i++) {
          cd s = C[(size_t)i * M + b];
          for (uint32_t k = 0; k < i; k++) s -= L[i * K + k] * z[k];
          z[i] = s / L[i * K + i];
        }
        for (int i = (int)K - 1; i >= 0; i--) {
          cd s = z[i];
          for (uint32_t k = i + 1; k < K; k++) s -= std::conj(L[k * K + i]) * z[k];
          z[i] = s / L[i * K + i];
        }
      }
      for (uint32_t u = 0; u < K; u++) {
        uint64_t o = (uint64_t)g * M * K + (uint64_t)b * K + u;
        W[2 * o] = (float)z[u].real();
        W[2 * o + 1] = (float)z[u].imag();
      }
    }
    if (!ok) bad++;
  }
  return bad;
}

/* beam_utils.cuh:40-80: P[g][u][b] = W[g][b][u] / max|W[g]| in float. */
void orc_precoder(const float *W, uint32_t G, uint32_t M, uint32_t K,
                  float *P) {
  for (uint32_t g = 0; g < G; g++) {
    const float *w = W + 2 * (uint64_t)g * M * K;
    float *p = P + 2 * (uint64_t)g * M * K;
    float mx = 0.f;
    for (uint64_t i = 0; i < (uint64_t)M * K; i++)
      mx = fmaxf(mx, sqrtf(w[2 * i] * w[2 * i] + w[2 * i + 1] * w[2 * i + 1]));
    float inv = 1.0f / mx;
    for (uint32_t b = 0; b < M; b++)
      for (uint32_t u = 0; u < K; u++) {
        uint64_t i = (uint64_t)b * K + u, o = (uint64_t)u * M + b;
        p[2 * o] = w[2 * i] * inv;
        p[2 * o + 1] = w[2 * i + 1] * inv;
      }
  }
}

/* ------------------------------------------------------ equalize/precode */
void orc_equalize(const float *W, const float *y, uint32_t K, uint32_t M,
                  uint32_t S, uint32_t sg, int Qm, uint64_t cb_size,
                  uint64_t cb_stride, uint64_t zeros, uint32_t cb_blocks,
                  uint16_t *llr, float *x_out, const uint8_t *seq_bits,
                  uint64_t seq_len, uint64_t seq_user_stride,
                  uint8_t *hard_bytes) {
  uint64_t row = cb_stride * cb_blocks;
  uint64_t n_valid = std::min<uint64_t>((uint64_t)S * Qm, cb_size * cb_blocks);
  uint64_t hrow = (n_valid + 7) / 8;
  if (hard_bytes) memset(hard_bytes, 0, hrow * K);
  for (uint32_t s = 0; s < S; s++) {
    uint32_t g = s / sg;
    for (uint32_t u = 0; u < K; u++) {
      cd acc = 0;
      for (uint32_t b = 0; b < M; b++) {
        uint64_t wi = (uint64_t)g * M * K + (uint64_t)b * K + u;
        uint64_t yi = (uint64_t)b * S + s;
        acc += cd(W[2 * wi], W[2 * wi + 1]) * cd(y[2 * yi], y[2 * yi + 1]);
      }
      float xr = (float)acc.real(), xi = (float)acc.imag();
      if (x_out) {
        x_out[2 * ((uint64_t)u * S + s)] = xr;
        x_out[2 * ((uint64_t)u * S + s) + 1] = xi;
      }
      uint16_t l[8];
      orc_demod(Qm, xr, xi, l);
      uint64_t t0 = (uint64_t)s * Qm;
      uint64_t cb = t0 / cb_size;
      if (llr && cb < cb_blocks) {
        uint64_t base = cb * cb_stride + zeros + t0 % cb_size;
        for (int q = 0; q < Qm; q++)
          if (base + q < row) llr[(uint64_t)u * row + base + q] = l[q];
      }
      if (hard_bytes)
        for (int q = 0; q < Qm; q++) {
          uint64_t t = t0 + q;
          if (t >= n_valid) break;
          uint8_t h = (orc_h2f(l[q]) < 0.f) ? 1 : 0;
          h ^= seq_bits[u * seq_user_stride + t % seq_len];
          hard_bytes[u * hrow + t / 8] |= (uint8_t)(h << (7 - t % 8));
        }
    }
  }
}

/* precode_kernel.cuh:255-262 (naive spec :348-386), with s laid out
 * [K][S] (subcarrier fastest, precode.cu:61-67): out[b][(s+start+N/2)%N] =
 * sum_u P[g][u][b] s[u][s]; guard bins are written as zero. */
void orc_precode(const float *P, const float *sv, uint32_t M, uint32_t K,
                 uint32_t S, uint32_t sg, uint32_t N, uint32_t start,
                 float *out) {
  memset(out, 0, sizeof(float) * 2 * (uint64_t)M * N);
  for (uint32_t b = 0; b < M; b++)
    for (uint32_t s = 0; s < S; s++) {
      uint32_t g = s / sg;
      cd acc = 0;
      for (uint32_t u = 0; u < K; u++) {
        uint64_t pi = (uint64_t)g * M * K + (uint64_t)u * M + b;
        uint64_t si = (uint64_t)u * S + s;
        acc += cd(P[2 * pi], P[2 * pi + 1]) * cd(sv[2 * si], sv[2 * si + 1]);
      }
      uint64_t o = (uint64_t)b * N + (s + start + N / 2) % N;
      out[2 * o] = (float)acc.real();
      out[2 * o + 1] = (float)acc.imag();
    }
}

/* ------------------------------------------------------------ LDPC sizes */
/* config.cc:84-135 with cuPHY's BG1/BG2 info columns (22/10) and the two
 * punctured columns of TS 38.212 5.3.2 (ldpc/config.h:27-73). */
void orc_ldpc_sizes(uint64_t S, int Qm, double rate, int bg,
                    uint64_t pilot_spacing, int downlink, uint64_t *encoded,
                    uint64_t *punctured, uint64_t *decoded) {
  static const uint64_t zc_set[] = {
      2,   4,   8,   16, 32, 64,  128, 256, 3,   6,   12,  24, 48,
      96,  192, 384, 5,  10, 20,  40,  80,  160, 320, 7,   14, 28,
      56,  112, 224, 9,  18, 36,  72,  144, 288, 11,  22,  44, 88,
      176, 352, 13,  26, 52, 104, 208, 15,  30,  60,  120, 240};
  std::vector<uint64_t> zc(zc_set, zc_set + sizeof(zc_set) / sizeof(zc_set[0]));
  std::sort(zc.begin(), zc.end());
  uint64_t kb = bg == 1 ? 22 : 10;
  uint64_t data = downlink && pilot_spacing ? S - S / pilot_spacing : S;
  uint64_t uncoded = (uint64_t)((double)(data * Qm) * rate);
  uint64_t z = zc.back();
  for (size_t i = 0; i + 1 < zc.size(); i++)
    if (kb * zc[i] <= uncoded && kb * zc[i + 1] > uncoded) {
      z = zc[i];
      break;
    }
  uint64_t rows = (uint64_t)llround(kb / rate) - (kb - 2);
  *encoded = (kb - 2 + rows) * z;
  *decoded = kb * z;
  *punctured = 2 * z;
}

/* --------------------------------------------------- host slot baseline */
/* One uplink slot in FP32 on the host, parallelised with OpenMP, in the
 * stage order of BandProcess::process (baseband/process.cc:161-193):
 * pilot FFT + LS estimate per pilot symbol, per-group Cholesky ZF
 * (beamform.cu:74-122), then per uplink symbol FFT, equalize and demod with
 * descrambled hard bits.  csi_work holds G*M*K complex, y_work U*M*S. */
int orc_slot_uplink_cpu(const void *iq, int dtype, uint32_t P, uint32_t U,
                        uint32_t M, uint32_t K, uint32_t N, uint32_t S,
                        uint32_t sg, int Qm, uint64_t cb_size,
                        uint64_t cb_stride, uint64_t zeros,
                        const float *pilot_sign, const uint8_t *seq_bits,
                        uint64_t seq_len, float *csi_work, float *y_work,
                        uint16_t *llr, uint8_t *hard_bytes, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  const uint32_t G = (S + sg - 1) / sg;
  const uint32_t start = (N - S) / 2;
  const uint64_t sym_in = (uint64_t)M * N;
  const size_t in_elem = dtype == 0 ? 8 : dtype == 2 ? 2 : 4;
  auto tw = twiddles<float>(N);
  int bad = 0;

#pragma omp parallel for schedule(static)
  for (int64_t pb = 0; pb < (int64_t)P * M; pb++) {
    uint32_t p = (uint32_t)(pb / M), b = (uint32_t)(pb % M);
    std::vector<cf> row(N);
    const char *src = (const char *)iq + in_elem * 2 * 0 + (uint64_t)p * sym_in * in_elem;
    for (uint32_t k = 0; k < N; k++)
      row[k] = load_iq<float>(src, dtype, (uint64_t)b * N + k);
    fft_inplace<float>(row.data(), N, 0, tw.data());
    for (uint32_t i = 0; i < S; i++) {
      uint32_t u = p * sg + i % sg;
      if (u >= K) continue;
      cf x = row[(i + start + N / 2) % N];
      float pr = pilot_sign[2 * i], pi = pilot_sign[2 * i + 1];
      uint64_t o = (uint64_t)(i / sg) * M * K + (uint64_t)b * K + u;
      csi_work[2 * o] = x.real() * pr + x.imag() * pi;
      csi_work[2 * o + 1] = x.real() * pi - x.imag() * pr;
    }
  }

#pragma omp parallel for schedule(dynamic) reduction(+ : bad)
  for (int64_t g = 0; g < (int64_t)G; g++) {
    std::vector<cf> C((size_t)K * M), A((size_t)K * K), L((size_t)K * K);
    for (uint32_t u = 0; u < K; u++) {
      uint32_t gs = src_group((uint32_t)g, u, G, S, sg);
      for (uint32_t b = 0; b < M; b++) {
        uint64_t o = (uint64_t)gs * M * K + (uint64_t)b * K + u;
        C[(size_t)u * M + b] = cf(csi_work[2 * o], csi_work[2 * o + 1]);
      }
    }
    for (uint32_t i = 0; i < K; i++)
      for (uint32_t j = 0; j <= i; j++) {
        float sr = 0, si = 0;
        const cf *ci = &C[(size_t)i * M], *cj = &C[(size_t)j * M];
        for (uint32_t b = 0; b < M; b++) {
          sr += ci[b].real() * cj[b].real() + ci[b].imag() * cj[b].imag();
          si += ci[b].imag() * cj[b].real() - ci[b].real() * cj[b].imag();
        }
        A[i * K + j] = cf(sr, si);
      }
    bool ok = true;
    for (uint32_t j = 0; j < K && ok; j++) {
      float d = A[j * K + j].real();
      for (uint32_t k = 0; k < j; k++) d -= std::norm(L[j * K + k]);
      if (!(d > 0)) {
        ok = false;
        break;
      }
      float ljj = sqrtf(d);
      L[j * K + j] = ljj;
      for (uint32_t i = j + 1; i < K; i++) {
        cf s = A[i * K + j];
        for (uint32_t k = 0; k < j; k++) s -= L[i * K + k] * std::conj(L[j * K + k]);
        L[i * K + j] = s / ljj;
      }
    }
    if (!ok) bad++;
    std::vector<cf> z(K);
    for (uint32_t b = 0; b < M; b++) {
      for (uint32_t i = 0; i < K; i++) {
        cf s = ok ? C[(size_t)i * M + b] : cf(0, 0);
        for (uint32_t k = 0; k < i && ok; k++) s -= L[i * K + k] * z[k];
        z[i] = ok ? s / L[i * K + i] : cf(0, 0);
      }
      for (int i = (int)K - 1; i >= 0 && ok; i--) {
        cf s = z[i];
        for (uint32_t k = i + 1; k < K; k++) s -= std::conj(L[k * K + i]) * z[k];
        z[i] = s / L[i * K + i];
      }
      for (uint32_t u = 0; u < K; u++) {
        uint64_t o = (uint64_t)g * M * K + (uint64_t)b * K + u;
        csi_work[2 * o] = z[u].real();
        csi_work[2 * o + 1] = z[u].imag();
      }
    }
  }

#pragma omp parallel for schedule(static)
  for (int64_t lb = 0; lb < (int64_t)U * M; lb++) {
    uint32_t l = (uint32_t)(lb / M), b = (uint32_t)(lb % M);
    std::vector<cf> row(N);
    const char *src = (const char *)iq + (uint64_t)(P + l) * sym_in * in_elem;
    for (uint32_t k = 0; k < N; k++)
      row[k] = load_iq<float>(src, dtype, (uint64_t)b * N + k);
    fft_inplace<float>(row.data(), N, 0, tw.data());
    float *yo = y_work + 2 * ((uint64_t)l * M + b) * S;
    for (uint32_t i = 0; i < S; i++) {
      cf v = row[(i + start + N / 2) % N];
      yo[2 * i] = v.real();
      yo[2 * i + 1] = v.imag();
    }
  }

  const uint64_t row_len = cb_stride;
  const uint64_t n_valid = std::min<uint64_t>((uint64_t)S * Qm, cb_size);
  const uint64_t hrow = (n_valid + 7) / 8;
  if (hard_bytes) memset(hard_bytes, 0, hrow * K * U);
#pragma omp parallel for schedule(dynamic)
  for (int64_t lg = 0; lg < (int64_t)U * G; lg++) {
    uint32_t l = (uint32_t)(lg / G), g = (uint32_t)(lg % G);
    const float *y = y_work + 2 * (uint64_t)l * M * S;
    const float *w = csi_work + 2 * (uint64_t)g * M * K;
    uint32_t s_end = std::min(S, (g + 1) * sg);
    for (uint32_t s = g * sg; s < s_end; s++)
      for (uint32_t u = 0; u < K; u++) {
        float xr = 0, xi = 0;
        for (uint32_t b = 0; b < M; b++) {
          float wr = w[2 * (b * K + u)], wi = w[2 * (b * K + u) + 1];
          float yr = y[2 * ((uint64_t)b * S + s)], yi = y[2 * ((uint64_t)b * S + s) + 1];
          xr += wr * yr - wi * yi;
          xi += wr * yi + wi * yr;
        }
        uint16_t lv[8];
        orc_demod(Qm, xr, xi, lv);
        uint64_t t0 = (uint64_t)s * Qm, cb = t0 / cb_size;
        uint16_t *lo = llr + ((uint64_t)l * K + u) * row_len;
        if (cb < 1) {
          uint64_t base = zeros + t0 % cb_size;
          for (int q = 0; q < Qm; q++)
            if (base + q < row_len) lo[base + q] = lv[q];
        }
        if (hard_bytes)
          for (int q = 0; q < Qm; q++) {
            uint64_t t = t0 + q;
            if (t >= n_valid) break;
            uint8_t h = (orc_h2f(lv[q]) < 0.f) ? 1 : 0;
            h ^= seq_bits[t % seq_len];
            if (h) {
              uint8_t *hb = hard_bytes + ((uint64_t)l * K + u) * hrow + t / 8;
#pragma omp atomic
              *hb |= (uint8_t)(1u << (7 - t % 8));
            }
          }
      }
  }
  return bad;
}

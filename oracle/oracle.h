/*
 * oracle.h -- CPU restatement of the MegaStation per-slot baseband operators.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py use it, as the checker and as the timed host baseline.
 *
 * Every function cites the reference file:line whose behaviour it restates
 * (paths relative to the MegaStation source tree).  Two precisions exist:
 *   - FP64 functions (orc_*): the accuracy oracle for the GPU path;
 *   - reference-faithful FP32/FP16 details where bit-exactness matters
 *     (pilot tables, demodulation in half arithmetic, IFFT quantisation).
 * Parity is pinned by the golden vectors of the reference's own unit tests
 * (test/fft, test/beamform, test/sgemv), committed under tests/golden/.
 *
 * Complex arrays are interleaved (re, im) float or double.
 * IQ dtype codes: 0 = complex float32, 1 = int16 IQ, 2 = int8 IQ, 3 = fp16 IQ.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* IEEE binary16 conversions (round to nearest even). */
uint16_t orc_f2h(float f);
float orc_h2f(uint16_t h);

/* ---- sequences (src/operators/utils.h:54-95, fft/fft_op.cu:176-192) ---- */
void orc_zadoff_chu(uint64_t len, float *out);
void orc_cyclic_shift(const float *in, float *out, uint64_t len, float alpha);
void orc_pilot_sign(uint64_t S, float *out);
/* per-user DM-RS table of the modulator (modulation/modulation.cu:82-86) */
void orc_dmrs_table(uint64_t S, uint64_t K, float *out);

/* ---- scrambler (scrambler/scrambler.cu:22-31, scrambler_kernel.cuh:36-56) */
void orc_scrambler_seq127(uint8_t *seq);
void orc_scramble_bytes(uint8_t *out, const uint8_t *in, uint64_t num_bytes,
                        uint64_t batch);
/* 3GPP TS 38.211 5.2.1 length-31 Gold sequence c(n), n in [0, n_bits) */
void orc_gold_seq(uint32_t c_init, uint64_t n_bits, uint8_t *bits);

/* ---- modulation (modulation/modulation.cu:22-72, modulation_kernel.cuh) - */
void orc_mod_table(int Qm, float *table);
void orc_modulate(const uint8_t *in, float *out, uint64_t in_bytes,
                  uint64_t num_carriers, uint64_t num_ues, int Qm,
                  uint32_t pilot_spacing, const float *pilot_table);
/* soft demapper in half arithmetic (modulation/demodulation.h:30-67) */
void orc_demod(int Qm, float re, float im, uint16_t *llr);

/* ---- FFT operators (fft/fft_op.cu, fft_callback.cuh, ifft_callback.cuh) - */
void orc_fft_d(double *x, uint32_t n, int inverse);
void orc_uplink_fft(const void *in, int dtype, uint32_t M, uint32_t N,
                    uint32_t S, uint32_t start, float *out);
void orc_pilot_fft(const void *in, int dtype, uint32_t M, uint32_t N,
                   uint32_t S, uint32_t start, uint32_t K, uint32_t sg,
                   uint32_t ue_start, const float *pilot_sign, float *csi);
void orc_ifft_downlink(const float *in, uint32_t M, uint32_t N, int out_dtype,
                       void *out);

/* ---- zero forcing (beamform/beamform.cu:74-122, beam_utils.cuh:40-80) -- */
int orc_zf(const float *csi, uint32_t G, uint32_t M, uint32_t K, uint32_t S,
           uint32_t sg, float *W, double *cond);
void orc_precoder(const float *W, uint32_t G, uint32_t M, uint32_t K,
                  float *P);

/* ---- equalize / precode (sgemv/equalize_kernel.cuh, precode_kernel.cuh) */
/* x[u][s] = sum_b W[g][b][u] y[b][s] in FP64; LLRs follow the production
 * kernel's placement (equalize_kernel.cuh:272-287,330-352): the Qm LLRs of
 * subcarrier s start at (t/cb)*cb_stride + zeros + t%cb, t = s*Qm, and are
 * dropped when t/cb >= cb_blocks.  Hard bits (llr < 0) of stream bits
 * t < min(S*Qm, cb*cb_blocks) are XORed with seq[u*seq_user_stride +
 * t % seq_len] and packed MSB-first (the scrambler's byte convention,
 * scrambler_kernel.cuh:43-50).  x_out, hard_bytes may be NULL. */
void orc_equalize(const float *W, const float *y, uint32_t K, uint32_t M,
                  uint32_t S, uint32_t sg, int Qm, uint64_t cb_size,
                  uint64_t cb_stride, uint64_t zeros, uint32_t cb_blocks,
                  uint16_t *llr, float *x_out, const uint8_t *seq_bits,
                  uint64_t seq_len, uint64_t seq_user_stride,
                  uint8_t *hard_bytes);
void orc_precode(const float *P, const float *s, uint32_t M, uint32_t K,
                 uint32_t S, uint32_t sg, uint32_t N, uint32_t start,
                 float *out);

/* ---- LDPC sizing (config/config.cc:84-135, ldpc/config.h:27-73) -------- */
void orc_ldpc_sizes(uint64_t S, int Qm, double rate, int base_graph,
                    uint64_t pilot_spacing, int downlink, uint64_t *encoded,
                    uint64_t *punctured, uint64_t *decoded);

/* ---- host baseline: one uplink slot, FP32, OpenMP ---------------------- */
int orc_slot_uplink_cpu(const void *iq, int dtype, uint32_t P, uint32_t U,
                        uint32_t M, uint32_t K, uint32_t N, uint32_t S,
                        uint32_t sg, int Qm, uint64_t cb_size,
                        uint64_t cb_stride, uint64_t zeros,
                        const float *pilot_sign, const uint8_t *seq_bits,
                        uint64_t seq_len, float *csi_work, float *y_work,
                        uint16_t *llr, uint8_t *hard_bytes, int threads);

#ifdef __cplusplus
}
#endif

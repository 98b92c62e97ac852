/*
 * megastation_b200.h -- C ABI of the B200-native (sm_100a) MegaStation
 * per-slot baseband hot path.
 *
 * Plain C: pointers, sizes and status codes; no C++ or torch types.  Every
 * device pointer is caller-owned device memory; every `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).  Operators
 * own only their scratch and tables, sized at create time; no entry point
 * allocates device memory on the hot path.  No function throws; each
 * returns an mb_status.
 *
 * Layouts follow the reference's Matrix convention (dims[0] fastest,
 * src/operators/matrix/matrix.h:95-117), written here slowest-first:
 *   IQ samples       [sym][M][N]   complex (c32, or int16/int8/fp16 pairs)
 *   uplink FFT out   [sym][M][S]   c32          (baseband/buffers.cc:87-88)
 *   CSI / detector W [G][M][K]     c32          (buffers.cc:77-78)
 *   precoder P       [G][K][M]     c32          (buffers.cc:79-80)
 *   LLR              [sym][K][cb_stride*cb_blocks] fp16 (buffers.cc:96-99,
 *                    tight stride: cb_stride >= zeros + cb_size)
 *   user symbols     [sym][K][S]   c32          (buffers.cc:135-136)
 *   precoded         [sym][M][N]   c32          (buffers.cc:140-141)
 * with M antennas, K users, N FFT size, S data subcarriers, sg subcarrier
 * group size and G = ceil(S / sg) groups.
 *
 * Threading (as in the reference, scheduler/gpu_engine.cc:77-430): a handle
 * is used by one host thread / one stream at a time; distinct handles are
 * independent.  mb_tables_init is idempotent and thread-safe.
 */
#ifndef MEGASTATION_B200_H_
#define MEGASTATION_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MB_OK = 0,
  MB_BAD_SHAPE = 1,    /* sizes inconsistent or outside supported range */
  MB_BAD_ARG = 2,      /* NULL pointer, bad enum, misaligned buffer */
  MB_NOT_PD = 3,       /* a Gram matrix was not positive definite */
  MB_CUDA_ERROR = 4,   /* a CUDA runtime call failed */
  MB_TIMEOUT = 5,      /* a bounded device-side wait gave up */
  MB_NO_MEMORY = 6,    /* create-time allocation failed */
  MB_UNSUPPORTED = 7,  /* valid request this build does not implement */
  MB_TOO_LARGE = 8     /* request needs more than mb_equalize_tc_noalloc's
                          fixed scratch */
} mb_status;

typedef enum {
  MB_IQ_C32 = 0, /* complex float32 */
  MB_IQ_I16 = 1, /* int16 I/Q pairs, value / 32768 (fft_utils.h:19-22) */
  MB_IQ_I8 = 2,  /* int8 I/Q pairs, value / 128 (QuanT = char, types.h:26) */
  MB_IQ_F16 = 3  /* fp16 I/Q pairs */
} mb_iq_dtype;

typedef struct {
  float re, im;
} mb_c32;

typedef struct mb_mlp mb_mlp; /* the learned initialiser's network (below) */
typedef struct mb_ldpc mb_ldpc; /* an LDPC code over a caller-supplied base graph (below) */

const char *mb_status_str(mb_status s);
/* Version string of this library build. */
const char *mb_version(void);

/* ------------------------------------------------------------- tables --- */
/* Per-device constant tables (QAM maps, 127-bit scrambler sequence, FFT
 * twiddles).  Replaces Modulation::init / Scrambler::init / PilotSign::init
 * (modulation/modulation.cu:78-113, scrambler/scrambler.cu:22-38,
 * fft/fft_op.cu:176-192); idempotent and thread-safe.  Called implicitly by
 * every create function for the current device. */
mb_status mb_tables_init(int device);

/* Device error word of the current device: bits set by kernels whose
 * bounded waits gave up (1 = mbarrier wait timeout), OR-ed with the word of
 * mb_equalize_tc_noalloc's kernels.  Synchronises the device, copies the
 * word to *out and clears both when clear != 0. */
mb_status mb_device_error(int *out, int clear);

/* Self-test of the bounded device wait (no reference counterpart): one
 * warp waits on a shared-memory mbarrier through the wait the tensor-core
 * kernels use, giving up after limit_ns (1 .. 1e9) nanoseconds.  With
 * arm = 0 nothing arrives, the wait runs out and mb_device_error then
 * reports the timeout bit (1); with arm != 0 the barrier completes and no
 * bit is set.  Shows, without faulting or hanging the GPU, that an expired
 * wait ends the kernel with an error the host can read. */
mb_status mb_selftest_wait(uint64_t limit_ns, int arm, void *stream);

/* Host-side pilot sequence p/|p|^2 of length S (fft/fft_op.cu:176-192 over
 * utils.h:54-95).  out: S host complex values. */
mb_status mb_pilot_sign(uint64_t S, mb_c32 *out);
/* Host-side per-user DM-RS table [K][S] (modulation/modulation.cu:82-86). */
mb_status mb_dmrs_table(uint64_t S, uint64_t K, mb_c32 *out);
/* LDPC code-block sizing of config/config.cc:84-135 (TS 38.212 lifting
 * sizes; BG1 22 / BG2 10 information columns, 2 punctured columns). */
mb_status mb_ldpc_sizes(uint64_t S, uint32_t Qm, double code_rate,
                        uint32_t base_graph, uint64_t pilot_spacing,
                        int downlink, uint64_t *encoded_bits,
                        uint64_t *punctured_bits, uint64_t *decoded_bits);

/* ---------------------------------------------------------------- FFT --- */
/* Replaces UplinkFFT / PilotFFT / DownlinkIFFT (fft/fft_op.h:50-120).  One
 * handle per (start, N, S, M, K, sg) shape, like the reference objects
 * constructed per frame (baseband/process.cc:66-87).  N is a power of two
 * in [16, 8192]; S <= N; start + S <= N is not required (indices wrap mod N
 * as in fft_callback.cuh:52-53). */
typedef struct {
  uint32_t ofdm_start; /* first data subcarrier, (N - S) / 2 (config.cc:31) */
  uint32_t ofdm_ca;    /* N, FFT size */
  uint32_t ofdm_num;   /* S, data subcarriers */
  uint32_t bs_num;     /* M, antennas */
  uint32_t ue_num;     /* K, users (pilot FFT only) */
  uint32_t sc_group;   /* sg, subcarrier group (pilot FFT only) */
} mb_fft_desc;

typedef struct mb_fft mb_fft;
mb_status mb_fft_create(const mb_fft_desc *desc, mb_fft **out);
mb_status mb_fft_destroy(mb_fft *fft);

/* UplinkFFT::operator() (fft/fft_op.cu:135-143): for n_sym symbols, the
 * unnormalised forward FFT of each antenna row with the shift gather
 * out[b][i] = X[b][(i + start + N/2) % N], i < S.  iq: [n_sym][M][N],
 * out: [n_sym][M][S]. */
mb_status mb_fft_uplink(mb_fft *fft, const void *iq, int iq_dtype,
                        uint32_t n_sym, mb_c32 *out, void *stream);

/* Mixed-precision uplink FFT (no reference counterpart; same transform and
 * shift gather as mb_fft_uplink): the output is planar BF16 rows
 * out[n_sym][re|im][M][row_pitch], subcarrier i < S at column i, the layout
 * the tensor-core equalizer reads.  Columns from S up to S rounded up to a
 * multiple of 8 may be overwritten with other FFT bins; columns beyond that
 * are left as they are.  For N = 4096 with row_pitch % 8 == 0 and 16-byte
 * aligned buffers the butterflies run on the tensor cores (FP16 operands
 * scaled per row by a power of two, FP32 accumulation); otherwise in FP32. */
mb_status mb_fft_uplink_bf16(mb_fft *fft, const void *iq, int iq_dtype,
                             uint32_t n_sym, void *out, uint32_t row_pitch,
                             void *stream);

/* PilotFFT::operator()(in, out, ue_start) (fft/fft_op.cu:145-165): symbol p
 * of n_sym carries the comb pilots of users ue_start + p*sg + (i % sg); the
 * LS estimate conj(X)*p/|p|^2 of subcarrier i is stored at
 * csi[i/sg][b][u] (fft_callback.cuh:76-108).  csi: [G][M][K]. */
mb_status mb_fft_pilot(mb_fft *fft, const void *iq, int iq_dtype,
                       uint32_t n_sym, uint32_t ue_start, mb_c32 *csi,
                       void *stream);

/* Mixed-precision pilot FFT (no reference counterpart): the contract of
 * mb_fft_pilot; for N = 4096 with a 16-byte aligned input the butterflies
 * run on the tensor cores (FP16 operands scaled per row by a power of two,
 * FP32 accumulation), otherwise it is mb_fft_pilot. */
mb_status mb_fft_pilot_mixed(mb_fft *fft, const void *iq, int iq_dtype,
                             uint32_t n_sym, uint32_t ue_start, mb_c32 *csi,
                             void *stream);

/* DownlinkIFFT::operator() (fft/fft_op.cu:167-174, ifft_callback.cuh:21-59):
 * unnormalised inverse FFT of each [M][N] row, then for int16/int8 outputs
 * q = saturate(rint(x * (max+1) / N)); for MB_IQ_F16 / MB_IQ_C32 outputs
 * x / N.  in: [n_sym][M][N] c32, out: [n_sym][M][N] pairs of out_dtype. */
mb_status mb_ifft_downlink(mb_fft *fft, const mb_c32 *in, uint32_t n_sym,
                           void *out, int out_dtype, void *stream);

/* Mixed-precision inverse FFT (no reference counterpart; the transform and
 * quantiser of mb_ifft_downlink): in [n_sym][M][N] pairs of in_dtype
 * (MB_IQ_C32 or MB_IQ_F16), out [n_sym][M][N] pairs of out_dtype.  For
 * N = 4096, 16-byte aligned buffers and int16, int8 or FP16 outputs the
 * butterflies run on the tensor cores (FP16 operands scaled per row by a
 * power of two, FP32 accumulation); otherwise mb_ifft_downlink (c32 input
 * only: MB_UNSUPPORTED for FP16 input then). */
mb_status mb_ifft_downlink_mixed(mb_fft *fft, const void *in, int in_dtype, uint32_t n_sym, void *out,
                                 int out_dtype, void *stream);

/* ------------------------------------------------------- zero forcing --- */
/* Replaces Beamform (beamform/beamform.h:27-84). */
typedef enum {
  /* FP32 Gram + FP32 Cholesky + triangular solves: the reference's math
   * (cuBLAS Cgemm + cuSOLVER potrf/potrs, beamform.cu:74-122) */
  MB_ZF_FP32 = 0,
  /* BF16 Gram on tensor cores (FP32 accumulate), FP32 inverse refined by
   * Newton-Schulz, FP64 Cholesky for groups above cond_threshold */
  MB_ZF_MIXED = 1,
  /* FP64 Cholesky for every group */
  MB_ZF_FP64 = 2
} mb_zf_precision;

typedef struct {
  uint32_t precision;     /* mb_zf_precision */
  uint32_t ns_iters;      /* Newton-Schulz refinements (MIXED), e.g. 2 */
  float cond_threshold;   /* FP64 fallback above this estimate, e.g. 1e4 */
  uint32_t init;          /* MIXED initial iterate: 0 = exact inverse (FP32
                             Gauss-Jordan); 1 = learned polynomial
                             (mb_zf_set_init_net), exact inverse where the
                             learned iterate is not accepted */
} mb_zf_opts;

typedef struct mb_zf mb_zf;
/* Beamform(num_bs, num_ue, max_batch) (beamform.cu:19-31). */
mb_status mb_zf_create(uint32_t num_bs, uint32_t num_ue, uint32_t max_groups,
                       mb_zf **out);
mb_status mb_zf_destroy(mb_zf *zf);

/* Beamform::beamform_uplink (beamform.cu:74-122, 144-152): for each group g,
 * C = csi[g] viewed as K x M column-major, W = (C C^H)^{-1} C overwrites
 * csi[g].  S and sc_group locate a short last group (S % sg != 0), whose
 * users without a pilot subcarrier take group G-2's estimate.
 * group_status (device, nullable): per group 0 = ok, 1 = not positive
 * definite (W zeroed), 2 = solved on the FP64 fallback.  When not NULL,
 * group_cond (device) receives the condition estimate per group. */
mb_status mb_zf_uplink(mb_zf *zf, mb_c32 *csi, uint32_t groups, uint32_t S,
                       uint32_t sc_group, const mb_zf_opts *opts,
                       int32_t *group_status, float *group_cond,
                       void *stream);

/* Learned initial iterate of the mixed ZF (no reference counterpart): the
 * network net (an mb_mlp with 6 inputs, width <= 256 and 4 outputs; not
 * owned, read at every launch, so later training takes effect) maps six
 * scale-free spectral features of a group's Gram G to the coefficients a of
 * X0 = (a0 I + a1 Gn + a2 Gn^2 + a3 Gn^3) / tau, Gn = G / tau,
 * tau = tr(G) / K; the features, with t_k = tr(Gn^k) / K: t2 - 1,
 * t3 - 3 t2 + 2, t4 - 4 t3 + 6 t2 - 3, min and max of diag(Gn) minus 1,
 * K / M.  ns_iters Newton-Schulz steps follow (at most two more while
 * 0.04 < ||I - G X||_F < 0.3); a group whose last residual before the final
 * step exceeds 0.04 is solved by the exact inverse instead.  Used when
 * mb_zf_opts.init = 1; group_status then reports 3 for groups solved from
 * the learned iterate.  net NULL clears it. */
mb_status mb_zf_set_init_net(mb_zf *zf, const mb_mlp *net);

/* Training data of that network (no reference counterpart): for each group
 * g of csi [G][M][K] (K <= 64), in FP64, features [G][6] as above and the
 * quadratic form of the normalised squared residual,
 * ||I - Gn p_a(Gn)||_F^2 / K = a^T A a - 2 b^T a + 1 with A [G][4][4],
 * A_ij = t_(i+j+2), and b [G][4], b_i = t_(i+1) (device FP32 outputs; the
 * mb_mlp_loss_grad loss with c = 1). */
mb_status mb_zf_init_targets(const mb_c32 *csi, uint32_t groups, uint32_t M, uint32_t K,
                             float *features, float *A, float *b, void *stream);

/* Beamform::beamform_downlink (beamform.cu:154-168, beam_utils.cuh:40-80):
 * P[g][u][b] = W[g][b][u] / max_{b,u} |W[g][b][u]|. */
mb_status mb_zf_precoder(const mb_c32 *W, mb_c32 *P, uint32_t num_bs,
                         uint32_t num_ue, uint32_t groups, void *stream);

/* ----------------------------------------------------- equalize + demod -- */
typedef struct mb_scrambler mb_scrambler;
typedef enum {
  /* 127-periodic x^7+x^4+1 LFSR from state 0x5D, shared by all users
   * (scrambler/scrambler.cu:22-31): the reference's sequence */
  MB_SCR_LFSR127 = 0,
  /* TS 38.211 5.2.1 Gold sequence per user, c_init(u) = c_init + u */
  MB_SCR_GOLD = 1
} mb_scrambler_mode;
mb_status mb_scrambler_create(int mode, uint32_t c_init, uint32_t num_ue,
                              uint64_t num_bits, mb_scrambler **out);
mb_status mb_scrambler_destroy(mb_scrambler *scr);

/* Equalize::equalize (sgemv/equalize.h:70-73, equalize.cu:53-67) batched
 * over n_sym symbols: x[u][s] = sum_b W[g(s)][b][u] y[b][s], g(s) = s / sg,
 * then the soft demapper (modulation/demodulation.h:30-67) in FP16.  The Qm
 * LLRs of subcarrier s start at (t/cb_size)*cb_stride + zeros +
 * t % cb_size, t = s*Qm, and are dropped when t/cb_size >= cb_blocks
 * (equalize_kernel.cuh:272-287).  Slots outside the written positions are
 * left untouched.
 * hard (nullable): descrambled hard decisions (llr < 0) of stream bits
 * t < min(S*Qm, cb_size*cb_blocks), packed MSB-first per (symbol, user)
 * row of ceil(n/8) bytes; requires sg*Qm % 8 == 0.  scr NULL means no
 * descrambling.  x (nullable): the equalized symbols [n_sym][K][S].
 * y: [n_sym][M][S], llr: [n_sym][K][cb_stride*cb_blocks]. */
mb_status mb_equalize(const mb_c32 *W, const mb_c32 *y, uint32_t K,
                      uint32_t M, uint32_t S, uint32_t sg, uint32_t n_sym,
                      uint32_t Qm, uint64_t cb_size, uint64_t cb_stride,
                      uint64_t zeros, uint32_t cb_blocks, uint16_t *llr,
                      uint8_t *hard, const mb_scrambler *scr, mb_c32 *x,
                      void *stream);

/* Mixed-precision equalize on the tensor cores (no reference counterpart;
 * same contract and outputs as mb_equalize): BF16 W and y, FP32
 * accumulation (tcgen05.mma), the same FP16 demapper and layouts.  The
 * caller provides two device scratch buffers whose sizes
 * mb_equalize_tc_scratch returns.  Requires sg % 8 == 0 and K <= 64. */
mb_status mb_equalize_tc_scratch(uint32_t K, uint32_t M, uint32_t S,
                                 uint32_t sg, uint32_t n_sym,
                                 uint64_t *img_bytes, uint64_t *ylp_bytes);
mb_status mb_equalize_tc(const mb_c32 *W, const mb_c32 *y, uint32_t K,
                         uint32_t M, uint32_t S, uint32_t sg, uint32_t n_sym,
                         uint32_t Qm, uint64_t cb_size, uint64_t cb_stride,
                         uint64_t zeros, uint32_t cb_blocks, uint16_t *llr,
                         uint8_t *hard, const mb_scrambler *scr, mb_c32 *x,
                         void *scratch_img, void *scratch_ylp, void *stream);

/* The same mixed-precision equalize for callers that cannot allocate device
 * memory (no counterpart in the reference): hosts whose real-time threads
 * may not enter the driver's allocator, or whose device memory is fixed at
 * start-up by a framework that owns every allocation.  Inputs, outputs and
 * results are those of mb_equalize_tc, but the scratch lives in one 32 MiB
 * array compiled into the library (held by every device that loads it until
 * the process exits), so the caller passes no scratch and nothing is
 * allocated or freed.  Limit: the BF16 detector images of all groups plus
 * the BF16 rows of one symbol, 4*M*ceil8(S) bytes, must fit in 32 MiB;
 * larger requests return MB_TOO_LARGE (e.g. 256 antennas x 32 users with
 * 3276 subcarriers fits; symbols beyond what fits are processed in turn).
 * The first call on each device looks the array's device address up with
 * cudaGetSymbolAddress (device current); make that first call before any
 * stream capture.  All calls on a device share the array and it keeps the
 * previous call's contents: calls that can overlap on the GPU (different
 * streams, other host threads) race and must be serialised by the caller.
 * Nothing in the scratch needs to start at zero: every byte a call reads was
 * written earlier in the same call.  A bounded device wait that gives up
 * sets bit 1 of an error word that is also fixed in the library (the
 * library's own word is allocated on first use); mb_device_error reports
 * and clears it together with that word.  The device addresses looked up
 * at the first call belong to the device's context: after cudaDeviceReset
 * this entry point must not be called again in the process. */
mb_status mb_equalize_tc_noalloc(const mb_c32 *W, const mb_c32 *y, uint32_t K,
                                 uint32_t M, uint32_t S, uint32_t sg,
                                 uint32_t n_sym, uint32_t Qm, uint64_t cb_size,
                                 uint64_t cb_stride, uint64_t zeros,
                                 uint32_t cb_blocks, uint16_t *llr,
                                 uint8_t *hard, const mb_scrambler *scr,
                                 mb_c32 *x, void *stream);

/* ------------------------------------------------------------ precode --- */
/* Precode::precode (sgemv/precode.h:59-61, precode_kernel.cuh:255-262)
 * batched over n_sym symbols: out[b][(s + start + N/2) % N] =
 * sum_u P[g(s)][u][b] s[u][s]; unlike the reference every guard bin of the
 * N-row is written as zero.  s: [n_sym][K][S], out: [n_sym][M][N]. */
mb_status mb_precode(const mb_c32 *P, const mb_c32 *s, uint32_t M,
                     uint32_t K, uint32_t S, uint32_t sg, uint32_t N,
                     uint32_t start, uint32_t n_sym, mb_c32 *out,
                     void *stream);

/* Mixed-precision precode on the tensor cores (no reference counterpart;
 * the contract of mb_precode): z [n_sym][M][N] FP16 (re, im) pairs at the
 * data bins (s + start + N/2) mod N; the guard bins are left as they are
 * (zero them once).  BF16 operands, FP32 accumulation (tcgen05.mma): a CTA
 * per subcarrier group, 128 antennas and up to 128 (symbol, subcarrier)
 * columns.  The caller provides a device scratch buffer of
 * mb_precode_tc_scratch bytes for the BF16 precoder images (built from P
 * in the call).  Requires K <= 64. */
mb_status mb_precode_tc_scratch(uint32_t M, uint32_t K, uint32_t S, uint32_t sg, uint64_t *img_bytes);
mb_status mb_precode_tc(const mb_c32 *P, const mb_c32 *s, uint32_t M, uint32_t K, uint32_t S,
                        uint32_t sg, uint32_t N, uint32_t start, uint32_t n_sym, void *z,
                        void *scratch_img, void *stream);

/* -------------------------------------------------- modulate / scramble -- */
/* Modulation::modulate (modulation/modulation.cu:115-128,
 * modulation_kernel.cuh:37-68): bits of user u (in_bytes per user, LSB
 * first) to Gray QAM; with pilot_spacing > 0 every pilot_spacing-th
 * subcarrier carries pilot_table[u][c] (device, [K][S]).  out: [K][S]. */
mb_status mb_modulate(const uint8_t *in, mb_c32 *out, uint64_t in_bytes,
                      uint64_t num_carriers, uint64_t num_ues, uint32_t Qm,
                      uint32_t pilot_spacing, const mb_c32 *pilot_table,
                      void *stream);

/* Scrambler::scrambler (scrambler/scrambler.cu:40-50,
 * scrambler_kernel.cuh:36-56): out[j] = in[j] ^ (8 sequence bits, first in
 * the MSB); in == out allowed.  [batch][num_bytes]. */
mb_status mb_scramble(uint8_t *out, const uint8_t *in, uint64_t num_bytes,
                      uint64_t batch, void *stream);


/* --------------------------------------------------------- slot runner --- */
/* Single-GPU stage sequencer replacing BandProcess::process
 * (baseband/process.cc:134-225) and the multi-GPU scheduler
 * (scheduler/gpu_engine.cc:253-409): per slot, the pilot FFT of all P pilot
 * symbols (one launch), the ZF detector (+ downlink precoder) over all
 * groups, then uplink FFT + equalize/demod/descramble in batches of
 * sym_batch symbols, on one stream with a side stream that overlaps the
 * first uplink FFT batch with the ZF solve.  All buffers are allocated at
 * create; a slot call allocates nothing. */
typedef struct {
  uint32_t M, K, N, S, sg, Qm;  /* antennas, users, FFT, data subcarriers */
  uint32_t P, U, D;             /* pilot, uplink, downlink symbols */
  int32_t iq_dtype;             /* mb_iq_dtype of the uplink samples */
  uint64_t cb_size, cb_stride, zeros; /* uplink LLR layout, one code block */
  uint32_t zf_precision;        /* mb_zf_precision */
  uint32_t ns_iters;
  float cond_threshold;
  uint32_t scrambler_mode;      /* mb_scrambler_mode; descrambles hard bits */
  uint32_t c_init;
  int32_t out_dtype;            /* downlink IFFT output mb_iq_dtype */
  uint32_t sym_batch;           /* uplink symbols per FFT/equalize batch */
  uint32_t use_graph;           /* replay the uplink slot as a CUDA graph */
} mb_cell_desc;

typedef struct mb_slot mb_slot;
mb_status mb_slot_create(const mb_cell_desc *cell, mb_slot **out);
mb_status mb_slot_destroy(mb_slot *slot);

/* One uplink slot: iq [P+U][M][N] (device) -> llr [U][K][cb_stride] fp16,
 * hard [U][K][ceil(min(S*Qm, cb_size)/8)] (nullable).  group_status
 * (device, nullable) [G] as in mb_zf_uplink. */
mb_status mb_slot_uplink(mb_slot *slot, const void *iq, uint16_t *llr,
                         uint8_t *hard, int32_t *group_status, void *stream);

/* Downlink of the same slot: precode the D symbol vectors [D][K][S] with
 * the precoder of the last uplink ZF, then IFFT to out [D][M][N] pairs of
 * out_dtype. */
mb_status mb_slot_downlink(mb_slot *slot, const mb_c32 *symbols, void *out,
                           void *stream);

/* The downlink branch of BandProcess::process (baseband/process.cc:196-214)
 * from encoded bits: Modulation::modulate of each downlink symbol's K user
 * rows (bits [D][K][in_bytes], in_bytes >= ceil(S Qm / 8); stream bit t is
 * bit t % 8 of byte t / 8, and the first of a subcarrier's Qm bits is the
 * MSB of its QAM index, modulation.cu:115-128), then mb_slot_downlink.  The
 * reference scrambles and LDPC-encodes the MAC bits before (process.cc:
 * 198-201); those bits come from the caller's encoder. */
mb_status mb_slot_downlink_bits(mb_slot *slot, const uint8_t *bits, uint64_t in_bytes, void *out,
                                void *stream);

/* The rest of the uplink branch of BandProcess::process (process.cc:
 * 186-189): LDPC-decode every (symbol, user) LLR row of the last uplink
 * (one code block per row, llr as mb_slot_uplink wrote it) and descramble
 * the decoded bits (Scrambler::scrambler, the LFSR mode).  mb_slot_set_ldpc
 * attaches the code (not owned; NULL detaches), which must fit the cell's
 * layout: zeros = 2Z, cb_size = (kb - 2 + parity_nodes) Z, cb_stride >=
 * (kb + parity_nodes) Z; max_iter 1 .. 32; with downlink symbols it also
 * allocates the buffers of mb_slot_downlink_info.  decoded: [U][K][ceil(kb
 * Z / 8)] bytes, MSB first. */
mb_status mb_slot_set_ldpc(mb_slot *slot, mb_ldpc *code, uint32_t max_iter);
mb_status mb_slot_decode(mb_slot *slot, const uint16_t *llr, uint8_t *decoded, void *stream);
/* The whole downlink branch of BandProcess::process (process.cc:196-214)
 * from information bits [D][K][ceil(kb Z / 8)] (MSB first): scramble (the
 * LFSR mode), LDPC-encode with the attached code, modulate, precode,
 * inverse FFT into out as mb_slot_downlink.  Codeword bits past the code
 * block up to S Qm are zero.  mb_slot_set_ldpc allocates its buffers. */
mb_status mb_slot_downlink_info(mb_slot *slot, const uint8_t *info, void *out, void *stream);

/* Single-GPU slot pipeline over host buffers (scheduler/gpu_engine.cc:77-437
 * and cpu_buffer.cc:5-49 for one GPU): each submitted slot's samples are
 * copied to a ring of `depth` device buffers, the slot runs (an mb_slot
 * with this cell description), and its FP16 LLRs and hard bits are copied
 * back, on three streams ordered by events, so the samples of slot k+1
 * cross PCIe while slot k computes and slot k-1's results come back.
 * mb_pipe_submit does not block; the host buffers of a slot must stay valid
 * (and unmodified, for the samples) until mb_pipe_wait(ticket) returns MB_OK.
 * Pinned host memory (cudaHostAlloc) lets the copies overlap; pageable
 * memory works but copies synchronously.  Sizes: mb_pipe_io_bytes.
 * mb_pipe_wait gives up after timeout_ms (UINT32_MAX: no limit) with
 * MB_TIMEOUT; the slot's work stays queued. */
typedef struct mb_pipe mb_pipe;
mb_status mb_pipe_create(const mb_cell_desc *cell, uint32_t depth, mb_pipe **out);
mb_status mb_pipe_destroy(mb_pipe *pipe);
mb_status mb_pipe_io_bytes(const mb_pipe *pipe, uint64_t *iq_bytes,
                           uint64_t *llr_bytes, uint64_t *hard_bytes);
mb_status mb_pipe_submit(mb_pipe *pipe, const void *iq_host, uint16_t *llr_host,
                         uint8_t *hard_host, uint64_t *ticket);
mb_status mb_pipe_wait(mb_pipe *pipe, uint64_t ticket, uint32_t timeout_ms);
/* The pipeline's slots take the mixed ZF's learned initial iterate
 * (mb_slot_set_zf_init); waits for the slots in flight first. */
mb_status mb_pipe_set_zf_init(mb_pipe *pipe, const mb_mlp *net);
/* Device timer: after mb_pipe_timer_start, the next submitted slot records
 * a start event before its sample copy and every slot after it an end
 * event after its result copies; mb_pipe_timer_ms waits for the last end
 * event and returns the device time between the two (CUDA events). */
mb_status mb_pipe_timer_start(mb_pipe *pipe);
mb_status mb_pipe_timer_ms(mb_pipe *pipe, double *ms);

/* Stage timing.  mb_slot_timing(slot, n) makes the next n slot calls record
 * CUDA events around each stage on the launching stream (0 disables);
 * mb_slot_stage_ms waits for those events and returns, summed over the
 * recorded calls (while timing, every kernel runs alone on the launching
 * stream, the first FFT batch included): [0] pilot FFT, [1] ZF (+ tail
 * fill), [2] uplink FFT batches, [3] equalize, [4] whole slot,
 * [5] number of uplink FFT launches timed in [2], [6] equalize launches
 * (0 when the mixed-precision slot equalized inside its ZF kernel: one
 * batch of all uplink symbols, K <= 32, M <= 256, sc_group a multiple of
 * 16 and U * sc_group <= 128; the ZF stage [1] then holds both),
 * [7] recorded calls; then clears the record. */
mb_status mb_slot_timing(mb_slot *slot, uint32_t max_calls);
mb_status mb_slot_stage_ms(mb_slot *slot, double *out8);

/* The mixed-precision slot's ZF from the learned initial iterate of
 * mb_zf_set_init_net (net an mb_mlp of that shape, not owned; NULL: the
 * exact inverse).  Captured slot graphs are dropped and captured again. */
mb_status mb_slot_set_zf_init(mb_slot *slot, const mb_mlp *net);

/* Device views of the slot's internal buffers (for inspection and tests):
 * CSI/W [G][M][K], precoder [G][K][M].  In the mixed-precision path without
 * downlink symbols (D = 0) the equalizer reads only the detector images, and
 * the CSI/W buffer is left as ZF scratch. */
mb_status mb_slot_buffers(mb_slot *slot, mb_c32 **csi, mb_c32 **precoder);

/* -------------------------------------------------------- batched cells --- */
/* No counterpart in the reference, which processes one cell per
 * BandProcess.  A set of cells of uneven shape (each an mb_cell_desc) runs
 * one uplink slot per call as ONE CUDA graph launch: the graph forks into a
 * branch per cell (that cell's slot) and joins, so the cells' kernels run
 * concurrently.  Graphs are captured once per (pointer set, stream).  Every
 * argument array has one entry per cell, in creation order; llr, hard and
 * group_status arrays (and their entries) may be NULL as in
 * mb_slot_uplink.  stream must not be the legacy default stream. */
typedef struct mb_cells mb_cells;
mb_status mb_cells_create(const mb_cell_desc *cells, uint32_t ncells, mb_cells **out);
mb_status mb_cells_destroy(mb_cells *cells);
mb_status mb_cells_uplink(mb_cells *cells, const void *const *iq, uint16_t *const *llr,
                          uint8_t *const *hard, int32_t *const *group_status, void *stream);

/* Tuning knobs per cell: sym_batch (uplink symbols per FFT/equalize batch,
 * 1..U) and eq_cols (tensor-core equalizer (symbol, subcarrier) columns per
 * CTA, a multiple of 8 up to 128).  mb_cells_autotune measures the batched
 * slot (reps timed graph launches per candidate, CUDA events on stream) and
 * keeps, per class of equal-shaped cells, the fastest candidate by
 * coordinate descent; it writes the choice per cell (nullable outputs) and
 * the tuned time in microseconds per slot.  Outputs of the tuning launches
 * land in llr / hard. */
mb_status mb_cells_autotune(mb_cells *cells, const void *const *iq, uint16_t *const *llr,
                            uint8_t *const *hard, uint32_t reps, void *stream,
                            uint32_t *sym_batch_out, uint32_t *eq_cols_out,
                            double *us_per_slot);
mb_status mb_cells_get_tuning(const mb_cells *cells, uint32_t *sym_batch, uint32_t *eq_cols);
/* The third knob, per cell: the CTAs of each tensor-core FFT launch (cells
 * with N = 4096 in mixed precision; 0 = one per SM, the default).  A CTA
 * of that FFT holds a whole SM, so fewer CTAs (each taking more two-row
 * units) leave SMs to the other cells' kernels; mb_cells_autotune tries
 * 74, 37 and 18 per class after the other knobs. */
mb_status mb_cells_get_fft_ctas(const mb_cells *cells, uint32_t *fft_ctas);
mb_status mb_cells_set_fft_ctas(mb_cells *cells, const uint32_t *fft_ctas);
/* The fourth knob, per cell: where the mixed-precision ZF's inverse runs
 * its matrix products when K <= 32 -- 0 by K (the tensor cores for
 * 16 < K, the CUDA cores below; the default), 1 the CUDA cores, 2 the
 * tensor cores (tcgen05, split-BF16 operands, FP32 accumulation; its
 * round trips cost more than a small group's products).  mb_cells_autotune
 * tries the choice the rule did not make per class, last. */
mb_status mb_cells_get_zf_path(const mb_cells *cells, uint32_t *zf_path);
mb_status mb_cells_set_zf_path(mb_cells *cells, const uint32_t *zf_path);
mb_status mb_cells_set_tuning(mb_cells *cells, const uint32_t *sym_batch,
                              const uint32_t *eq_cols);

/* ----------------------------------------------------------------- LDPC --- */
/* LDPCEncoder / LDPCDecoder (ldpc/encoder.h:48-75, decoder.h:28-87, sized by
 * ldpc/config.h and config/config.cc:84-135), which the reference takes from
 * cuPHY.  The base graph is the caller's: the library ships no graph
 * tables.  It must have the block structure of both NR base graphs (TS
 * 38.212 5.3.2): block rows 0..3 over the kb information and the four core
 * parity columns kb..kb+3 (whose 4Z x 4Z block must be invertible), every
 * later row r with one more column kb + r, an identity block.  Entry k is
 * block (row[k], col[k]): the Z x Z identity with its columns cyclically
 * shifted right by shift[k] mod Z (row i has its one in column
 * (i + shift) mod Z), so the standard's V values can be passed as they are.
 * Host arrays, read at create. */
typedef struct {
  uint32_t kb;                 /* information block columns (22: BG1, 10: BG2) */
  uint32_t rows;               /* block rows given */
  uint32_t nnz;                /* entries */
  const uint16_t *row, *col, *shift;
} mb_ldpc_graph;
/* parity_nodes: block rows used (LDPCConfig::parity_nodes, 4 .. rows; the
 * code rate); max_batch: code blocks a decode launch keeps state for (a
 * larger batch is decoded in turns).  Z <= 384, at most 27 circulants per
 * row.  Allocates the graph tables, the core block's inverse and the
 * decoder's check-node state. */
mb_status mb_ldpc_create(const mb_ldpc_graph *graph, uint32_t Z, uint32_t parity_nodes, uint32_t max_batch,
                         mb_ldpc **out);
mb_status mb_ldpc_destroy(mb_ldpc *ldpc);
/* info [batch][info_stride] bytes, kb Z bits each, MSB first -> codewords
 * [batch][cw_stride] bytes: the (kb - 2 + parity_nodes) Z encoded bits after
 * the 2Z punctured systematic ones (cuPHY's puncture option, nrLDPCEncode),
 * MSB first: LDPCEncoder's output and the uplink LLR rows' cb_size. */
mb_status mb_ldpc_encode(mb_ldpc *ldpc, const uint8_t *info, uint64_t info_stride, uint8_t *codewords,
                         uint64_t cw_stride, uint32_t batch, void *stream);
/* llr [batch][llr_stride] FP16: the (kb + parity_nodes) Z LLRs of a code
 * block with the 2Z punctured ones first (zero), i.e. the equalizer's LLR
 * rows (zeros = 2Z, cb_size = (kb - 2 + parity_nodes) Z, cb_stride the
 * stride), positive for bit 0 -> the kb Z information bits, MSB first,
 * [batch][out_stride] bytes.  Layered normalized min-sum (the rows in order
 * as layers, messages 0.75 min), max_iter passes (at most 32), no early
 * stop, in FP16 arithmetic (the precision of the reference's cuPHY decoder;
 * two code blocks per CTA in the halves of FP16 pairs).  Channel LLRs are
 * clamped to +-1024 and messages to +-256, which keeps every value finite;
 * NaN inputs give undefined bits.  The check-node state lives in the handle:
 * decodes on one handle that can overlap on the GPU (different streams)
 * race, so serialise them or give each stream its own handle. */
mb_status mb_ldpc_decode(mb_ldpc *ldpc, const uint16_t *llr, uint64_t llr_stride, uint8_t *out,
                         uint64_t out_stride, uint32_t batch, uint32_t max_iter, void *stream);

/* ------------------------------------------------ learned ZF initialiser --- */
/* No counterpart in the reference.  A 3-layer MLP (n_in -> width -> width
 * -> n_out, ReLU) with FP32 master weights, BF16 weights in every product
 * and FP32 accumulation, trained by the library's own forward, backward and
 * Adam kernels on the quadratic loss y^T A y - 2 b^T y + c per sample
 * (A [batch][n_out][n_out], b [batch][n_out], c [batch] or NULL for 0),
 * averaged over the batch.  Parameters are flat FP32: W1 [n_in][width], b1,
 * W2 [width][width], b2, W3 [width][n_out], b3.  All x / y / A / b / c /
 * loss pointers are device memory; params and grads copies are host. */
mb_status mb_mlp_create(uint32_t n_in, uint32_t width, uint32_t n_out, uint32_t max_batch,
                        uint64_t seed, mb_mlp **out);
mb_status mb_mlp_destroy(mb_mlp *mlp);
mb_status mb_mlp_num_params(const mb_mlp *mlp, uint64_t *count);
mb_status mb_mlp_get_params(const mb_mlp *mlp, float *host);
mb_status mb_mlp_set_params(mb_mlp *mlp, const float *host); /* also resets Adam */
mb_status mb_mlp_get_grads(const mb_mlp *mlp, float *host);  /* of the last loss_grad */
mb_status mb_mlp_forward(mb_mlp *mlp, const float *x, uint32_t batch, float *y, void *stream);
mb_status mb_mlp_loss_grad(mb_mlp *mlp, const float *x, const float *A, const float *b,
                           const float *c, uint32_t batch, float *loss, void *stream);
mb_status mb_mlp_adam_step(mb_mlp *mlp, float lr, void *stream);

/* Per-subcarrier ZF from the comb-pilot CSI [G][M][K] (K <= 32; M K up to
 * what one subcarrier's FP64 CSI needs in shared memory, M K <= 14336 on a
 * B200, e.g. 256 x 32):
 * each user's pilots are interpolated linearly along frequency to a CSI
 * estimate c_s [M][K] per subcarrier, G_s is the reference's Gram C C^H of
 * it (C[u][b] = c_s[b][u]), the Grams at the group centres (subcarrier g sg + sg/2) are inverted
 * exactly, and the initial iterate of every subcarrier is the group's own
 * centre inverse (MB_LZF_COARSE), a blend of the centre inverses of groups
 * g-1..g+2 with weights from the MLP (MB_LZF_LEARNED; n_in = sg + 6,
 * n_out = 4), or the exact inverse of G_s (MB_LZF_EXACT); ns_iters
 * Newton-Schulz steps follow.  W [S][M][K] is the per-subcarrier detector,
 * usable by mb_equalize with sc_group = 1. */
enum { MB_LZF_COARSE = 0, MB_LZF_LEARNED = 1, MB_LZF_EXACT = 2 };
typedef struct mb_lzf mb_lzf;
mb_status mb_lzf_create(uint32_t M, uint32_t K, uint32_t S, uint32_t sg, mb_lzf **out);
mb_status mb_lzf_destroy(mb_lzf *lzf);
uint32_t mb_lzf_num_features(uint32_t sg);
/* features [S][sg + 6] (device, FP32) of every subcarrier: one-hot offset in
 * its group, then for the groups g-1, g+1, g+2 the relative Frobenius
 * distance of their centre Gram to group g's and the trace ratio minus 1 */
mb_status mb_lzf_features(mb_lzf *lzf, const mb_c32 *csi, float *features, void *stream);
/* training targets of the blend from an FP64 pass: A [S][4][4], b [S][4] so
 * that alpha^T A alpha - 2 b^T alpha + 1 = ||X0(alpha) - G_s^{-1}||^2 /
 * ||G_s^{-1}||^2 */
mb_status mb_lzf_targets(mb_lzf *lzf, const mb_c32 *csi, float *A, float *b, void *stream);
mb_status mb_lzf_run(mb_lzf *lzf, const mb_c32 *csi, mb_mlp *mlp, int init, uint32_t ns_iters,
                     mb_c32 *W, void *stream);
/* Per subcarrier of the last run, flags [S] (device): 0 = Newton-Schulz
 * from the chosen start, 1 = the Gram was not positive definite, 2 = the
 * start was too far off for Newton-Schulz to converge (||I - G_s X0||_F >= 1)
 * and the exact inverse was taken instead. */
mb_status mb_lzf_flags(mb_lzf *lzf, int32_t *flags, void *stream);
/* ||I - G_s X_s||_F per subcarrier of the last run, res [S] (device) */
mb_status mb_lzf_residual(mb_lzf *lzf, float *res, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MEGASTATION_B200_H_ */

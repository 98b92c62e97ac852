// slot.cu -- single-GPU slot runner: the stage sequence of
// BandProcess::process (baseband/process.cc:134-225) for one cell, with the
// buffers of BandBuffers::init (baseband/buffers.cc:40-156) allocated once
// at create.  The reference issues one operator per symbol on a stream per
// symbol and synchronises the host after the pilots (process.cc:167-173);
// here a whole slot is issued without host synchronisation: pilot FFT for
// all pilot symbols in one launch, ZF over all groups in one launch, and the
// uplink symbols in batches (FFT then fused equalize), with the first batch's
// FFT forked onto a side stream so it overlaps the ZF solve.  Optionally the
// whole uplink slot is captured once into a CUDA graph and replayed.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "ldpc.cuh"
#include "slot.cuh"
#include "sgemv.cuh"
#include "eq_tc.cuh"
#include "fft.cuh"
#include "zf.cuh"
#include "precode_tc.cuh"

using namespace mb;

struct mb_slot {
  mb_cell_desc c;
  uint32_t G;
  uint64_t n_valid, hrow;
  mb_fft *fft;
  mb_scrambler *scr;
  float2 *csi;        // [G][M][K]: CSI, then W in place
  float2 *precoder;   // [G][K][M]
  float *wmax;        // [G] max |W| per group (mixed path with a downlink)
  float2 *y;          // [sym_batch][M][S] uplink FFT output (FP32 path)
  void *y_lp;         // [sym_batch][re|im][M][S_pad] BF16 (mixed path)
  void *img_w;        // detector images for the tensor-core equalizer
  uint32_t S_pad;
  uint32_t sb_cap;    // uplink symbols the y / y_lp buffers hold (>= sym_batch)
  uint32_t eq_cols;   // tensor-core equalizer columns per CTA (0: 128)
  uint32_t fft_ctas;  // CTAs of each tensor-core FFT launch (0: one per SM)
  uint32_t zf_path;   // mixed ZF, K <= 32: 0 by K, 1 CUDA-core products, 2 tensor-core products
  mb_ldpc *ldpc = nullptr;  // decode stage's code (not owned), or null
  uint32_t ldpc_iters = 0;
  // downlink from information bits: the scrambled bits [D][K][info bytes]
  // and the codewords [D][K][dl_row] (their tail past the code block zero)
  uint8_t *dl_info = nullptr, *dl_cw = nullptr;
  uint64_t dl_row = 0;
  bool eq_fused = false;  // the last uplink equalized inside the ZF kernel
  float2 *precoded;   // [D][M][N]
  const mb_mlp *zf_net;  // learned initial iterate of the mixed ZF (not owned), or null
  // mixed-precision downlink on the tensor cores (N = 4096): the BF16
  // precoder images (built with the precoder in the uplink's ZF stage) and
  // the FP16 precoded spectra [D][M][N], whose guard bins stay zero
  void *pc_img;
  void *z16;
  mb_c32 *dl_sym;  // [D][K][S] modulated symbols of mb_slot_downlink_bits
  cudaStream_t side;
  cudaStream_t crit;  // pilot FFT -> ZF: the critical path, at the highest stream priority
  cudaEvent_t ev_fork, ev_join, ev_crit;
  // captured uplink slots, one per (input, outputs, stream) pointer set,
  // least recently used evicted beyond kGraphCache entries
  struct GraphEntry {
    const void *iq;
    uint16_t *llr;
    uint8_t *hard;
    int32_t *status;
    cudaStream_t stream;
    cudaGraphExec_t exec;
    uint64_t last_use;
  };
  std::vector<GraphEntry> graphs;
  uint64_t graph_clock = 0;
  // stage timing: per recorded call, events at stage boundaries
  // With timing on, every kernel runs on the slot stream in turn (no side
  // stream), so each stage time is that kernel's time alone.
  struct Marks {
    cudaEvent_t start, pilot_b, pilot, zf, end;
    std::vector<cudaEvent_t> fft_b, fft_e, eq_b, eq_e;
  };
  std::vector<Marks> marks;
  uint32_t marks_used = 0, marks_max = 0;
};

static mb_status slot_equalize(mb_slot *s, uint32_t nb, uint16_t *llr, uint8_t *hard,
                               cudaStream_t st);

static cudaEvent_t new_event() {
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// the current call's marks, or null when timing is off or exhausted
static mb_slot::Marks *next_marks(mb_slot *s) {
  if (s->marks_used >= s->marks_max) return nullptr;
  if (s->marks.size() <= s->marks_used) {
    mb_slot::Marks m;
    m.start = new_event();
    m.pilot_b = new_event();
    m.pilot = new_event();
    m.zf = new_event();
    m.end = new_event();
    const uint32_t nb = s->c.U + 1;  // batches of any sym_batch
    for (uint32_t i = 0; i < nb; i++) {
      m.fft_b.push_back(new_event());
      m.fft_e.push_back(new_event());
      m.eq_b.push_back(new_event());
      m.eq_e.push_back(new_event());
    }
    s->marks.push_back(m);
  }
  return &s->marks[s->marks_used++];
}

static void free_marks(mb_slot *s) {
  for (auto &m : s->marks) {
    cudaEventDestroy(m.start);
    cudaEventDestroy(m.pilot_b);
    cudaEventDestroy(m.pilot);
    cudaEventDestroy(m.zf);
    cudaEventDestroy(m.end);
    for (auto *v : {&m.fft_b, &m.fft_e, &m.eq_b, &m.eq_e})
      for (auto e : *v) cudaEventDestroy(e);
  }
  s->marks.clear();
}

static size_t iq_elem_bytes(int dt) {
  return dt == MB_IQ_C32 ? 8 : dt == MB_IQ_I8 ? 2 : 4;
}

extern "C" mb_status mb_slot_destroy(mb_slot *s) {
  if (!s) return MB_BAD_ARG;
  for (auto &e : s->graphs) cudaGraphExecDestroy(e.exec);
  free_marks(s);
  if (s->fft) mb_fft_destroy(s->fft);
  if (s->scr) mb_scrambler_destroy(s->scr);
  cudaFree(s->csi);
  cudaFree(s->precoder);
  cudaFree(s->wmax);
  cudaFree(s->y);
  cudaFree(s->y_lp);
  cudaFree(s->img_w);
  cudaFree(s->precoded);
  cudaFree(s->pc_img);
  cudaFree(s->z16);
  cudaFree(s->dl_sym);
  cudaFree(s->dl_info);
  cudaFree(s->dl_cw);
  if (s->side) cudaStreamDestroy(s->side);
  if (s->crit) cudaStreamDestroy(s->crit);
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  if (s->ev_crit) cudaEventDestroy(s->ev_crit);
  delete s;
  return MB_OK;
}

// sb_cap_all: size the batch buffers for all U symbols, so that sym_batch
// may later change (the batched-cells autotuner)
static mb_status slot_create(const mb_cell_desc *cell, bool sb_cap_all, mb_slot **out) {
  if (!cell || !out) return MB_BAD_ARG;
  *out = nullptr;
  const mb_cell_desc &c = *cell;
  if (c.M == 0 || c.K == 0 || c.K > c.M || c.K > 64 || c.sg == 0 || c.S == 0 ||
      c.S > c.N || !is_pow2(c.N))
    return MB_BAD_SHAPE;
  if ((uint64_t)c.P * c.sg < c.K) return MB_BAD_SHAPE;  // config.cc:75-82
  if (c.Qm != 2 && c.Qm != 4 && c.Qm != 6 && c.Qm != 8) return MB_BAD_ARG;
  if (c.U && (c.cb_size == 0 || c.cb_stride < c.zeros + c.cb_size)) return MB_BAD_SHAPE;
  mb_slot *s = new mb_slot();
  s->c = c;
  if (s->c.sym_batch == 0) s->c.sym_batch = 4;
  s->c.sym_batch = std::min(s->c.sym_batch, std::max<uint32_t>(c.U, 1));
  s->sb_cap = sb_cap_all ? std::max<uint32_t>(c.U, 1) : s->c.sym_batch;
  s->eq_cols = 0;
  s->fft_ctas = 0;
  s->zf_path = 0;
  s->G = (c.S + c.sg - 1) / c.sg;
  s->n_valid = std::min<uint64_t>((uint64_t)c.S * c.Qm, c.cb_size);
  s->hrow = (s->n_valid + 7) / 8;
  mb_fft_desc fd{(c.N - c.S) / 2, c.N, c.S, c.M, c.K, c.sg};
  mb_status st = mb_fft_create(&fd, &s->fft);
  if (st == MB_OK && c.U)
    st = mb_scrambler_create((int)c.scrambler_mode, c.c_init, c.K, s->n_valid, &s->scr);
  auto alloc = [&](void **p, size_t bytes) {
    if (st != MB_OK || bytes == 0) return;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) st = record_error(e);
  };
  const size_t gmk = (size_t)s->G * c.M * c.K;
  alloc((void **)&s->csi, sizeof(float2) * gmk);
  alloc((void **)&s->precoder, sizeof(float2) * gmk);
  if (c.D) alloc((void **)&s->wmax, sizeof(float) * s->G);
  alloc((void **)&s->precoded, sizeof(float2) * (size_t)c.D * c.M * c.N);
  alloc((void **)&s->dl_sym, sizeof(mb_c32) * (size_t)c.D * c.K * c.S);
  if (c.D && c.zf_precision == MB_ZF_MIXED && c.N == 4096 && precode_tc_supported(c.K, c.sg) &&
      (c.out_dtype == MB_IQ_I16 || c.out_dtype == MB_IQ_I8 || c.out_dtype == MB_IQ_F16)) {
    alloc(&s->pc_img, (size_t)s->G * precode_tc_shape(c.M, c.K).img_group_bytes);
    alloc(&s->z16, sizeof(__half2) * (size_t)c.D * c.M * c.N);
    if (s->z16) {
      const cudaError_t e = cudaMemset(s->z16, 0, sizeof(__half2) * (size_t)c.D * c.M * c.N);
      if (e != cudaSuccess) st = record_error(e);
    }
  }
  const bool mixed = c.zf_precision == MB_ZF_MIXED;
  if (mixed && st == MB_OK && !equalize_tc_supported(c.K, c.sg, s->c.sym_batch))
    st = MB_UNSUPPORTED;
  s->S_pad = (c.S + 7) / 8 * 8;
  const size_t ylp_bytes = (size_t)s->sb_cap * 2 * c.M * s->S_pad * 2;
  if (mixed) {
    alloc(&s->y_lp, ylp_bytes);
    alloc(&s->img_w, zf_mixed_scratch_bytes(s->G, c.M, c.K));
    if (st == MB_OK) {
      // the S_pad - S padding columns are never written by the FFT
      cudaError_t e = cudaMemset(s->y_lp, 0, ylp_bytes);
      if (e != cudaSuccess) st = record_error(e);
    }
  } else {
    alloc((void **)&s->y, sizeof(float2) * (size_t)s->sb_cap * c.M * c.S);
  }
  if (st == MB_OK) {
    // the uplink FFT batch that overlaps the ZF runs at the lowest priority,
    // the pilot FFT and ZF it overlaps at the highest (CTAs of the critical
    // path are scheduled first whenever both are pending)
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, least);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->crit, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_crit, cudaEventDisableTiming);
    if (e != cudaSuccess) st = record_error(e);
  }
  if (st == MB_OK && s->csi) {
    // a short last group reads pilots of users it has no comb position for;
    // start from zeros so those entries are defined before the tail fill
    cudaError_t e = cudaMemset(s->csi, 0, sizeof(float2) * gmk);
    if (e != cudaSuccess) st = record_error(e);
  }
  if (st != MB_OK) {
    mb_slot_destroy(s);
    return st;
  }
  *out = s;
  return MB_OK;
}

// bytes of one slot's samples, LLRs and hard bits (the pipeline sizes its
// device rings with them)
void mb::slot_io_bytes(const mb_slot *s, uint64_t *iq, uint64_t *llr, uint64_t *hard) {
  const mb_cell_desc &c = s->c;
  *iq = (uint64_t)(c.P + c.U) * iq_elem_bytes(c.iq_dtype) * c.M * c.N;
  *llr = (uint64_t)c.U * c.K * c.cb_stride * 2;
  *hard = (uint64_t)c.U * c.K * s->hrow;
}

extern "C" mb_status mb_slot_create(const mb_cell_desc *cell, mb_slot **out) {
  return slot_create(cell, false, out);
}

static mb_status issue_uplink(mb_slot *s, const void *iq, uint16_t *llr,
                              uint8_t *hard, int32_t *status,
                              cudaStream_t st, mb_slot::Marks *mk) {
  const mb_cell_desc &c = s->c;
#define MARK(ev) \
  if (mk) MB_CUDA_TRY(cudaEventRecord((ev), st))
  MARK(mk->start);
  const size_t sym_bytes = iq_elem_bytes(c.iq_dtype) * c.M * c.N;
  const char *iq_b = reinterpret_cast<const char *>(iq);
  mb_status r;
  const bool mixed = c.zf_precision == MB_ZF_MIXED;
  // uplink FFT of nb symbols from l0: FP32 rows for the SIMT equalizer, or
  // planar BF16 rows for the tensor-core equalizer
  auto fft_batch = [&](uint32_t l0, uint32_t nb, cudaStream_t fs) {
    const void *src = iq_b + (size_t)(c.P + l0) * sym_bytes;
    return mixed ? fft_uplink_lp(s->fft, src, c.iq_dtype, nb, s->y_lp, s->S_pad, fs, s->fft_ctas)
                 : mb_fft_uplink(s->fft, src, c.iq_dtype, nb, reinterpret_cast<mb_c32 *>(s->y), fs);
  };
  // Mixed precision at N = 4096: the pilot symbols and the first uplink
  // batch are adjacent rows of iq and go through ONE tensor-core FFT launch
  // on the critical stream (CSI and planar BF16 rows).  That kernel holds a
  // whole SM per CTA, so nothing would run beside a separate pilot launch
  // anyway, and the pilots ride in its pipeline instead of paying a
  // latency-bound launch of their own.
  const uint32_t nb0 = std::min(c.sym_batch, c.U);
  const bool combined = mixed && c.U && fft_slot_tc_ok(s->fft, iq, s->S_pad, s->y_lp);
  // otherwise fork: the first uplink FFT batch only needs the samples
  // (serialised and timed on the slot stream when timing is on)
  if (!combined && c.U && mk) {
    MARK(mk->fft_b[0]);
    r = fft_batch(0, nb0, st);
    if (r != MB_OK) return r;
    MARK(mk->fft_e[0]);
  } else if (!combined && c.U) {
    MB_CUDA_TRY(cudaEventRecord(s->ev_fork, st));
    MB_CUDA_TRY(cudaStreamWaitEvent(s->side, s->ev_fork, 0));
    r = fft_batch(0, nb0, s->side);
    if (r != MB_OK) return r;
    MB_CUDA_TRY(cudaEventRecord(s->ev_join, s->side));
  }
  // pilots -> CSI -> W (+ precoder) on the high-priority stream (the slot
  // stream itself while timing)
  cudaStream_t cs = st;
  if (!mk) {
    if (!c.U || combined) MB_CUDA_TRY(cudaEventRecord(s->ev_fork, st));
    MB_CUDA_TRY(cudaStreamWaitEvent(s->crit, s->ev_fork, 0));
    cs = s->crit;
  }
  if (combined) {
    MARK(mk->fft_b[0]);
    r = fft_slot_tc(s->fft, iq, c.iq_dtype, c.P, nb0, reinterpret_cast<mb_c32 *>(s->csi), s->y_lp, s->S_pad, cs,
                    s->fft_ctas);
    if (r != MB_OK) return r;
    MARK(mk->fft_e[0]);
  }
  MARK(mk->pilot_b);
  // pilot FFT with the short last group's tail fill in its epilogue.  The
  // FP32 kernel's many small CTAs finish a few pilot symbols sooner than
  // the tensor-core kernel's one-CTA-per-SM pipeline (18 vs 22 us for 512
  // rows of 4096), so the pilots stay on it in both precisions.
  if (!combined) {
    r = fft_pilot_fill(s->fft, iq, c.iq_dtype, c.P, reinterpret_cast<mb_c32 *>(s->csi), cs);
    if (r != MB_OK) return r;
  }
  MARK(mk->pilot);
  float2 *prec = c.D ? s->precoder : nullptr;
  s->eq_fused = false;
  if (mixed) {
    mb_zf_opts o{c.zf_precision, c.ns_iters, c.cond_threshold, s->zf_net ? 1u : 0u};
    ZfNetView v{};
    if (s->zf_net) {
      r = mlp_zf_init_view(s->zf_net, &v);
      if (r != MB_OK) return r;
    }
    // every uplink symbol already planarised by the combined FFT: the ZF
    // kernel equalizes each group's columns itself, from the detector image
    // in shared memory (shapes it cannot take fall back to two launches)
    if (combined && nb0 == c.U) {
      EqParams p;
      r = equalize_prepare(p, reinterpret_cast<const mb_c32 *>(s->csi), reinterpret_cast<const mb_c32 *>(s->y_lp),
                           c.K, c.M, c.S, c.sg, c.U, c.Qm, c.cb_size, c.cb_stride, c.zeros, 1, llr, hard, s->scr);
      if (r != MB_OK) return r;
      r = zf_mixed_eq_run(s->csi, s->G, c.M, c.K, &o, status, nullptr, cs, prec != nullptr, s->wmax, &v, p,
                          s->y_lp, s->S_pad, c.U, s->zf_path);
      if (r == MB_OK) s->eq_fused = true;
      else if (r != MB_UNSUPPORTED) return r;
    }
    // W in FP32 only feeds the downlink precoder; the equalizer reads the image
    if (!s->eq_fused)
      r = zf_mixed_run(s->csi, s->img_w, s->G, c.M, c.K, &o, status, nullptr, cs, prec != nullptr, s->wmax,
                       &v, s->zf_path);
    else
      r = MB_OK;
    if (r == MB_OK && prec) r = precoder_scale(s->csi, prec, s->wmax, c.M, c.K, s->G, cs);
    // the tensor-core downlink's BF16 precoder images, from the same precoder
    if (r == MB_OK && prec && s->pc_img) r = precoder_image(prec, s->pc_img, s->G, c.M, c.K, cs);
  } else {
    r = zf_chol(s->csi, prec, s->G, c.M, c.K, c.zf_precision == MB_ZF_FP64, status, nullptr, cs);
  }
  if (r != MB_OK) return r;
  if (!mk) {
    MB_CUDA_TRY(cudaEventRecord(s->ev_crit, s->crit));
    MB_CUDA_TRY(cudaStreamWaitEvent(st, s->ev_crit, 0));
  }
  MARK(mk->zf);
  if (!c.U) {
    MARK(mk->end);
    return MB_OK;
  }
  if (!mk && !combined) MB_CUDA_TRY(cudaStreamWaitEvent(st, s->ev_join, 0));
  if (s->eq_fused) {
    // equalized in the ZF stage (timing: an empty equalize stage)
    MARK(mk->eq_b[0]);
    MARK(mk->eq_e[0]);
    MARK(mk->end);
    return MB_OK;
  }
  const uint64_t llr_sym = (uint64_t)c.K * c.cb_stride;
  const uint64_t hard_sym = (uint64_t)c.K * s->hrow;
  uint32_t bi = 0;
  for (uint32_t l0 = 0; l0 < c.U; l0 += c.sym_batch, bi++) {
    const uint32_t nb = std::min(c.sym_batch, c.U - l0);
    if (l0) {
      MARK(mk->fft_b[bi]);
      r = fft_batch(l0, nb, st);
      if (r != MB_OK) return r;
      MARK(mk->fft_e[bi]);
    }
    MARK(mk->eq_b[bi]);
    r = slot_equalize(s, nb, llr + l0 * llr_sym, hard ? hard + l0 * hard_sym : nullptr, st);
    if (r != MB_OK) return r;
    MARK(mk->eq_e[bi]);
  }
  MARK(mk->end);
#undef MARK
  return MB_OK;
}

// equalize one batch of nb symbols whose FFT output sits in the slot's
// y (FP32) or y_lp (BF16) buffer; llr / hard point at the batch's rows
static mb_status slot_equalize(mb_slot *s, uint32_t nb, uint16_t *llr, uint8_t *hard,
                               cudaStream_t st) {
  const mb_cell_desc &c = s->c;
  if (c.zf_precision != MB_ZF_MIXED)
    return mb_equalize(reinterpret_cast<const mb_c32 *>(s->csi),
                       reinterpret_cast<const mb_c32 *>(s->y), c.K, c.M, c.S, c.sg, nb,
                       c.Qm, c.cb_size, c.cb_stride, c.zeros, 1, llr, hard, s->scr,
                       nullptr, st);
  EqParams p;
  mb_status r = equalize_prepare(p, reinterpret_cast<const mb_c32 *>(s->csi),
                                 reinterpret_cast<const mb_c32 *>(s->y_lp), c.K, c.M, c.S,
                                 c.sg, nb, c.Qm, c.cb_size, c.cb_stride, c.zeros, 1, llr,
                                 hard, s->scr);
  if (r != MB_OK) return r;
  const DeviceTables *tab = device_tables();
  return equalize_tc(p, s->img_w, s->y_lp, s->S_pad, 0, nb, tab ? tab->err : nullptr, st,
                     s->eq_cols);
}

extern "C" mb_status mb_slot_uplink(mb_slot *s, const void *iq, uint16_t *llr,
                                    uint8_t *hard, int32_t *status,
                                    void *stream) {
  if (!s || !iq || (s->c.U && !llr)) return MB_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  if (!s->c.use_graph || s->marks_max)
    return issue_uplink(s, iq, llr, hard, status, st, next_marks(s));
  if (!st) return MB_BAD_ARG;  // the legacy stream cannot be captured
  constexpr size_t kGraphCache = 16;
  mb_slot::GraphEntry *hit = nullptr;
  for (auto &e : s->graphs)
    if (e.iq == iq && e.llr == llr && e.hard == hard && e.status == status && e.stream == st) hit = &e;
  if (!hit) {
    MB_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    mb_status r = issue_uplink(s, iq, llr, hard, status, st, nullptr);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (r != MB_OK) {
      if (g) cudaGraphDestroy(g);
      return r;
    }
    if (e != cudaSuccess) return record_error(e);
    cudaGraphExec_t exec = nullptr;
    // kernel nodes keep the priority of the stream they were captured on
    e = cudaGraphInstantiate(&exec, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return record_error(e);
    if (s->graphs.size() >= kGraphCache) {
      auto lru = s->graphs.begin();
      for (auto it = s->graphs.begin(); it != s->graphs.end(); ++it)
        if (it->last_use < lru->last_use) lru = it;
      cudaGraphExecDestroy(lru->exec);
      s->graphs.erase(lru);
    }
    s->graphs.push_back({iq, llr, hard, status, st, exec, 0});
    hit = &s->graphs.back();
  }
  hit->last_use = ++s->graph_clock;
  MB_CUDA_TRY(cudaGraphLaunch(hit->exec, st));
  return MB_OK;
}

extern "C" mb_status mb_slot_downlink(mb_slot *s, const mb_c32 *symbols,
                                      void *out, void *stream) {
  if (!s || !symbols || !out) return MB_BAD_ARG;
  const mb_cell_desc &c = s->c;
  if (!c.D) return MB_BAD_SHAPE;
  cudaStream_t st = as_stream(stream);
  if (s->pc_img && fft_ifft_tc_ok(s->fft, s->z16, MB_IQ_F16, out, c.out_dtype)) {
    // mixed precision: precode on the tensor cores into FP16 spectra, then
    // the tensor-core inverse FFT with the output quantiser
    const DeviceTables *tab = device_tables();
    if (!tab) return MB_CUDA_ERROR;
    mb_status r = precode_tc(s->pc_img, reinterpret_cast<const float2 *>(symbols), s->z16, c.M, c.K, c.S, c.sg,
                             c.N, (c.N - c.S) / 2, c.D, tab->err, st);
    if (r != MB_OK) return r;
    return fft_tc_inverse_slot(s->fft, s->z16, c.D, out, c.out_dtype, st);
  }
  mb_status r = mb_precode(reinterpret_cast<const mb_c32 *>(s->precoder), symbols,
                           c.M, c.K, c.S, c.sg, c.N, (c.N - c.S) / 2, c.D,
                           reinterpret_cast<mb_c32 *>(s->precoded), st);
  if (r != MB_OK) return r;
  return mb_ifft_downlink(s->fft, reinterpret_cast<const mb_c32 *>(s->precoded), c.D,
                          out, c.out_dtype, st);
}

extern "C" mb_status mb_slot_downlink_bits(mb_slot *s, const uint8_t *bits, uint64_t in_bytes, void *out,
                                           void *stream) {
  if (!s || !bits || !out) return MB_BAD_ARG;
  const mb_cell_desc &c = s->c;
  if (!c.D || !s->dl_sym) return MB_BAD_SHAPE;
  // every user row holds at least the S Qm bits of its symbol
  if (in_bytes < ((uint64_t)c.S * c.Qm + 7) / 8) return MB_BAD_SHAPE;
  // the D symbols' K user rows are independent: one modulate launch
  mb_status r = mb_modulate(bits, s->dl_sym, in_bytes, c.S, (uint64_t)c.D * c.K, c.Qm, 0, nullptr, stream);
  if (r != MB_OK) return r;
  return mb_slot_downlink(s, s->dl_sym, out, stream);
}

extern "C" mb_status mb_slot_set_ldpc(mb_slot *s, mb_ldpc *code, uint32_t max_iter) {
  if (!s) return MB_BAD_ARG;
  if (code) {
    // the code block must be the cell's: zeros = 2Z punctured LLRs, then
    // cb_size = (kb - 2 + mb) Z, within the row stride
    const mb_cell_desc &c = s->c;
    if (c.zeros != 2ull * code->Z || c.cb_size != (uint64_t)(code->kb - 2 + code->mb) * code->Z ||
        c.cb_stride < (uint64_t)(code->kb + code->mb) * code->Z)
      return MB_BAD_SHAPE;
    if (max_iter == 0 || max_iter > 32) return MB_BAD_ARG;  // mb_ldpc_decode's range
  }
  s->ldpc = code;
  s->ldpc_iters = max_iter;
  cudaFree(s->dl_info);
  cudaFree(s->dl_cw);
  s->dl_info = s->dl_cw = nullptr;
  s->dl_row = 0;
  if (code && s->c.D) {
    // the downlink's buffers: a codeword row holds at least the S Qm bits
    // the modulator reads
    const mb_cell_desc &c = s->c;
    const uint64_t info_bytes = ((uint64_t)code->kb * code->Z + 7) / 8;
    s->dl_row = std::max((c.cb_size + 7) / 8, ((uint64_t)c.S * c.Qm + 7) / 8);
    const uint64_t rows = (uint64_t)c.D * c.K;
    MB_CUDA_TRY(cudaMalloc((void **)&s->dl_info, rows * info_bytes));
    MB_CUDA_TRY(cudaMalloc((void **)&s->dl_cw, rows * s->dl_row));
    MB_CUDA_TRY(cudaMemset(s->dl_cw, 0, rows * s->dl_row));
  }
  return MB_OK;
}

extern "C" mb_status mb_slot_downlink_info(mb_slot *s, const uint8_t *info, void *out, void *stream) {
  if (!s || !info || !out) return MB_BAD_ARG;
  const mb_cell_desc &c = s->c;
  if (!c.D || !s->ldpc || !s->dl_cw) return MB_BAD_SHAPE;
  if (c.scrambler_mode != MB_SCR_LFSR127) return MB_UNSUPPORTED;
  const uint64_t info_bytes = ((uint64_t)s->ldpc->kb * s->ldpc->Z + 7) / 8;
  const uint32_t rows = c.D * c.K;
  // process.cc:198-208: scramble, LDPC-encode, modulate, precode, IFFT
  mb_status r = mb_scramble(s->dl_info, info, info_bytes, rows, stream);
  if (r == MB_OK) r = mb_ldpc_encode(s->ldpc, s->dl_info, info_bytes, s->dl_cw, s->dl_row, rows, stream);
  if (r == MB_OK) r = mb_slot_downlink_bits(s, s->dl_cw, s->dl_row, out, stream);
  return r;
}

extern "C" mb_status mb_slot_decode(mb_slot *s, const uint16_t *llr, uint8_t *decoded, void *stream) {
  if (!s || !llr || !decoded) return MB_BAD_ARG;
  if (!s->ldpc) return MB_BAD_SHAPE;
  const mb_cell_desc &c = s->c;
  if (c.scrambler_mode != MB_SCR_LFSR127) return MB_UNSUPPORTED;
  const uint64_t bytes = ((uint64_t)s->ldpc->kb * s->ldpc->Z + 7) / 8;
  const uint32_t blocks = c.U * c.K;  // one code block per (symbol, user) row
  mb_status r = mb_ldpc_decode(s->ldpc, llr, c.cb_stride, decoded, bytes, blocks, s->ldpc_iters, stream);
  if (r != MB_OK) return r;
  // the decoded bits are descrambled (process.cc:188, Scrambler::scrambler
  // on every row)
  return mb_scramble(decoded, decoded, bytes, blocks, stream);
}

extern "C" mb_status mb_slot_timing(mb_slot *s, uint32_t max_calls) {
  if (!s) return MB_BAD_ARG;
  s->marks_max = max_calls;
  s->marks_used = 0;
  // create the events now, outside any timed region
  for (uint32_t i = 0; i < max_calls; i++) next_marks(s);
  s->marks_used = 0;
  return MB_OK;
}

extern "C" mb_status mb_slot_stage_ms(mb_slot *s, double *out) {
  if (!s || !out) return MB_BAD_ARG;
  for (int i = 0; i < 8; i++) out[i] = 0;
  auto ms = [](cudaEvent_t a, cudaEvent_t b) {
    float v = 0.f;
    cudaEventElapsedTime(&v, a, b);
    return (double)v;
  };
  for (uint32_t k = 0; k < s->marks_used; k++) {
    auto &m = s->marks[k];
    MB_CUDA_TRY(cudaEventSynchronize(m.end));
    out[0] += ms(m.pilot_b, m.pilot);
    out[1] += ms(m.pilot, m.zf);
    out[4] += ms(m.start, m.end);
    uint32_t bi = 0;
    for (uint32_t l0 = 0; l0 < s->c.U; l0 += s->c.sym_batch, bi++) {
      out[2] += ms(m.fft_b[bi], m.fft_e[bi]);
      out[5] += 1;
      out[3] += ms(m.eq_b[bi], m.eq_e[bi]);
      out[6] += s->eq_fused ? 0 : 1;  // no equalize launch of its own when fused
    }
    out[7] += 1;
  }
  s->marks_used = 0;
  return MB_OK;
}

extern "C" mb_status mb_slot_buffers(mb_slot *s, mb_c32 **csi, mb_c32 **precoder) {
  if (!s) return MB_BAD_ARG;
  if (csi) *csi = reinterpret_cast<mb_c32 *>(s->csi);
  if (precoder) *precoder = reinterpret_cast<mb_c32 *>(s->precoder);
  return MB_OK;
}

extern "C" mb_status mb_slot_set_zf_init(mb_slot *s, const mb_mlp *net) {
  if (!s) return MB_BAD_ARG;
  if (net && s->c.zf_precision != MB_ZF_MIXED) return MB_UNSUPPORTED;
  if (net) {
    ZfNetView v;
    const mb_status r = mlp_zf_init_view(net, &v);
    if (r != MB_OK) return r;
  }
  if (net == s->zf_net) return MB_OK;
  // captured slots hold the previous choice in their kernel parameters
  for (auto &e : s->graphs) cudaGraphExecDestroy(e.exec);
  s->graphs.clear();
  s->zf_net = net;
  return MB_OK;
}

// ---------------------------------------------------------------- cells
// Many cells of uneven shape per slot in ONE CUDA graph launch: the graph
// forks from the launching stream into one branch per cell (each branch is
// that cell's slot: pilot FFT, ZF, uplink FFT batches, equalize) and joins
// back, so the cells' kernels run concurrently and the host issues a single
// cudaGraphLaunch per slot.  The reference runs one cell per BandProcess and
// has no batched form.
struct mb_cells {
  std::vector<mb_slot *> slots;
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
  struct Entry {
    std::vector<const void *> key;
    cudaGraphExec_t exec;
    uint64_t last_use;
  };
  std::vector<Entry> graphs;
  uint64_t clock = 0;
};

static void cells_drop_graphs(mb_cells *cs) {
  for (auto &e : cs->graphs) cudaGraphExecDestroy(e.exec);
  cs->graphs.clear();
}

extern "C" mb_status mb_cells_destroy(mb_cells *cs) {
  if (!cs) return MB_BAD_ARG;
  cells_drop_graphs(cs);
  for (auto *s : cs->slots) mb_slot_destroy(s);
  for (auto b : cs->branch) cudaStreamDestroy(b);
  for (auto e : cs->join) cudaEventDestroy(e);
  if (cs->fork) cudaEventDestroy(cs->fork);
  delete cs;
  return MB_OK;
}

extern "C" mb_status mb_cells_create(const mb_cell_desc *cells, uint32_t n, mb_cells **out) {
  if (!cells || !out || n == 0) return MB_BAD_ARG;
  *out = nullptr;
  mb_cells *cs = new mb_cells();
  mb_status st = MB_OK;
  for (uint32_t c = 0; c < n && st == MB_OK; c++) {
    mb_cell_desc d = cells[c];
    d.use_graph = 0;  // the cells object captures all of them together
    mb_slot *s = nullptr;
    st = slot_create(&d, true, &s);
    if (st == MB_OK) cs->slots.push_back(s);
    cudaStream_t b = nullptr;
    cudaEvent_t e = nullptr;
    if (st == MB_OK) {
      cudaError_t ce = cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking);
      if (ce == cudaSuccess) cs->branch.push_back(b);
      if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
      if (ce == cudaSuccess) cs->join.push_back(e);
      if (ce != cudaSuccess) st = record_error(ce);
    }
  }
  if (st == MB_OK) {
    cudaError_t ce = cudaEventCreateWithFlags(&cs->fork, cudaEventDisableTiming);
    if (ce != cudaSuccess) st = record_error(ce);
  }
  if (st != MB_OK) {
    mb_cells_destroy(cs);
    return st;
  }
  *out = cs;
  return MB_OK;
}

// one slot of every cell, captured into one graph per pointer set and stream
static mb_status cells_launch(mb_cells *cs, const void *const *iq, uint16_t *const *llr,
                              uint8_t *const *hard, int32_t *const *status, cudaStream_t st) {
  const uint32_t n = (uint32_t)cs->slots.size();
  std::vector<const void *> key;
  key.reserve(4 * n + 1);
  for (uint32_t c = 0; c < n; c++) {
    if (!iq[c] || (cs->slots[c]->c.U && (!llr || !llr[c]))) return MB_BAD_ARG;
    key.push_back(iq[c]);
    key.push_back(llr ? llr[c] : nullptr);
    key.push_back(hard ? hard[c] : nullptr);
    key.push_back(status ? status[c] : nullptr);
  }
  key.push_back(st);
  mb_cells::Entry *hit = nullptr;
  for (auto &e : cs->graphs)
    if (e.key == key) hit = &e;
  if (!hit) {
    MB_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    mb_status r = MB_OK;
    cudaError_t ce = cudaEventRecord(cs->fork, st);
    for (uint32_t c = 0; c < n && r == MB_OK && ce == cudaSuccess; c++) {
      ce = cudaStreamWaitEvent(cs->branch[c], cs->fork, 0);
      if (ce != cudaSuccess) break;
      r = issue_uplink(cs->slots[c], iq[c], llr ? llr[c] : nullptr, hard ? hard[c] : nullptr,
                       status ? status[c] : nullptr, cs->branch[c], nullptr);
      if (r != MB_OK) break;
      ce = cudaEventRecord(cs->join[c], cs->branch[c]);
      if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st, cs->join[c], 0);
    }
    cudaGraph_t g = nullptr;
    cudaError_t ee = cudaStreamEndCapture(st, &g);
    if (r != MB_OK || ce != cudaSuccess || ee != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      (void)cudaGetLastError();
      return r != MB_OK ? r : record_error(ce != cudaSuccess ? ce : ee);
    }
    cudaGraphExec_t exec = nullptr;
    ce = cudaGraphInstantiate(&exec, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return record_error(ce);
    constexpr size_t kGraphCache = 8;
    if (cs->graphs.size() >= kGraphCache) {
      auto lru = cs->graphs.begin();
      for (auto it = cs->graphs.begin(); it != cs->graphs.end(); ++it)
        if (it->last_use < lru->last_use) lru = it;
      cudaGraphExecDestroy(lru->exec);
      cs->graphs.erase(lru);
    }
    cs->graphs.push_back({key, exec, 0});
    hit = &cs->graphs.back();
  }
  hit->last_use = ++cs->clock;
  MB_CUDA_TRY(cudaGraphLaunch(hit->exec, st));
  return MB_OK;
}

extern "C" mb_status mb_cells_uplink(mb_cells *cs, const void *const *iq, uint16_t *const *llr,
                                     uint8_t *const *hard, int32_t *const *status, void *stream) {
  if (!cs || !iq) return MB_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  if (!st) return MB_BAD_ARG;  // the legacy stream cannot be captured
  return cells_launch(cs, iq, llr, hard, status, st);
}

extern "C" mb_status mb_cells_get_tuning(const mb_cells *cs, uint32_t *sym_batch,
                                         uint32_t *eq_cols) {
  if (!cs) return MB_BAD_ARG;
  for (size_t c = 0; c < cs->slots.size(); c++) {
    if (sym_batch) sym_batch[c] = cs->slots[c]->c.sym_batch;
    if (eq_cols) eq_cols[c] = cs->slots[c]->eq_cols ? cs->slots[c]->eq_cols : 128;
  }
  return MB_OK;
}

extern "C" mb_status mb_cells_set_tuning(mb_cells *cs, const uint32_t *sym_batch,
                                         const uint32_t *eq_cols) {
  if (!cs) return MB_BAD_ARG;
  for (size_t c = 0; c < cs->slots.size(); c++) {
    mb_slot *s = cs->slots[c];
    if (sym_batch && (sym_batch[c] == 0 || sym_batch[c] > s->sb_cap)) return MB_BAD_ARG;
    if (eq_cols && eq_cols[c] != 0 && (eq_cols[c] % 8 || eq_cols[c] > 128)) return MB_BAD_ARG;
  }
  for (size_t c = 0; c < cs->slots.size(); c++) {
    if (sym_batch) cs->slots[c]->c.sym_batch = sym_batch[c];
    if (eq_cols) cs->slots[c]->eq_cols = eq_cols[c] == 128 ? 0 : eq_cols[c];
  }
  cells_drop_graphs(cs);  // the captured work changes
  return MB_OK;
}

extern "C" mb_status mb_cells_get_fft_ctas(const mb_cells *cs, uint32_t *fft_ctas) {
  if (!cs || !fft_ctas) return MB_BAD_ARG;
  for (size_t c = 0; c < cs->slots.size(); c++) fft_ctas[c] = cs->slots[c]->fft_ctas;
  return MB_OK;
}

extern "C" mb_status mb_cells_set_fft_ctas(mb_cells *cs, const uint32_t *fft_ctas) {
  if (!cs || !fft_ctas) return MB_BAD_ARG;
  for (size_t c = 0; c < cs->slots.size(); c++) cs->slots[c]->fft_ctas = fft_ctas[c];
  cells_drop_graphs(cs);  // the captured launches change
  return MB_OK;
}

extern "C" mb_status mb_cells_get_zf_path(const mb_cells *cs, uint32_t *zf_path) {
  if (!cs || !zf_path) return MB_BAD_ARG;
  for (size_t c = 0; c < cs->slots.size(); c++) zf_path[c] = cs->slots[c]->zf_path;
  return MB_OK;
}

extern "C" mb_status mb_cells_set_zf_path(mb_cells *cs, const uint32_t *zf_path) {
  if (!cs || !zf_path) return MB_BAD_ARG;
  for (size_t c = 0; c < cs->slots.size(); c++)
    if (zf_path[c] > 2) return MB_BAD_ARG;
  for (size_t c = 0; c < cs->slots.size(); c++) cs->slots[c]->zf_path = zf_path[c];
  cells_drop_graphs(cs);  // the captured launches change
  return MB_OK;
}

// microseconds per slot of the current tuning: warm-up, then reps graph
// launches timed with CUDA events on st
static mb_status cells_time(mb_cells *cs, const void *const *iq, uint16_t *const *llr,
                            uint8_t *const *hard, uint32_t reps, cudaStream_t st, double *us) {
  for (int w = 0; w < 3; w++) {
    mb_status r = cells_launch(cs, iq, llr, hard, nullptr, st);
    if (r != MB_OK) return r;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  MB_CUDA_TRY(cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return record_error(ce);
  }
  mb_status r = MB_OK;
  ce = cudaEventRecord(e0, st);
  for (uint32_t k = 0; k < reps && r == MB_OK && ce == cudaSuccess; k++)
    r = cells_launch(cs, iq, llr, hard, nullptr, st);
  if (ce == cudaSuccess) ce = cudaEventRecord(e1, st);
  if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r != MB_OK) return r;
  if (ce != cudaSuccess) return record_error(ce);
  *us = 1e3 * ms / std::max<uint32_t>(reps, 1);
  return MB_OK;
}

// Autotuner: the knobs are, per cell, the uplink symbols per FFT/equalize
// batch (sym_batch), the tensor-core equalizer's (symbol, subcarrier)
// columns per CTA (its MMA tile) and, for cells whose FFT runs on the tensor
// cores (mixed, N = 4096), the CTAs of each FFT launch: one CTA holds a whole
// SM, so a cell's FFT on every SM keeps the other cells' kernels waiting,
// while fewer CTAs with more two-row units each let the cells' FFTs and
// solves share the GPU.  Cells of one shape form a class and share a choice;
// classes are visited by decreasing work, each trying its candidates with
// the others fixed (coordinate descent on the measured time of the whole
// batched slot, first over (sym_batch, eq_cols), then over the FFT's CTAs)
// and keeping a candidate only if it is at least 1% faster.  The tuning
// stays on the object (later mb_cells_uplink calls use it) and is returned
// per cell.
extern "C" mb_status mb_cells_autotune(mb_cells *cs, const void *const *iq, uint16_t *const *llr,
                                       uint8_t *const *hard, uint32_t reps, void *stream,
                                       uint32_t *sym_batch_out, uint32_t *eq_cols_out,
                                       double *us_per_slot) {
  if (!cs || !iq) return MB_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  if (!st) return MB_BAD_ARG;
  const uint32_t n = (uint32_t)cs->slots.size();
  if (reps == 0) reps = 20;
  // shape classes
  std::vector<int> cls(n, -1);
  std::vector<std::vector<uint32_t>> members;
  std::vector<double> work;
  for (uint32_t c = 0; c < n; c++) {
    const mb_cell_desc &a = cs->slots[c]->c;
    for (size_t k = 0; k < members.size(); k++) {
      const mb_cell_desc &b = cs->slots[members[k][0]]->c;
      if (a.M == b.M && a.K == b.K && a.N == b.N && a.S == b.S && a.sg == b.sg && a.Qm == b.Qm &&
          a.U == b.U && a.P == b.P && a.zf_precision == b.zf_precision) {
        cls[c] = (int)k;
        break;
      }
    }
    if (cls[c] < 0) {
      cls[c] = (int)members.size();
      members.push_back({});
      work.push_back(0.0);
    }
    members[cls[c]].push_back(c);
    work[cls[c]] += (double)a.M * a.N * (a.P + a.U);
  }
  std::vector<uint32_t> order(members.size());
  for (size_t k = 0; k < order.size(); k++) order[k] = (uint32_t)k;
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return work[a] > work[b]; });

  std::vector<uint32_t> sb(n), cols(n);
  for (uint32_t c = 0; c < n; c++) {
    sb[c] = std::max<uint32_t>(cs->slots[c]->c.U, 1);
    cols[c] = 128;
  }
  mb_status r = mb_cells_set_tuning(cs, sb.data(), cols.data());
  double best = 0.0;
  if (r == MB_OK) r = cells_time(cs, iq, llr, hard, reps, st, &best);
  for (uint32_t k : order) {
    if (r != MB_OK) break;
    const mb_cell_desc &d = cs->slots[members[k][0]]->c;
    const uint32_t U = std::max<uint32_t>(d.U, 1);
    std::vector<std::pair<uint32_t, uint32_t>> cand;
    for (uint32_t parts = 1; parts <= 3; parts++) {
      const uint32_t b = (U + parts - 1) / parts;
      for (uint32_t cl : {128u, 64u}) {
        if (d.zf_precision != MB_ZF_MIXED && cl != 128) continue;
        bool dup = false;
        for (auto &x : cand) dup |= x.first == b && x.second == cl;
        if (!dup) cand.push_back({b, cl});
      }
    }
    std::pair<uint32_t, uint32_t> cur{sb[members[k][0]], cols[members[k][0]]};
    for (auto &cv : cand) {
      if (cv == cur) continue;
      for (uint32_t c : members[k]) {
        sb[c] = cv.first;
        cols[c] = cv.second;
      }
      double t = 0.0;
      r = mb_cells_set_tuning(cs, sb.data(), cols.data());
      if (r == MB_OK) r = cells_time(cs, iq, llr, hard, reps, st, &t);
      if (r != MB_OK) break;
      if (t < 0.99 * best) {
        best = t;
        cur = cv;
      }
    }
    for (uint32_t c : members[k]) {
      sb[c] = cur.first;
      cols[c] = cur.second;
    }
  }
  if (r == MB_OK) r = mb_cells_set_tuning(cs, sb.data(), cols.data());
  // the tensor-core FFT's CTAs per launch
  std::vector<uint32_t> fc(n, 0);
  if (r == MB_OK) r = mb_cells_set_fft_ctas(cs, fc.data());
  for (uint32_t k : order) {
    if (r != MB_OK) break;
    const mb_cell_desc &d = cs->slots[members[k][0]]->c;
    if (d.zf_precision != MB_ZF_MIXED || d.N != 4096) continue;
    uint32_t cur = 0;
    for (uint32_t cand : {74u, 37u, 18u}) {
      for (uint32_t c : members[k]) fc[c] = cand;
      double t = 0.0;
      r = mb_cells_set_fft_ctas(cs, fc.data());
      if (r == MB_OK) r = cells_time(cs, iq, llr, hard, reps, st, &t);
      if (r != MB_OK) break;
      if (t < 0.99 * best) {
        best = t;
        cur = cand;
      }
    }
    for (uint32_t c : members[k]) fc[c] = cur;
  }
  if (r == MB_OK) r = mb_cells_set_fft_ctas(cs, fc.data());
  // where the mixed ZF's inverse runs its products (K <= 32): the CUDA or
  // the tensor cores, from the rule by K
  std::vector<uint32_t> zp(n, 0);
  if (r == MB_OK) r = mb_cells_set_zf_path(cs, zp.data());
  for (uint32_t k : order) {
    if (r != MB_OK) break;
    const mb_cell_desc &d = cs->slots[members[k][0]]->c;
    if (d.zf_precision != MB_ZF_MIXED || d.K > 32) continue;
    uint32_t cur = 0;
    for (uint32_t cand : {1u, 2u}) {
      if ((cand == 2) == (d.K > 16)) continue;  // the rule's choice is the current one
      for (uint32_t c : members[k]) zp[c] = cand;
      double t = 0.0;
      r = mb_cells_set_zf_path(cs, zp.data());
      if (r == MB_OK) r = cells_time(cs, iq, llr, hard, reps, st, &t);
      if (r != MB_OK) break;
      if (t < 0.99 * best) {
        best = t;
        cur = cand;
      }
    }
    for (uint32_t c : members[k]) zp[c] = cur;
  }
  if (r == MB_OK) r = mb_cells_set_zf_path(cs, zp.data());
  if (r != MB_OK) return r;
  if (sym_batch_out) std::copy(sb.begin(), sb.end(), sym_batch_out);
  if (eq_cols_out) std::copy(cols.begin(), cols.end(), eq_cols_out);
  if (us_per_slot) *us_per_slot = best;
  return MB_OK;
}

// pipe.cu -- single-GPU slot pipeline over host buffers.
//
// Replaces, for one GPU, what the reference's scheduler does around each
// slot (scheduler/gpu_engine.cc:77-437 with cpu_buffer.cc:5-49): copy the
// fronthaul samples of a slot to the device, run the slot, copy its LLRs
// and hard bits back.  Here the three steps run on three streams ordered by
// events over rings of `depth` device buffers, so the samples of slot k+1
// cross PCIe while slot k computes and slot k-1's results come back, and
// the host submits without blocking.  The slot itself is one mb_slot (its
// captured graphs are cached per ring buffer); slots compute one after the
// other on the compute stream, only the copies overlap them.
#include <chrono>
#include <thread>
#include <vector>

#include "common.cuh"
#include "slot.cuh"

using namespace mb;

struct mb_pipe {
  mb_slot *slot = nullptr;
  uint32_t depth = 0;
  uint64_t iq_bytes = 0, llr_bytes = 0, hard_bytes = 0;
  cudaStream_t h2d = nullptr, comp = nullptr, d2h = nullptr;
  std::vector<void *> iq;        // [depth] device samples
  std::vector<uint16_t *> llr;   // [depth] device LLRs
  std::vector<uint8_t *> hard;   // [depth] device hard bits
  std::vector<int32_t *> status; // [depth] per-group ZF status
  std::vector<cudaEvent_t> ev_in, ev_done, ev_out;  // [depth]
  std::vector<uint64_t> owner;   // [depth] ticket that last used the buffer
  uint64_t next = 0;             // next ticket
  cudaEvent_t t_start = nullptr, t_end = nullptr;  // device timer
  bool timer_armed = false, timer_started = false;
};

static void pipe_free(mb_pipe *p) {
  if (!p) return;
  if (p->comp) cudaStreamSynchronize(p->comp);
  if (p->h2d) cudaStreamSynchronize(p->h2d);
  if (p->d2h) cudaStreamSynchronize(p->d2h);
  for (auto v : p->iq) cudaFree(v);
  for (auto v : p->llr) cudaFree(v);
  for (auto v : p->hard) cudaFree(v);
  for (auto v : p->status) cudaFree(v);
  for (auto e : p->ev_in) cudaEventDestroy(e);
  for (auto e : p->ev_done) cudaEventDestroy(e);
  for (auto e : p->ev_out) cudaEventDestroy(e);
  if (p->t_start) cudaEventDestroy(p->t_start);
  if (p->t_end) cudaEventDestroy(p->t_end);
  if (p->h2d) cudaStreamDestroy(p->h2d);
  if (p->comp) cudaStreamDestroy(p->comp);
  if (p->d2h) cudaStreamDestroy(p->d2h);
  if (p->slot) mb_slot_destroy(p->slot);
  delete p;
}

extern "C" mb_status mb_pipe_create(const mb_cell_desc *cell, uint32_t depth, mb_pipe **out) {
  if (!cell || !out || depth < 2 || depth > 16) return MB_BAD_ARG;
  *out = nullptr;
  if (cell->U == 0) return MB_BAD_SHAPE;
  mb_pipe *p = new mb_pipe();
  p->depth = depth;
  mb_status r = mb_slot_create(cell, &p->slot);
  if (r != MB_OK) {
    pipe_free(p);
    return r;
  }
  slot_io_bytes(p->slot, &p->iq_bytes, &p->llr_bytes, &p->hard_bytes);
  uint32_t G = (cell->S + cell->sg - 1) / cell->sg;
  cudaError_t e = cudaStreamCreateWithFlags(&p->h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->comp, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->d2h, cudaStreamNonBlocking);
  p->iq.assign(depth, nullptr);
  p->llr.assign(depth, nullptr);
  p->hard.assign(depth, nullptr);
  p->status.assign(depth, nullptr);
  p->ev_in.assign(depth, nullptr);
  p->ev_done.assign(depth, nullptr);
  p->ev_out.assign(depth, nullptr);
  p->owner.assign(depth, UINT64_MAX);
  if (e == cudaSuccess) e = cudaEventCreate(&p->t_start);
  if (e == cudaSuccess) e = cudaEventCreate(&p->t_end);
  for (uint32_t b = 0; b < depth && e == cudaSuccess; b++) {
    e = cudaMalloc(&p->iq[b], p->iq_bytes);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&p->llr[b]), p->llr_bytes);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&p->hard[b]), p->hard_bytes);
    // the slot never writes an LLR row's punctured and padding positions:
    // they stay zero, as in a caller's zeroed buffer
    if (e == cudaSuccess) e = cudaMemset(p->llr[b], 0, p->llr_bytes);
    if (e == cudaSuccess) e = cudaMemset(p->hard[b], 0, p->hard_bytes);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&p->status[b]), sizeof(int32_t) * G);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_in[b], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_done[b], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_out[b], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    pipe_free(p);
    return e == cudaErrorMemoryAllocation ? MB_NO_MEMORY : record_error(e);
  }
  *out = p;
  return MB_OK;
}

extern "C" mb_status mb_pipe_destroy(mb_pipe *p) {
  if (!p) return MB_BAD_ARG;
  pipe_free(p);
  return MB_OK;
}

extern "C" mb_status mb_pipe_submit(mb_pipe *p, const void *iq_host, uint16_t *llr_host, uint8_t *hard_host,
                                    uint64_t *ticket) {
  if (!p || !iq_host || !llr_host) return MB_BAD_ARG;
  const uint64_t k = p->next;
  const uint32_t b = (uint32_t)(k % p->depth);
  const bool reused = p->owner[b] != UINT64_MAX;
  // samples in: the buffer is free once the slot that last read it is done
  if (reused) MB_CUDA_TRY(cudaStreamWaitEvent(p->h2d, p->ev_done[b], 0));
  if (p->timer_armed) {
    MB_CUDA_TRY(cudaEventRecord(p->t_start, p->h2d));
    p->timer_armed = false;
    p->timer_started = true;
  }
  MB_CUDA_TRY(cudaMemcpyAsync(p->iq[b], iq_host, p->iq_bytes, cudaMemcpyHostToDevice, p->h2d));
  MB_CUDA_TRY(cudaEventRecord(p->ev_in[b], p->h2d));
  // the slot: after its samples, and after the results that last sat in
  // its output buffers have been copied out
  MB_CUDA_TRY(cudaStreamWaitEvent(p->comp, p->ev_in[b], 0));
  if (reused) MB_CUDA_TRY(cudaStreamWaitEvent(p->comp, p->ev_out[b], 0));
  mb_status r = mb_slot_uplink(p->slot, p->iq[b], p->llr[b], hard_host ? p->hard[b] : nullptr, p->status[b],
                               p->comp);
  if (r != MB_OK) return r;
  MB_CUDA_TRY(cudaEventRecord(p->ev_done[b], p->comp));
  // results out
  MB_CUDA_TRY(cudaStreamWaitEvent(p->d2h, p->ev_done[b], 0));
  MB_CUDA_TRY(cudaMemcpyAsync(llr_host, p->llr[b], p->llr_bytes, cudaMemcpyDeviceToHost, p->d2h));
  if (hard_host)
    MB_CUDA_TRY(cudaMemcpyAsync(hard_host, p->hard[b], p->hard_bytes, cudaMemcpyDeviceToHost, p->d2h));
  MB_CUDA_TRY(cudaEventRecord(p->ev_out[b], p->d2h));
  if (p->timer_started) MB_CUDA_TRY(cudaEventRecord(p->t_end, p->d2h));
  p->owner[b] = k;
  p->next = k + 1;
  if (ticket) *ticket = k;
  return MB_OK;
}

extern "C" mb_status mb_pipe_wait(mb_pipe *p, uint64_t ticket, uint32_t timeout_ms) {
  if (!p || ticket >= p->next) return MB_BAD_ARG;
  const uint32_t b = (uint32_t)(ticket % p->depth);
  // the buffer's last user is this ticket or a later one, which finishes
  // after it (the streams keep submission order)
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaEventQuery(p->ev_out[b]);
    if (e == cudaSuccess) return MB_OK;
    if (e != cudaErrorNotReady) return record_error(e);
    if (timeout_ms != UINT32_MAX &&
        std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms))
      return MB_TIMEOUT;
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

extern "C" mb_status mb_pipe_set_zf_init(mb_pipe *p, const mb_mlp *net) {
  if (!p || !p->slot) return MB_BAD_ARG;
  // no slot of the pipeline may be in flight while the choice changes
  if (p->comp) MB_CUDA_TRY(cudaStreamSynchronize(p->comp));
  return mb_slot_set_zf_init(p->slot, net);
}

extern "C" mb_status mb_pipe_io_bytes(const mb_pipe *p, uint64_t *iq, uint64_t *llr, uint64_t *hard) {
  if (!p || !iq || !llr || !hard) return MB_BAD_ARG;
  *iq = p->iq_bytes;
  *llr = p->llr_bytes;
  *hard = p->hard_bytes;
  return MB_OK;
}

extern "C" mb_status mb_pipe_timer_start(mb_pipe *p) {
  if (!p) return MB_BAD_ARG;
  p->timer_armed = true;
  p->timer_started = false;
  return MB_OK;
}

extern "C" mb_status mb_pipe_timer_ms(mb_pipe *p, double *ms) {
  if (!p || !ms || !p->timer_started) return MB_BAD_ARG;
  MB_CUDA_TRY(cudaEventSynchronize(p->t_end));
  float f = 0.f;
  MB_CUDA_TRY(cudaEventElapsedTime(&f, p->t_start, p->t_end));
  *ms = f;
  return MB_OK;
}

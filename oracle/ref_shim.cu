// ref_shim.cu -- TEST INFRASTRUCTURE ONLY: a C interface over the
// reference's own CUDA operators (UplinkFFT / PilotFFT, fft/fft_op.h:50-110;
// Beamform, beamform/beamform.h:27-84; Equalize, sgemv/equalize.h:70-73),
// compiled together with their sources by oracle/ref_ops.mk into
// oracle/_ref/libref_ops.so.  Used by the GPU parity tests and by the bench
// as the reference GPU baseline; the product package never loads it.
//
// ref_slot_uplink issues one uplink slot the way BandProcess::process does
// (baseband/process.cc:161-185): a pilot FFT per pilot symbol into the CSI
// (ue_start = p * sg), the beamformer (W in place, precoder into nmcsi),
// then per uplink symbol the FFT and the equalizer; all on one stream, so
// the host synchronisations of process.cc:167-173 are not needed.
//
// Samples are int16 pairs (ref_slot_create) or int8 pairs, the reference's
// production QuanT = char (utils/types.h:26; ref_slot_create_iq with
// iq8 = 1): the two sample types fft_op.cu:194-200 instantiates.
#include <cuda_fp16.h>

#include <cstdint>
#include <new>

#include "beamform/beamform.h"
#include "fft/fft_op.h"
#include "sgemv/equalize.h"

using namespace mega;

struct ref_slot {
  uint32_t M, K, N, S, sg, Qm, P, U, G, Gb;
  uint64_t cb_size, zeros, cb_stride;
  uint32_t iq8;  // 1: int8 samples, 0: int16
  UplinkFFT<short> *ufft = nullptr;
  PilotFFT<short> *pfft = nullptr;
  UplinkFFT<char> *ufft8 = nullptr;
  PilotFFT<char> *pfft8 = nullptr;
  Beamform *bf = nullptr;
  Complex *csi = nullptr, *nmcsi = nullptr, *y = nullptr;
};

template <typename QT>
static void ref_run(ref_slot *r, UplinkFFT<QT> *ufft, PilotFFT<QT> *pfft, const void *iq, void *llr,
                    cudaStream_t st) {
  const Matrix in_desc(2 * sizeof(QT), r->N, r->M);
  const Matrix csi_desc(sizeof(Complex), r->K, r->M, r->G);
  const Matrix csib_desc(sizeof(Complex), r->K, r->M, r->Gb);
  const Matrix y_desc(sizeof(Complex), r->S, r->M);
  const Matrix llr_desc(sizeof(half), (uint32_t)r->cb_stride, r->K);
  const char *iqb = reinterpret_cast<const char *>(iq);
  const size_t sym = (size_t)r->M * r->N * 2 * sizeof(QT);
  for (uint32_t p = 0; p < r->P; p++)
    (*pfft)(in_desc.wrap(const_cast<char *>(iqb) + p * sym), csi_desc.wrap(r->csi), p * r->sg, st);
  r->bf->beamformer(csib_desc.wrap(r->csi), csib_desc.wrap(r->nmcsi), st);
  for (uint32_t l = 0; l < r->U; l++) {
    (*ufft)(in_desc.wrap(const_cast<char *>(iqb) + (r->P + l) * sym), y_desc.wrap(r->y), st);
    Equalize::equalize(csi_desc.wrap(r->csi), y_desc.wrap(r->y),
                       llr_desc.wrap(reinterpret_cast<half *>(llr) + (size_t)l * r->K * r->cb_stride),
                       r->sg, (uint8_t)r->Qm, r->cb_size, r->zeros, 1, st);
  }
}

extern "C" {

void ref_slot_destroy(ref_slot *r);

ref_slot *ref_slot_create_iq(uint32_t M, uint32_t K, uint32_t N, uint32_t S, uint32_t sg, uint32_t Qm,
                             uint32_t P, uint32_t U, uint64_t cb_size, uint64_t zeros,
                             uint64_t cb_stride, uint32_t iq8) {
  ref_slot *r = new (std::nothrow) ref_slot();
  if (!r) return nullptr;
  r->M = M; r->K = K; r->N = N; r->S = S; r->sg = sg; r->Qm = Qm; r->P = P; r->U = U;
  r->cb_size = cb_size; r->zeros = zeros; r->cb_stride = cb_stride;
  r->iq8 = iq8 ? 1 : 0;
  r->G = (S + sg - 1) / sg;  // the pilot storer writes every subcarrier's group
  r->Gb = S / sg;            // the reference beamforms whole groups only
  const uint32_t start = (N - S) / 2;
  PilotSign::init(S);
  if (r->iq8) {
    r->ufft8 = new UplinkFFT<char>(start, N, S, M);
    r->pfft8 = new PilotFFT<char>(start, N, S, M, K, sg);
  } else {
    r->ufft = new UplinkFFT<short>(start, N, S, M);
    r->pfft = new PilotFFT<short>(start, N, S, M, K, sg);
  }
  r->bf = new Beamform(M, K, r->G);
  cudaMalloc(&r->csi, sizeof(Complex) * r->G * M * K);
  cudaMalloc(&r->nmcsi, sizeof(Complex) * r->G * M * K);
  cudaMalloc(&r->y, sizeof(Complex) * (size_t)M * S);
  cudaMemset(r->csi, 0, sizeof(Complex) * r->G * M * K);
  if (cudaGetLastError() != cudaSuccess) {
    ref_slot_destroy(r);
    return nullptr;
  }
  return r;
}

ref_slot *ref_slot_create(uint32_t M, uint32_t K, uint32_t N, uint32_t S, uint32_t sg, uint32_t Qm,
                          uint32_t P, uint32_t U, uint64_t cb_size, uint64_t zeros,
                          uint64_t cb_stride) {
  return ref_slot_create_iq(M, K, N, S, sg, Qm, P, U, cb_size, zeros, cb_stride, 0);
}

void ref_slot_destroy(ref_slot *r) {
  if (!r) return;
  delete r->ufft;
  delete r->pfft;
  delete r->ufft8;
  delete r->pfft8;
  delete r->bf;
  cudaFree(r->csi);
  cudaFree(r->nmcsi);
  cudaFree(r->y);
  delete r;
}

// iq: device [P+U][M][N] pairs of int16 (or int8, as created); llr: device
// [U][K][cb_stride] FP16
int ref_slot_uplink(ref_slot *r, const void *iq, void *llr, void *stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  try {
    if (r->iq8)
      ref_run(r, r->ufft8, r->pfft8, iq, llr, st);
    else
      ref_run(r, r->ufft, r->pfft, iq, llr, st);
  } catch (...) {
    return 1;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// device views of the slot's CSI / W [G][M][K] buffer
void *ref_slot_csi(ref_slot *r) { return r ? r->csi : nullptr; }

}  // extern "C"

// megastation_b200.hpp -- the reference's operator classes over the C ABI.
//
// Header-only C++ mirror of MegaStation's src/operators API with the same
// class names, constructor arguments and call signatures, so call sites such
// as BandProcess::process (baseband/process.cc:161-214) compile against it
// unchanged apart from the namespace.  Each method forwards to one entry
// point of megastation_b200.h; errors throw std::runtime_error like the
// reference's shape checks (beamform.cu:131-168, scrambler.cu:52-63).
// Matrix is a non-owning view with the reference's dims-fastest-first
// convention (matrix/matrix.h:95-117, Matrix::wrap :401-406).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>

#include "megastation_b200.h"

namespace mega_b200 {

inline void check(mb_status s, const char *where) {
  if (s != MB_OK) throw std::runtime_error(std::string(where) + ": " + mb_status_str(s));
}

// Non-owning strided view: dims[0] is the fastest dimension.
class Matrix {
 public:
  Matrix() = default;
  Matrix(void *data, size_t elem_bytes, uint64_t d0, uint64_t d1 = 1, uint64_t d2 = 1)
      : data_(data), elem_(elem_bytes), ndim_(d2 > 1 ? 3 : d1 > 1 ? 2 : 1) {
    dims_[0] = d0;
    dims_[1] = d1;
    dims_[2] = d2;
  }
  static Matrix wrap(void *data, size_t elem_bytes, uint64_t d0, uint64_t d1 = 1, uint64_t d2 = 1) {
    return Matrix(data, elem_bytes, d0, d1, d2);
  }
  template <typename T = void>
  T *ptr() const {
    return reinterpret_cast<T *>(data_);
  }
  uint64_t dim(int i) const { return dims_[i]; }
  int nDim() const { return ndim_; }
  // elements between consecutive indices of dimension i
  uint64_t stride(int i) const {
    uint64_t s = 1;
    for (int k = 0; k < i; k++) s *= dims_[k];
    return s;
  }
  uint64_t szBytes() const { return elem_ * dims_[0] * dims_[1] * dims_[2]; }

 private:
  void *data_ = nullptr;
  size_t elem_ = 0;
  uint64_t dims_[3] = {0, 1, 1};
  int ndim_ = 0;
};

template <typename QuanT>
constexpr int iq_dtype() {
  return sizeof(QuanT) == 1 ? MB_IQ_I8 : sizeof(QuanT) == 2 ? MB_IQ_I16 : MB_IQ_C32;
}

namespace detail {
struct FftDeleter {
  void operator()(mb_fft *f) const { mb_fft_destroy(f); }
};
inline std::shared_ptr<mb_fft> make_fft(uint32_t start, uint32_t ca, uint32_t num, uint32_t bs,
                                        uint32_t ue = 0, uint32_t sg = 0) {
  mb_fft_desc d{start, ca, num, bs, ue, sg};
  mb_fft *f = nullptr;
  check(mb_fft_create(&d, &f), "FFT");
  return std::shared_ptr<mb_fft>(f, FftDeleter());
}
inline uint32_t symbols_of(const Matrix &in, uint64_t per_symbol) {
  return (uint32_t)(in.dim(0) * in.dim(1) * in.dim(2) / per_symbol);
}
}  // namespace detail

// fft/fft_op.h:50-65
template <typename QuanT = short>
class UplinkFFT {
 public:
  UplinkFFT() = default;
  UplinkFFT(uint32_t ofdm_start, uint32_t ofdm_ca, uint32_t ofdm_num, uint32_t bs_num)
      : h_(detail::make_fft(ofdm_start, ofdm_ca, ofdm_num, bs_num)), ca_(ofdm_ca), bs_(bs_num) {}
  void operator()(const Matrix &in, const Matrix &out, cudaStream_t stream = nullptr) {
    check(mb_fft_uplink(h_.get(), in.ptr(), iq_dtype<QuanT>(),
                        detail::symbols_of(in, (uint64_t)ca_ * bs_), out.ptr<mb_c32>(), stream),
          "UplinkFFT");
  }

 private:
  std::shared_ptr<mb_fft> h_;
  uint32_t ca_ = 0, bs_ = 0;
};

// fft/fft_op.h:93-110 (PilotSign::init is implicit: the handle builds the table)
template <typename QuanT = short>
class PilotFFT {
 public:
  PilotFFT() = default;
  PilotFFT(uint32_t ofdm_start, uint32_t ofdm_ca, uint32_t ofdm_num, uint32_t bs_num, uint32_t ue_num,
           uint32_t sc_group)
      : h_(detail::make_fft(ofdm_start, ofdm_ca, ofdm_num, bs_num, ue_num, sc_group)),
        ca_(ofdm_ca),
        bs_(bs_num) {}
  void operator()(const Matrix &in, const Matrix &out, cudaStream_t stream = nullptr) {
    (*this)(in, out, 0, stream);
  }
  void operator()(const Matrix &in, const Matrix &out, uint32_t ue_start, cudaStream_t stream = nullptr) {
    check(mb_fft_pilot(h_.get(), in.ptr(), iq_dtype<QuanT>(), detail::symbols_of(in, (uint64_t)ca_ * bs_),
                       ue_start, out.ptr<mb_c32>(), stream),
          "PilotFFT");
  }

 private:
  std::shared_ptr<mb_fft> h_;
  uint32_t ca_ = 0, bs_ = 0;
};

// fft/fft_op.h:112-120
template <typename QuanT = short>
class DownlinkIFFT {
 public:
  DownlinkIFFT() = default;
  DownlinkIFFT(uint32_t ofdm_start, uint32_t ofdm_ca, uint32_t ofdm_num, uint32_t bs_num)
      : h_(detail::make_fft(ofdm_start, ofdm_ca, ofdm_num, bs_num)), ca_(ofdm_ca), bs_(bs_num) {}
  void operator()(const Matrix &in, const Matrix &out, cudaStream_t stream = nullptr) {
    check(mb_ifft_downlink(h_.get(), in.ptr<mb_c32>(), detail::symbols_of(in, (uint64_t)ca_ * bs_),
                           out.ptr(), iq_dtype<QuanT>(), stream),
          "DownlinkIFFT");
  }

 private:
  std::shared_ptr<mb_fft> h_;
  uint32_t ca_ = 0, bs_ = 0;
};

// beamform/beamform.h:27-84.  csi is (ue, bs, groups), precode (bs, ue, groups)
// in the reference's dims order.
class Beamform {
 public:
  Beamform() = default;
  Beamform(uint32_t num_bs, uint32_t num_ue, uint32_t batch_count, mb_zf_opts opts = {MB_ZF_FP32, 2, 1e4f, 0})
      : bs_(num_bs), ue_(num_ue), batch_(batch_count), opts_(opts) {
    mb_zf *z = nullptr;
    check(mb_zf_create(num_bs, num_ue, batch_count, &z), "Beamform");
    h_ = std::shared_ptr<mb_zf>(z, [](mb_zf *p) { mb_zf_destroy(p); });
  }
  // S: data subcarriers, sc_group: group size (they locate a short last group)
  void beamform_uplink(const Matrix &csi, uint32_t S, uint32_t sc_group, cudaStream_t stream = nullptr) {
    const uint32_t batch = (uint32_t)csi.dim(csi.nDim() - 1);
    if (batch > batch_)
      throw std::runtime_error("Batch size " + std::to_string(batch) + " exceeds the maximum batch size " +
                               std::to_string(batch_));
    check(mb_zf_uplink(h_.get(), csi.ptr<mb_c32>(), batch, S, sc_group, &opts_, nullptr, nullptr, stream),
          "Beamform::beamform_uplink");
  }
  void beamformer(const Matrix &csi, const Matrix &precode, uint32_t S, uint32_t sc_group,
                  cudaStream_t stream = nullptr) {
    if (precode.nDim() != csi.nDim() || csi.dim(csi.nDim() - 1) != precode.dim(precode.nDim() - 1))
      throw std::runtime_error("Csi & Precode mismatch");
    beamform_uplink(csi, S, sc_group, stream);
    beamform_downlink(csi, precode, stream);
  }
  static void beamform_downlink(const Matrix &csi, const Matrix &precode, cudaStream_t stream = nullptr) {
    const uint32_t batch = (uint32_t)csi.dim(csi.nDim() - 1);
    const uint32_t ue = (uint32_t)csi.dim(0), bs = (uint32_t)csi.dim(1);
    if (precode.nDim() != csi.nDim() || batch != precode.dim(precode.nDim() - 1))
      throw std::runtime_error("Csi & Precode mismatch");
    if (bs != precode.dim(0) || ue != precode.dim(1)) throw std::runtime_error("Precode dimension mismatch");
    check(mb_zf_precoder(csi.ptr<mb_c32>(), precode.ptr<mb_c32>(), bs, ue, csi.nDim() == 3 ? batch : 1, stream),
          "Beamform::beamform_downlink");
  }

 private:
  std::shared_ptr<mb_zf> h_;
  uint32_t bs_ = 0, ue_ = 0, batch_ = 0;
  mb_zf_opts opts_{};
};

// sgemv/equalize.h:70-73.  csi (ue, bs[, groups]), bsVec (S, bs[, syms]),
// ueVec (cb_stride, ue * cb_blocks[, syms]) halves.
struct Equalize {
  static void equalize(const Matrix &csi, const Matrix &bsVec, const Matrix &ueVec, uint64_t csi_skip,
                       uint8_t mod_order, uint64_t cb_size, uint64_t zeros, uint16_t cb_blocks,
                       cudaStream_t stream = nullptr) {
    const uint32_t K = (uint32_t)csi.dim(0), M = (uint32_t)csi.dim(1), S = (uint32_t)bsVec.dim(0);
    const uint32_t n_sym = (uint32_t)(bsVec.dim(2) > 1 ? bsVec.dim(2) : 1);
    check(mb_equalize(csi.ptr<mb_c32>(), bsVec.ptr<mb_c32>(), K, M, S, (uint32_t)csi_skip, n_sym, mod_order,
                      cb_size, ueVec.stride(1), zeros, cb_blocks, ueVec.ptr<uint16_t>(), nullptr, nullptr,
                      nullptr, stream),
          "Equalize::equalize");
  }
};

// sgemv/precode.h:59-61.  precoded (bs, ue[, groups]), ueVec (S, ue),
// bsVec (N, bs).
struct Precode {
  static void precode(const Matrix &precoded, const Matrix &ueVec, const Matrix &bsVec, uint64_t precode_skip,
                      uint64_t bs_start, cudaStream_t stream = nullptr) {
    const uint32_t M = (uint32_t)precoded.dim(0), K = (uint32_t)precoded.dim(1);
    const uint32_t S = (uint32_t)ueVec.dim(0), N = (uint32_t)bsVec.stride(1);
    check(mb_precode(precoded.ptr<mb_c32>(), ueVec.ptr<mb_c32>(), M, K, S, (uint32_t)precode_skip, N,
                     (uint32_t)bs_start, 1, bsVec.ptr<mb_c32>(), stream),
          "Precode::precode");
  }
};

// modulation/modulation.h:27-90 (order and DM-RS table given per call).
struct Modulation {
  static void modulate(const Matrix &in, const Matrix &out, uint32_t mod_order, uint32_t pilot_spacing = 0,
                       const mb_c32 *pilot_table = nullptr, cudaStream_t stream = nullptr) {
    check(mb_modulate(in.ptr<uint8_t>(), out.ptr<mb_c32>(), in.dim(0), out.dim(0), out.dim(1), mod_order,
                      pilot_spacing, pilot_table, stream),
          "Modulation::modulate");
  }
};

// scrambler/scrambler.h:32-75
struct Scrambler {
  static void scrambler(const Matrix &out_data, const Matrix &in_data, cudaStream_t stream = nullptr) {
    const uint64_t bytes = out_data.dim(0), batch = out_data.nDim() == 1 ? 1 : out_data.dim(1);
    if (out_data.nDim() != in_data.nDim() || bytes != in_data.dim(0) ||
        batch != (in_data.nDim() == 1 ? 1 : in_data.dim(1)))
      throw std::runtime_error("Input and output mismatch");
    check(mb_scramble(out_data.ptr<uint8_t>(), in_data.ptr<uint8_t>(), bytes, batch, stream),
          "Scrambler::scrambler");
  }
};

}  // namespace mega_b200

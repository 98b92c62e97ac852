// Drives the reference's golden unit-test cases through the C++ mirror of
// the operator classes (include/megastation_b200.hpp): the call shapes of
// test/sgemv/test_sgemv.cc:126-196, test/fft/test_fft.cc:106-215 and
// test/beamform/test_beamform.cc:67-95.  Exit status 0 = all match.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <vector>

#include "megastation_b200.hpp"

using mega_b200::Matrix;

static std::vector<char> load(const std::string &dir, const char *name) {
  std::ifstream f(dir + "/" + name, std::ios::binary);
  return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

template <typename T>
static T *dev(const std::vector<char> &h) {
  void *p = nullptr;
  cudaMalloc(&p, h.size());
  cudaMemcpy(p, h.data(), h.size(), cudaMemcpyHostToDevice);
  return reinterpret_cast<T *>(p);
}

static int fails = 0;
static void expect(bool ok, const char *what) {
  if (!ok) {
    std::printf("FAIL %s\n", what);
    fails++;
  }
}

int main(int argc, char **argv) {
  const std::string g = argc > 1 ? argv[1] : "tests/golden";
  // Equalize: K=4, M=8, 16 subcarriers, QPSK, cb 32, bit-exact FP16
  {
    auto csi = load(g, "sgemv/csi.data"), bs = load(g, "sgemv/bsVec.data"), ref = load(g, "sgemv/equalize.data");
    std::vector<char> bst(bs.size());
    const float *src = reinterpret_cast<const float *>(bs.data());
    float *dst = reinterpret_cast<float *>(bst.data());
    for (int i = 0; i < 16; i++)
      for (int j = 0; j < 8; j++) {
        dst[2 * (j * 16 + i)] = src[2 * (i * 8 + j)];
        dst[2 * (j * 16 + i) + 1] = src[2 * (i * 8 + j) + 1];
      }
    auto *dc = dev<char>(csi);
    auto *db = dev<char>(bst);
    void *dl = nullptr;
    cudaMalloc(&dl, ref.size());
    mega_b200::Equalize::equalize(Matrix(dc, 8, 4, 8), Matrix(db, 8, 16, 8), Matrix(dl, 2, 32, 4), 16, 2, 32, 0, 1);
    std::vector<char> out(ref.size());
    cudaMemcpy(out.data(), dl, out.size(), cudaMemcpyDeviceToHost);
    expect(std::memcmp(out.data(), ref.data(), ref.size()) == 0, "equalize golden (bit-exact)");
  }
  // Downlink IFFT: int16 out, bit-exact
  {
    auto in = load(g, "fft/ifft_in.data"), ref = load(g, "fft/ifft_out.data");
    auto *di = dev<char>(in);
    void *dout = nullptr;
    cudaMalloc(&dout, ref.size());
    mega_b200::DownlinkIFFT<short> ifft(8, 32, 16, 8);
    ifft(Matrix(di, 8, 32, 8), Matrix(dout, 4, 32, 8));
    std::vector<char> out(ref.size());
    cudaMemcpy(out.data(), dout, out.size(), cudaMemcpyDeviceToHost);
    expect(std::memcmp(out.data(), ref.data(), ref.size()) == 0, "downlink ifft golden (bit-exact)");
  }
  // Uplink FFT: int16 in, tolerance 1e-5
  {
    auto in = load(g, "fft/fft_in.data"), ref = load(g, "fft/fft_out.data");
    auto *di = dev<char>(in);
    void *dout = nullptr;
    cudaMalloc(&dout, 8 * 16 * 8);
    mega_b200::UplinkFFT<short> fft(8, 32, 16, 8);
    fft(Matrix(di, 4, 32, 8), Matrix(dout, 8, 16, 8));
    std::vector<float> out(8 * 16 * 2);
    cudaMemcpy(out.data(), dout, out.size() * 4, cudaMemcpyDeviceToHost);
    const float *r = reinterpret_cast<const float *>(ref.data());  // [16][8]
    double err = 0;
    for (int b = 0; b < 8; b++)
      for (int i = 0; i < 16; i++)
        for (int c = 0; c < 2; c++)
          err = std::fmax(err, std::fabs(out[2 * (b * 16 + i) + c] - r[2 * (i * 8 + b) + c]));
    expect(err <= 1e-5, "uplink fft golden (1e-5)");
  }
  // Beamform: K=4, M=8, two identical groups, tolerance 1e-5
  {
    auto csi = load(g, "beamform/csi_in.data"), rw = load(g, "beamform/csi_out.data"),
         rp = load(g, "beamform/precoder.data");
    std::vector<char> two(csi);
    two.insert(two.end(), csi.begin(), csi.end());
    auto *dc = dev<char>(two);
    void *dp = nullptr;
    cudaMalloc(&dp, two.size());
    mega_b200::Beamform beam(8, 4, 2);
    beam.beamformer(Matrix(dc, 8, 4, 8, 2), Matrix(dp, 8, 8, 4, 2), 32, 16);
    std::vector<float> w(two.size() / 4), p(two.size() / 4);
    cudaMemcpy(w.data(), dc, two.size(), cudaMemcpyDeviceToHost);
    cudaMemcpy(p.data(), dp, two.size(), cudaMemcpyDeviceToHost);
    const float *a = reinterpret_cast<const float *>(rw.data()), *b = reinterpret_cast<const float *>(rp.data());
    double ew = 0, ep = 0;
    for (int gidx = 0; gidx < 2; gidx++)
      for (int i = 0; i < 64; i++) {
        ew = std::fmax(ew, std::fabs(w[gidx * 64 + i] - a[i]));
        ep = std::fmax(ep, std::fabs(p[gidx * 64 + i] - b[i]));
      }
    expect(ew <= 1e-5 && ep <= 1e-5, "beamform golden (1e-5)");
  }
  // error behaviour: the reference throws on a batch above the maximum
  {
    bool threw = false;
    try {
      mega_b200::Beamform beam(8, 4, 1);
      beam.beamform_uplink(Matrix(nullptr, 8, 4, 8, 2), 32, 16);
    } catch (const std::runtime_error &) {
      threw = true;
    }
    expect(threw, "batch above maximum throws");
  }
  std::printf(fails ? "shim: %d failures\n" : "shim: all golden cases match\n", fails);
  return fails ? 1 : 0;
}

"""The tensor-core downlink operators against the FP64 oracle: the precode
on tcgen05 (mb_precode_tc: BF16 operands, FP32 accumulation, FP16 spectra
out; precode_kernel.cuh:255-262 with the FFT-shift scatter) and the inverse
FFT on the tensor cores with the output quantiser (mb_ifft_downlink_mixed:
FP16 operands, FP32 accumulation; fft_op.cu:167-174, ifft_callback.cuh:21-59).
Tolerances: the spectra within 1% of their RMS (BF16 operands), the time
samples within 0.5% of their RMS plus one LSB of the integer formats (FP16
operands, FP16 intermediate), the guard bins untouched."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mb():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import megastation_b200 as m
    return m


@pytest.mark.parametrize("M,K,S,sg,N,D", [(256, 64, 3276, 16, 4096, 5), (64, 16, 1200, 16, 2048, 3),
                                          (200, 20, 600, 8, 1024, 9)])
def test_precode_tc_vs_oracle(mb, M, K, S, sg, N, D):
    rng = np.random.default_rng(M + K + D)
    G = (S + sg - 1) // sg
    start = (N - S) // 2
    P = ((rng.standard_normal((G, K, M)) + 1j * rng.standard_normal((G, K, M))) / np.sqrt(2 * K)).astype(np.complex64)
    s = ((rng.standard_normal((D, K, S)) + 1j * rng.standard_normal((D, K, S))) / np.sqrt(2)).astype(np.complex64)
    z = torch.full((D, M, N, 2), 7.0, dtype=torch.float16, device="cuda")  # sentinel in the guard bins
    mb.Precode.precode_tc(torch.from_numpy(P).cuda(), torch.from_numpy(s).cuda(), z, sg, start)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    got = z.cpu().numpy().astype(np.float32)
    got = got[..., 0] + 1j * got[..., 1]
    bins = (np.arange(S) + start + N // 2) % N
    guard = np.ones(N, bool)
    guard[bins] = False
    for l in range(D):
        ref = orc.precode(P, s[l], sg, N, start)
        rms = np.sqrt(np.mean(np.abs(ref[:, bins]) ** 2))
        err = np.abs(got[l][:, bins] - ref[:, bins])
        assert np.sqrt(np.mean(err ** 2)) <= 1e-2 * rms and err.max() <= 8e-2 * rms, (l, err.max() / rms)
        assert (got[l][:, guard] == 7.0 + 7.0j).all()


@pytest.mark.parametrize("out_dtype", ["int16", "int8", "f16"])
@pytest.mark.parametrize("in_dtype", ["f16", "c64"])
def test_ifft_tc_vs_oracle(mb, in_dtype, out_dtype):
    M, N, S, D = 32, 4096, 3276, 3
    rng = np.random.default_rng(5)
    start = (N - S) // 2
    bins = (np.arange(S) + start + N // 2) % N
    x = np.zeros((D, M, N), np.complex64)
    # spectra sized so that the time samples span many LSBs of the format
    amp = {"int16": 0.05, "int8": 2.0, "f16": 1.0}[out_dtype]
    x[..., bins] = (amp * (rng.standard_normal((D, M, S)) + 1j * rng.standard_normal((D, M, S)))).astype(np.complex64)
    if in_dtype == "f16":
        xin = torch.from_numpy(np.stack([x.real, x.imag], -1).astype(np.float16)).cuda()
        x = xin.cpu().numpy().astype(np.float32)
        x = (x[..., 0] + 1j * x[..., 1]).astype(np.complex64)
    else:
        xin = torch.from_numpy(x).cuda()
    tdt = {"int16": torch.int16, "int8": torch.int8, "f16": torch.float16}[out_dtype]
    ndt = {"int16": np.int16, "int8": np.int8, "f16": np.float16}[out_dtype]
    out = torch.zeros(D, M, N, 2, dtype=tdt, device="cuda")
    mb.DownlinkIFFT(start, N, S, M).mixed(xin, out)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    got = out.cpu().numpy().astype(np.float64)
    ref = np.stack([orc.ifft_downlink(x[l], ndt) for l in range(D)]).astype(np.float64)
    rms = np.sqrt(np.mean(ref ** 2))
    lsb = 1.0 if out_dtype != "f16" else 0.0
    err = np.abs(got - ref)
    assert rms > (20.0 if out_dtype == "int16" else 2.0 if out_dtype == "int8" else 1e-3)
    assert np.sqrt(np.mean(err ** 2)) <= 5e-3 * rms + lsb, (np.sqrt(np.mean(err ** 2)), rms)
    assert err.max() <= 5e-2 * np.abs(ref).max() + lsb

"""Mixed-precision uplink FFT (planar BF16 rows for the tensor-core
equalizer) against the FP64 oracle FFT.  For N = 4096 the butterflies run on
the tensor cores (FP16 operands, rows scaled by powers of two, FP32
accumulation); other sizes and unaligned row pitches take the FP32 kernel.
Tolerance per output: BF16 rounding (2^-8 of the value) plus 2e-3 of the
row's RMS for the FP16 operands."""
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


def make_iq(x, dtype):
    if dtype == "c64":
        return x.astype(np.complex64)
    if dtype == "f16":
        return np.stack([x.real, x.imag], -1).astype(np.float16)
    qm = 32767 if dtype == "int16" else 127
    iq = np.clip(np.rint(np.stack([x.real, x.imag], -1) * (qm + 1)), -qm - 1, qm)
    return iq.astype(np.int16 if dtype == "int16" else np.int8)


def run_bf16(mb, iq, N, S, M, n_sym, pitch, start=None, sentinel=7.0):
    start = (N - S) // 2 if start is None else start
    out = torch.full((n_sym, 2, M, pitch), sentinel, dtype=torch.bfloat16, device="cuda")
    mb.UplinkFFT(start, N, S, M).uplink_bf16(torch.from_numpy(np.ascontiguousarray(iq)).cuda(), out, pitch)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    o = out.float().cpu().numpy()
    return o[:, 0] + 1j * o[:, 1], o, start


def check_rows(got, iq, N, S, start):
    for l in range(got.shape[0]):
        ref = orc.uplink_fft(iq[l], N, S, start)
        rms = np.sqrt(np.mean(np.abs(ref) ** 2, axis=-1, keepdims=True))
        err = np.abs(got[l, :, :S] - ref)
        tol = 2.0 ** -8 * np.abs(ref) + 2e-3 * rms + 1e-30
        assert (err <= tol).all(), (l, (err / tol).max())


@pytest.mark.parametrize("dtype", ["c64", "int16", "int8", "f16"])
@pytest.mark.parametrize("M,n_sym", [(4, 3), (3, 3)])
def test_fft_tc_4096_vs_oracle(mb, dtype, M, n_sym):
    N, S = 4096, 3276
    rng = np.random.default_rng(M * 10 + n_sym)
    x = (rng.standard_normal((n_sym, M, N)) + 1j * rng.standard_normal((n_sym, M, N))) * 0.1
    iq = make_iq(x, dtype)
    s8 = (S + 7) // 8 * 8
    got, o, start = run_bf16(mb, iq, N, S, M, n_sym, s8 + 16)
    check_rows(got, iq, N, S, start)
    # columns from S rounded up to 8 on are left as they were
    assert (o[..., s8:] == 7.0).all()


def test_fft_tc_row_scaling(mb):
    # rows 10 orders of magnitude apart, a zero row and an impulse: each is
    # scaled on its own, so relative accuracy holds for all of them
    N, S, M = 4096, 3276, 4
    rng = np.random.default_rng(3)
    x = rng.standard_normal((1, M, N)) + 1j * rng.standard_normal((1, M, N))
    x[0, 0] *= 1e-6
    x[0, 1] *= 1e4
    x[0, 2] = 0
    x[0, 3] = 0
    x[0, 3, 17] = 3.0 - 2.0j
    iq = x.astype(np.complex64)
    got, _, start = run_bf16(mb, iq, N, S, M, 1, S + 4)
    check_rows(got, iq, N, S, start)
    assert (got[0, 2, :S] == 0).all()


@pytest.mark.parametrize("N,S,start", [(4096, 4096, 0), (4096, 1200, 100), (4096, 3300, 1000)])
def test_fft_tc_band_placement(mb, N, S, start):
    # full band, a band well inside, and one that wraps past bin N-1
    rng = np.random.default_rng(S)
    x = (rng.standard_normal((2, 2, N)) + 1j * rng.standard_normal((2, 2, N))).astype(np.complex64)
    got, _, st = run_bf16(mb, x, N, S, 2, 2, (S + 7) // 8 * 8, start=start)
    check_rows(got, x, N, S, st)


@pytest.mark.parametrize("N,S,pitch", [(2048, 1200, 1200), (4096, 3276, 3277)])
def test_fft_bf16_fp32_kernel(mb, N, S, pitch):
    # sizes and pitches the tensor-core kernel does not take run in FP32
    rng = np.random.default_rng(N)
    x = (rng.standard_normal((2, 3, N)) + 1j * rng.standard_normal((2, 3, N))).astype(np.complex64)
    got, o, start = run_bf16(mb, x, N, S, 3, 2, pitch)
    check_rows(got, x, N, S, start)
    assert (o[..., S:] == 7.0).all()


@pytest.mark.parametrize("dtype,M,K,sg", [("c64", 4, 20, 16), ("int16", 5, 32, 16), ("c64", 3, 8, 8)])
def test_pilot_fft_mixed_vs_oracle(mb, dtype, M, K, sg):
    # LS pilot estimates from the tensor-core FFT: within 2e-3 of the RMS
    # estimate (FP16 operands) of the FP64 oracle
    N, S = 4096, 3276
    rng = np.random.default_rng(K + M)
    P = (K + sg - 1) // sg
    x = (rng.standard_normal((P, M, N)) + 1j * rng.standard_normal((P, M, N))) * 0.1
    iq = make_iq(x, dtype)
    start = (N - S) // 2
    G = (S + sg - 1) // sg
    csi = torch.zeros(G, M, K, dtype=torch.complex64, device="cuda")
    mb.PilotFFT(start, N, S, M, K, sg).mixed(torch.from_numpy(np.ascontiguousarray(iq)).cuda(), csi)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    ref = np.zeros((G, M, K), np.complex64)
    ps = orc.pilot_sign(S)
    for p in range(P):
        orc.pilot_fft(iq[p], N, S, start, K, sg, p * sg, ps, ref)
    got = csi.cpu().numpy()
    scale = np.sqrt(np.mean(np.abs(ref) ** 2))
    assert np.abs(got - ref).max() <= 2e-3 * scale


def test_fft_tc_many_units_per_cta(mb):
    # the bench's launch size: 12 symbols x 256 antennas = 1536 two-row units,
    # about 11 per CTA, so every ring slot and barrier of the pipeline turns
    # over many times (a barrier phase mix-up shows as a device error)
    N, S, M, n_sym = 4096, 3276, 256, 12
    rng = np.random.default_rng(99)
    # rows 2^-8 .. 2^8 apart, so a row scaled with another row's factor shows
    row_gain = 2.0 ** rng.integers(-8, 9, size=(n_sym, M, 1))
    x = ((rng.standard_normal((n_sym, M, N)) + 1j * rng.standard_normal((n_sym, M, N))) * row_gain).astype(np.complex64)
    got, _, start = run_bf16(mb, x, N, S, M, n_sym, (S + 7) // 8 * 8)
    check_rows(got[::5], x[::5], N, S, start)


def test_pilot_fft_mixed_many_units(mb):
    N, S, M, K, sg = 4096, 3276, 256, 64, 16
    P = K // sg
    rng = np.random.default_rng(7)
    row_gain = 2.0 ** rng.integers(-4, 5, size=(P, M, 1))
    x = ((rng.standard_normal((P, M, N)) + 1j * rng.standard_normal((P, M, N))) * row_gain).astype(np.complex64)
    start = (N - S) // 2
    G = (S + sg - 1) // sg
    csi = torch.zeros(G, M, K, dtype=torch.complex64, device="cuda")
    mb.PilotFFT(start, N, S, M, K, sg).mixed(torch.from_numpy(x).cuda(), csi)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    ref = np.zeros((G, M, K), np.complex64)
    ps = orc.pilot_sign(S)
    for p in range(P):
        orc.pilot_fft(x[p], N, S, start, K, sg, p * sg, ps, ref)
    # per (antenna, pilot symbol): each row has its own gain; user u's
    # estimate comes from pilot symbol u // sg
    got = csi.cpu().numpy().reshape(G, M, P, sg)
    r = ref.reshape(G, M, P, sg)
    scale = np.sqrt(np.mean(np.abs(r) ** 2, axis=(0, 3), keepdims=True))
    ratio = np.abs(got - r) / (2e-3 * scale)
    assert ratio.max() <= 1.0, (ratio.max(), np.unravel_index(ratio.argmax(), ratio.shape))

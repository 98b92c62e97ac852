"""GPU parity of every operator against the reference's golden vectors and
the CPU oracle, called through the C ABI (megastation_b200.ops -> ctypes ->
libmegastation_b200.so).

Tolerances: FFT outputs 1e-5 absolute on the golden cases (the reference's own
test tolerance, test/fft/test_fft.cc:141-172) and 2e-6 relative to the row RMS
on random cases; ZF W within 1e-5 (test_beamform.cc:91-92) on the golden case;
LLRs bit-exact on the golden case (test_sgemv.cc:156-158) and, on random cases,
hard bits bit-exact wherever |LLR_oracle| > 0.5 with FP16 LLRs within
4 ulp + 1e-3 * |x| scaled.
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def gold(sub, name, dtype):
    return np.fromfile(os.path.join(GOLD, sub, name + ".data"), dtype=dtype)


@pytest.fixture(scope="module")
def mb():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import megastation_b200 as m
    return m


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


# ------------------------------------------------------------------ golden
def test_uplink_fft_golden(mb):
    iq = gold("fft", "fft_in", np.int16).reshape(8, 32, 2)
    ref = gold("fft", "fft_out", np.complex64).reshape(16, 8)
    out = torch.zeros(8, 16, dtype=torch.complex64, device="cuda")
    mb.UplinkFFT(8, 32, 16, 8)(dev(iq), out)
    np.testing.assert_allclose(host(out).T, ref, atol=1e-5)


def test_pilot_fft_golden(mb):
    iq = gold("fft", "short_in", np.int16).reshape(8, 32, 2)
    ref = gold("fft", "complex_out", np.complex64).reshape(4, 8, 4)
    csi = torch.zeros(4, 8, 4, dtype=torch.complex64, device="cuda")
    mb.PilotFFT(8, 32, 16, 8, 4, 4)(dev(iq), csi)
    np.testing.assert_allclose(host(csi), ref, atol=1e-4)


def test_downlink_ifft_golden_bit_exact(mb):
    x = gold("fft", "ifft_in", np.complex64).reshape(8, 32)
    ref = gold("fft", "ifft_out", np.int16).reshape(8, 32, 2)
    out = torch.zeros(8, 32, 2, dtype=torch.int16, device="cuda")
    mb.DownlinkIFFT(8, 32, 16, 8)(dev(x), out)
    np.testing.assert_array_equal(host(out), ref)


def test_beamform_golden(mb):
    c = gold("beamform", "csi_in", np.complex64).reshape(1, 8, 4)
    csi = dev(np.concatenate([c, c]))
    prec = torch.zeros(2, 4, 8, dtype=torch.complex64, device="cuda")
    mb.Beamform(8, 4, 2).beamformer(csi, prec, S=32, sc_group=16)
    ref_w = gold("beamform", "csi_out", np.complex64).reshape(8, 4)
    ref_p = gold("beamform", "precoder", np.complex64).reshape(4, 8)
    W, P = host(csi), host(prec)
    for g in range(2):
        np.testing.assert_allclose(W[g], ref_w, atol=1e-5)
        np.testing.assert_allclose(P[g], ref_p, atol=1e-5)


def test_equalize_golden_bit_exact(mb):
    W = gold("sgemv", "csi", np.complex64).reshape(1, 8, 4)
    y = gold("sgemv", "bsVec", np.complex64).reshape(16, 8).T.copy()
    ref = gold("sgemv", "equalize", np.uint16).reshape(4, 32)
    llr = torch.zeros(4, 32, dtype=torch.float16, device="cuda")
    mb.Equalize.equalize(dev(W), dev(y), llr, 16, 2, 32, 0, 1)
    np.testing.assert_array_equal(host(llr).view(np.uint16), ref)


def test_precode_golden(mb):
    P = gold("sgemv", "prec", np.complex64).reshape(1, 4, 8)
    s = gold("sgemv", "ueVec", np.complex64).reshape(16, 4).T.copy()
    ref = gold("sgemv", "precoded", np.complex64).reshape(8, 32)
    out = torch.full((8, 32), 7.0 + 7.0j, dtype=torch.complex64, device="cuda")
    mb.Precode.precode(dev(P), dev(s), out, 16, 8)
    np.testing.assert_allclose(host(out), ref, atol=1e-5)


def test_modulate_64qam_round_trip(mb):
    vals = np.arange(64, dtype=np.uint8)
    bits = ((vals[:, None] >> np.arange(6)) & 1).astype(np.uint8).ravel()
    packed = np.tile(np.packbits(bits, bitorder="little"), (4, 1))
    out = torch.zeros(4, 64, dtype=torch.complex64, device="cuda")
    mb.Modulation.modulate(dev(packed), out, 6)
    sym = host(out)
    np.testing.assert_array_equal(sym, orc.modulate(packed, 64, 6))
    for u in range(4):
        llr = orc.demod(6, sym[u])
        got = ((llr.astype(np.float32) < 0).astype(np.int64) << np.arange(6)).sum(1)
        np.testing.assert_array_equal(got, vals)


def test_scrambler_involution_and_oracle(mb):
    rng = np.random.default_rng(3)
    data = rng.integers(0, 256, (4, 137), dtype=np.uint8)
    d = dev(data)
    out = torch.empty_like(d)
    mb.Scrambler.scrambler(out, d)
    np.testing.assert_array_equal(host(out), orc.scramble_bytes(data))
    mb.Scrambler.scrambler(out, out)
    np.testing.assert_array_equal(host(out), data)
    hello = dev(np.frombuffer(b"Hello World!\0", np.uint8).copy())
    mb.Scrambler.scrambler(hello, hello)
    mb.Scrambler.scrambler(hello, hello)
    assert bytes(host(hello)) == b"Hello World!\0"


# ------------------------------------------------------------- random cases
@pytest.mark.parametrize("N,S,M,n_sym,dtype", [
    (64, 48, 4, 1, "c64"), (256, 200, 8, 3, "int16"), (1024, 600, 16, 2, "int8"),
    (2048, 1200, 8, 2, "c64"), (4096, 3276, 4, 2, "f16"), (8192, 6552, 2, 1, "c64"),
    (16, 12, 3, 5, "c64"), (512, 300, 5, 1, "int16")])
def test_uplink_fft_vs_oracle(mb, N, S, M, n_sym, dtype):
    rng = np.random.default_rng(N + M)
    x = (rng.standard_normal((n_sym, M, N)) + 1j * rng.standard_normal((n_sym, M, N))) * 0.1
    if dtype == "c64":
        iq = x.astype(np.complex64)
    elif dtype == "f16":
        iq = np.stack([x.real, x.imag], -1).astype(np.float16)
    else:
        qm = 32767 if dtype == "int16" else 127
        iq = np.clip(np.rint(np.stack([x.real, x.imag], -1) * (qm + 1)), -qm - 1, qm)
        iq = iq.astype(np.int16 if dtype == "int16" else np.int8)
    start = (N - S) // 2
    out = torch.zeros(n_sym, M, S, dtype=torch.complex64, device="cuda")
    mb.UplinkFFT(start, N, S, M)(dev(iq), out)
    got = host(out)
    for l in range(n_sym):
        ref = orc.uplink_fft(iq[l], N, S, start)
        scale = np.sqrt(np.mean(np.abs(ref) ** 2))
        assert np.abs(got[l] - ref).max() <= 2e-6 * scale * np.log2(N), (l, np.abs(got[l] - ref).max(), scale)


@pytest.mark.parametrize("N,S,M,K,sg", [(256, 200, 8, 8, 4), (2048, 1200, 16, 32, 16), (4096, 3276, 4, 20, 16)])
def test_pilot_fft_vs_oracle(mb, N, S, M, K, sg):
    rng = np.random.default_rng(K)
    P = (K + sg - 1) // sg
    x = ((rng.standard_normal((P, M, N)) + 1j * rng.standard_normal((P, M, N))) * 0.1).astype(np.complex64)
    start = (N - S) // 2
    G = (S + sg - 1) // sg
    csi = torch.zeros(G, M, K, dtype=torch.complex64, device="cuda")
    mb.PilotFFT(start, N, S, M, K, sg)(dev(x), csi)
    ref = np.zeros((G, M, K), np.complex64)
    ps = orc.pilot_sign(S)
    for p in range(P):
        orc.pilot_fft(x[p], N, S, start, K, sg, p * sg, ps, ref)
    got = host(csi)
    scale = np.sqrt(np.mean(np.abs(ref) ** 2))
    assert np.abs(got - ref).max() <= 3e-6 * scale * np.log2(N)


@pytest.mark.parametrize("out_dtype", [np.int16, np.int8, np.float16, np.complex64])
def test_ifft_vs_oracle(mb, out_dtype):
    rng = np.random.default_rng(11)
    M, N = 6, 2048
    x = ((rng.standard_normal((2, M, N)) + 1j * rng.standard_normal((2, M, N))) * 30).astype(np.complex64)
    if out_dtype == np.complex64:
        out = torch.zeros(2, M, N, dtype=torch.complex64, device="cuda")
    else:
        out = torch.zeros(2, M, N, 2, dtype=getattr(torch, np.dtype(out_dtype).name), device="cuda")
    mb.DownlinkIFFT(0, N, N, M)(dev(x), out)
    got = host(out)
    for l in range(2):
        ref = orc.ifft_downlink(x[l], out_dtype)
        if out_dtype in (np.int16, np.int8):
            assert np.abs(got[l].astype(np.int32) - ref.astype(np.int32)).max() <= 1
        else:
            g = got[l].astype(np.complex64 if out_dtype == np.complex64 else np.float32)
            r = ref.astype(g.dtype)
            tol = 2e-6 if out_dtype == np.complex64 else 2e-3
            assert np.abs(g - r).max() <= tol * np.abs(r).max()


@pytest.mark.parametrize("M,K,G,S,sg", [(8, 4, 3, 48, 16), (64, 16, 10, 150, 16), (256, 32, 5, 80, 16),
                                        (128, 64, 3, 40, 16), (16, 16, 4, 64, 16), (32, 5, 6, 90, 16)])
def test_zf_fp32_vs_oracle(mb, M, K, G, S, sg):
    rng = np.random.default_rng(M * K)
    csi = ((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K))) / np.sqrt(2)).astype(np.complex64)
    d = dev(csi)
    status = torch.full((G,), -1, dtype=torch.int32, device="cuda")
    mb.Beamform(M, K, G).beamform_uplink(d, S=S, sc_group=sg, status=status)
    W, cond, bad = orc.zf(csi, S=S, sg=sg, with_cond=True)
    got = host(d)
    assert (host(status) == 0).all()
    for g in range(G):
        # FP32 Cholesky: error grows with cond(Gram)
        tol = 2e-6 * cond[g] * np.abs(W[g]).max() + 1e-7
        assert np.abs(got[g] - W[g]).max() <= tol, (g, cond[g])


def test_zf_not_positive_definite_reports(mb):
    # host-built singular Grams: two identical users, and an all-zero group
    M, K, G = 16, 4, 3
    rng = np.random.default_rng(5)
    csi = ((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K)))).astype(np.complex64)
    csi[1, :, 2] = csi[1, :, 1]
    csi[2] = 0
    d = dev(csi)
    status = torch.full((G,), -1, dtype=torch.int32, device="cuda")
    mb.Beamform(M, K, G).beamform_uplink(d, S=G * 16, sc_group=16, status=status)
    st = host(status)
    assert st[0] == 0 and st[2] == 1
    assert st[1] in (0, 1)  # exact singularity may round to a tiny pivot
    assert (host(d)[2] == 0).all()


def test_zf_fp64_vs_oracle(mb):
    rng = np.random.default_rng(9)
    M, K, G = 64, 16, 4
    csi = ((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K))) / np.sqrt(2)).astype(np.complex64)
    d = dev(csi)
    mb.Beamform(M, K, G, precision=2).beamform_uplink(d, S=G * 16, sc_group=16)
    W = orc.zf(csi, S=G * 16, sg=16)
    np.testing.assert_allclose(host(d), W, atol=1e-6 * np.abs(W).max())


@pytest.mark.parametrize("Qm", [2, 4, 6, 8])
@pytest.mark.parametrize("K,M,S,sg,n_sym", [(16, 64, 200, 16, 3), (32, 256, 100, 16, 2), (4, 8, 48, 4, 5),
                                            (64, 128, 64, 32, 1), (7, 20, 90, 16, 2)])
def test_equalize_vs_oracle(mb, Qm, K, M, S, sg, n_sym):
    rng = np.random.default_rng(Qm * 1000 + K)
    G = (S + sg - 1) // sg
    W = ((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K))) / np.sqrt(2 * M)).astype(np.complex64)
    y = ((rng.standard_normal((n_sym, M, S)) + 1j * rng.standard_normal((n_sym, M, S))) / np.sqrt(2)).astype(np.complex64)
    cb = (S * Qm * 9) // 10 // Qm * Qm  # drop the tail, as the LDPC sizing does
    zeros, stride = 2 * Qm + 2, cb + 2 * Qm + 6
    seq = orc.scrambler_seq127()
    llr_d = torch.zeros(n_sym, K, stride, dtype=torch.float16, device="cuda")
    n_valid = min(S * Qm, cb)
    hard_d = torch.zeros(n_sym, K, (n_valid + 7) // 8, dtype=torch.uint8, device="cuda")
    x_d = torch.zeros(n_sym, K, S, dtype=torch.complex64, device="cuda")
    scr = mb.Scrambler()
    mb.Equalize.equalize(dev(W), dev(y), llr_d, sg, Qm, cb, zeros, 1, hard=hard_d, scrambler=scr, x=x_d)
    llr_g, hard_g, x_g = host(llr_d), host(hard_d), host(x_d)
    for l in range(n_sym):
        llr_r, x_r, hard_r = orc.equalize(W, y[l], sg, Qm, cb, stride, zeros, seq=seq)
        assert np.abs(x_g[l] - x_r).max() <= 1e-5 * np.abs(x_r).max() + 1e-6
        lg = llr_g[l].astype(np.float32)
        lr = llr_r.astype(np.float32)
        assert np.abs(lg - lr).max() <= 0.05 + 2e-3 * np.abs(lr).max()
        # hard bits: bit-exact where the oracle's LLR is away from zero
        bits_g = np.unpackbits(hard_g[l], axis=1)[:, :n_valid]
        bits_r = np.unpackbits(hard_r, axis=1)[:, :n_valid]
        pos = np.arange(n_valid)
        llr_at = lr[:, zeros + pos]
        sure = np.abs(llr_at) > 0.5
        assert (bits_g[sure] == bits_r[sure]).all()
        assert (bits_g != bits_r).mean() < 1e-3


def test_equalize_gold_scrambler(mb):
    rng = np.random.default_rng(21)
    K, M, S, sg, Qm = 8, 32, 96, 16, 4
    G = S // sg
    W = ((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K))) / np.sqrt(2 * M)).astype(np.complex64)
    y = ((rng.standard_normal((1, M, S)) + 1j * rng.standard_normal((1, M, S))) / np.sqrt(2)).astype(np.complex64)
    cb, zeros = S * Qm, 0
    llr_d = torch.zeros(1, K, cb, dtype=torch.float16, device="cuda")
    hard_d = torch.zeros(1, K, cb // 8, dtype=torch.uint8, device="cuda")
    scr = mb.Scrambler(mode=1, c_init=0x55, num_ue=K, num_bits=cb)
    mb.Equalize.equalize(dev(W), dev(y), llr_d, sg, Qm, cb, zeros, 1, hard=hard_d, scrambler=scr)
    seq = np.stack([orc.gold_seq(0x55 + u, cb) for u in range(K)])
    llr_r, _, hard_r = orc.equalize(W, y[0], sg, Qm, cb, cb, zeros, seq=seq.ravel(), seq_user_stride=cb)
    lr = llr_r.astype(np.float32)
    sure = np.abs(lr) > 0.5
    bg = np.unpackbits(host(hard_d)[0], axis=1)
    br = np.unpackbits(hard_r, axis=1)
    assert (bg[sure] == br[sure]).all()


@pytest.mark.parametrize("M,K,S,sg,N,n_sym", [(64, 16, 1200, 16, 2048, 2), (8, 4, 30, 16, 64, 3), (256, 32, 3276, 16, 4096, 1)])
def test_precode_vs_oracle(mb, M, K, S, sg, N, n_sym):
    rng = np.random.default_rng(M + S)
    G = (S + sg - 1) // sg
    P = ((rng.standard_normal((G, K, M)) + 1j * rng.standard_normal((G, K, M))) * 0.1).astype(np.complex64)
    s = ((rng.standard_normal((n_sym, K, S)) + 1j * rng.standard_normal((n_sym, K, S)))).astype(np.complex64)
    start = (N - S) // 2
    out = torch.full((n_sym, M, N), 3.0 + 0j, dtype=torch.complex64, device="cuda")
    mb.Precode.precode(dev(P), dev(s), out, sg, start)
    got = host(out)
    for l in range(n_sym):
        ref = orc.precode(P, s[l], sg, N, start)
        assert np.abs(got[l] - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("Qm,ps", [(2, 0), (4, 16), (6, 0), (8, 12)])
def test_modulate_vs_oracle(mb, Qm, ps):
    rng = np.random.default_rng(Qm)
    K, S = 5, 1200
    in_bytes = (S * Qm + 7) // 8
    data = rng.integers(0, 256, (K, in_bytes), dtype=np.uint8)
    table = orc.dmrs_table(S, K)
    out = torch.zeros(K, S, dtype=torch.complex64, device="cuda")
    mb.Modulation.modulate(dev(data), out, Qm, ps, dev(table) if ps else None)
    np.testing.assert_array_equal(host(out), orc.modulate(data, S, Qm, ps, table))


def test_dmrs_table_matches_oracle(mb):
    np.testing.assert_allclose(mb.dmrs_table(600, 4).numpy(), orc.dmrs_table(600, 4), atol=2e-6)

"""Tensor-core (tcgen05, BF16 operands, FP32 accumulation) equalizer against
the FP64 oracle.  Tolerance: equalized symbols within 1% of their RMS (BF16
operands carry 8 significant bits); hard bits bit-exact wherever the
oracle's |LLR| > 4 (x at least 0.04 from a decision boundary), LLRs within
1% of the largest |LLR| + 0.5."""
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


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("K,M,S,sg,n_sym,Qm", [
    (32, 256, 3276, 16, 12, 6), (16, 64, 1200, 16, 4, 4), (4, 8, 48, 16, 3, 2),
    (64, 128, 96, 16, 2, 8), (32, 200, 100, 8, 5, 4), (24, 96, 256, 32, 3, 6)])
def test_equalize_tc_vs_oracle(mb, K, M, S, sg, n_sym, Qm):
    rng = np.random.default_rng(K * 7 + M)
    G = (S + sg - 1) // sg
    W = ((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K))) / np.sqrt(2 * M)).astype(np.complex64)
    y = ((rng.standard_normal((n_sym, M, S)) + 1j * rng.standard_normal((n_sym, M, S))) / np.sqrt(2)).astype(np.complex64)
    cb = (S * Qm * 9) // 10 // Qm * Qm
    zeros, stride = 2 * Qm + 2, cb + 2 * Qm + 6
    n_valid = min(S * Qm, cb)
    llr_d = torch.zeros(n_sym, K, stride, dtype=torch.float16, device="cuda")
    hard_d = torch.zeros(n_sym, K, (n_valid + 7) // 8, dtype=torch.uint8, device="cuda")
    x_d = torch.zeros(n_sym, K, S, dtype=torch.complex64, device="cuda")
    scr = mb.Scrambler()
    mb.Equalize.equalize_tc(dev(W), dev(y), llr_d, sg, Qm, cb, zeros, 1, hard=hard_d, scrambler=scr, x=x_d)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    llr_g, hard_g, x_g = llr_d.cpu().numpy(), hard_d.cpu().numpy(), x_d.cpu().numpy()
    seq = orc.scrambler_seq127()
    for l in range(n_sym):
        llr_r, x_r, hard_r = orc.equalize(W, y[l], sg, Qm, cb, stride, zeros, seq=seq)
        rms = np.sqrt(np.mean(np.abs(x_r) ** 2))
        assert np.abs(x_g[l] - x_r).max() <= 0.01 * rms * 4, (l, np.abs(x_g[l] - x_r).max(), rms)
        lr = llr_r.astype(np.float32)
        lg = llr_g[l].astype(np.float32)
        assert np.abs(lg - lr).max() <= 0.5 + 0.01 * np.abs(lr).max()
        bits_g = np.unpackbits(hard_g[l], axis=1)[:, :n_valid]
        bits_r = np.unpackbits(hard_r, axis=1)[:, :n_valid]
        sure = np.abs(lr[:, zeros:zeros + n_valid]) > 4.0
        assert (bits_g[sure] == bits_r[sure]).all()


@pytest.mark.parametrize("Qm", [2, 4, 6, 8])
def test_equalize_tc_demap_bit_exact(mb, Qm):
    # The tensor-core equalizer's LLRs are the reference's FP16 demapper
    # (the oracle's restatement, pinned bit-exact by the golden vectors)
    # applied to its own equalized symbols x, bit for bit; its hard bits are
    # those LLRs' signs (l < 0) descrambled by the LFSR sequence.
    K, M, S, sg, n_sym = 16, 64, 256, 16, 2
    rng = np.random.default_rng(900 + Qm)
    G = S // sg
    W = ((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K))) / np.sqrt(2 * M)).astype(np.complex64)
    y = ((rng.standard_normal((n_sym, M, S)) + 1j * rng.standard_normal((n_sym, M, S))) / np.sqrt(2)).astype(np.complex64)
    cb = (S * Qm * 9) // 10 // Qm * Qm
    zeros, stride = 2 * Qm + 2, cb + 2 * Qm + 6
    n_valid = min(S * Qm, cb)
    llr_d = torch.zeros(n_sym, K, stride, dtype=torch.float16, device="cuda")
    hard_d = torch.zeros(n_sym, K, (n_valid + 7) // 8, dtype=torch.uint8, device="cuda")
    x_d = torch.zeros(n_sym, K, S, dtype=torch.complex64, device="cuda")
    mb.Equalize.equalize_tc(dev(W), dev(y), llr_d, sg, Qm, cb, zeros, 1, hard=hard_d, scrambler=mb.Scrambler(),
                            x=x_d)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    llr_g, hard_g, x_g = llr_d.cpu().numpy(), hard_d.cpu().numpy(), x_d.cpu().numpy()
    seq = orc.scrambler_seq127()
    ns = n_valid // Qm  # whole subcarriers inside the code block
    for l in range(n_sym):
        ref = orc.demod(Qm, x_g[l, :, :ns]).reshape(K, ns * Qm)
        got = llr_g[l][:, zeros:zeros + ns * Qm]
        assert (got.view(np.uint16) == ref.view(np.uint16)).all()
        bits = (ref < 0).astype(np.uint8) ^ seq[np.arange(ns * Qm) % seq.size][None, :]
        assert (np.unpackbits(hard_g[l], axis=1)[:, :ns * Qm] == bits).all()


@pytest.mark.parametrize("M,K,G", [(256, 32, 7), (64, 16, 5), (128, 64, 3), (200, 24, 4), (8, 4, 2),
                                   (256, 64, 2), (384, 64, 3)])
def test_zf_mixed_vs_oracle(mb, M, K, G):
    # split-BF16 Gram on tensor cores + FP32 inverse + 2 Newton-Schulz steps;
    # W via tensor cores: within 1% of max|W| of the FP64 oracle.  384x64
    # does not fit its antenna tiles in shared memory and streams them.
    rng = np.random.default_rng(M + K)
    csi = ((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K))) / np.sqrt(2)).astype(np.complex64)
    d = dev(csi)
    status = torch.full((G,), -1, dtype=torch.int32, device="cuda")
    cond = torch.zeros(G, dtype=torch.float32, device="cuda")
    mb.Beamform(M, K, G, precision=1).beamform_uplink(d, S=G * 16, sc_group=16, status=status, cond=cond)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    W, cond_r, _ = orc.zf(csi, S=G * 16, sg=16, with_cond=True)
    got = d.cpu().numpy()
    assert (status.cpu().numpy() == 0).all()
    c = cond.cpu().numpy()
    # 1-norm estimate vs 2-norm condition: within a factor K either way
    assert ((c >= cond_r / K) & (c <= cond_r * K)).all(), (c, cond_r)
    for g in range(G):
        assert np.abs(got[g] - W[g]).max() <= 0.01 * np.abs(W[g]).max(), g


@pytest.mark.parametrize("M,K,ns_iters", [(256, 32, 2), (256, 32, 0), (128, 16, 2), (200, 24, 1), (256, 64, 2)])
def test_zf_mixed_inverse_accuracy(mb, M, K, ns_iters):
    # Integer CSI (|Re|, |Im| <= 3) is exact in BF16, so the split Gram is the
    # exact Gram in FP32 and the condition estimate ||G||_1 ||X||_1 that the
    # kernel reports measures how exact its inverse X is, where the W check
    # above only sees the BF16 detector.  For 16 < K <= 32 the iterate is
    # held as split BF16 (hi + lo, ~2^-17 of each entry) and the
    # Newton-Schulz products run on the tensor cores with FP32 accumulation
    # (~2^-16): within 2e-5 of the FP64 value (measured up to 6.3e-6 on a
    # B200; the CUDA-core FP32 form of the other K is within 1e-6), far below
    # the BF16 rounding (2^-9) of the detector X feeds.
    G = 8
    rng = np.random.default_rng(1000 + M + K)
    csi = (rng.integers(-3, 4, (G, M, K)) + 1j * rng.integers(-3, 4, (G, M, K))).astype(np.complex64)
    Gm = np.einsum("gbu,gbv->guv", csi.astype(np.complex128), np.conj(csi.astype(np.complex128)))
    n1 = lambda A: np.abs(A).sum(axis=-2).max(axis=-1)  # noqa: E731
    ref = n1(Gm) * n1(np.linalg.inv(Gm))
    d = dev(csi)
    status = torch.full((G,), -1, dtype=torch.int32, device="cuda")
    cond = torch.zeros(G, dtype=torch.float32, device="cuda")
    mb.Beamform(M, K, G, precision=1, ns_iters=ns_iters).beamform_uplink(d, S=G * 16, sc_group=16,
                                                                         status=status, cond=cond)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    assert (status.cpu().numpy() == 0).all()
    rel = np.abs(cond.cpu().numpy().astype(np.float64) - ref) / ref
    assert rel.max() <= (2e-5 if 16 < K <= 32 else 1e-6), rel


def test_zf_mixed_fp64_fallback(mb):
    # group 1 has two nearly collinear users (user 3 = user 2 + 1e-3 * an
    # independent vector): cond ~ 1e7 > 1e4 -> FP64 path
    M, K, G = 64, 8, 3
    rng = np.random.default_rng(77)
    csi = ((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K))) / np.sqrt(2)).astype(np.complex64)
    z = ((rng.standard_normal(M) + 1j * rng.standard_normal(M)) / np.sqrt(2)).astype(np.complex64)
    csi[1, :, 3] = csi[1, :, 2] + 1e-3 * z
    d = dev(csi)
    status = torch.full((G,), -1, dtype=torch.int32, device="cuda")
    cond = torch.zeros(G, dtype=torch.float32, device="cuda")
    mb.Beamform(M, K, G, precision=1).beamform_uplink(d, S=G * 16, sc_group=16, status=status, cond=cond)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    st = status.cpu().numpy()
    assert st[0] == 0 and st[2] == 0 and st[1] == 2, (st, cond.cpu().numpy())
    W = orc.zf(csi, S=G * 16, sg=16)
    got = d.cpu().numpy()
    assert np.abs(got[1] - W[1]).max() <= 1e-4 * np.abs(W[1]).max()


CASES = [
    dict(M=64, K=16, N=2048, S=1200, sg=16, Qm=4, U=5, snr_db=20.0, seed=11),
    dict(M=128, K=32, N=1024, S=600, sg=16, Qm=6, U=4, snr_db=28.0, seed=12, channel="tdl", rho=0.5,
         n_taps=4, tap_decay=1.0),
    dict(M=32, K=8, N=256, S=200, sg=8, Qm=2, U=3, snr_db=12.0, seed=13, iq_dtype="int16"),
    # antenna tiles streamed through shared memory in the mixed ZF
    dict(M=384, K=64, N=512, S=300, sg=16, Qm=4, U=3, snr_db=30.0, seed=14),
    # N = 4096: the uplink FFT on the tensor cores
    dict(M=64, K=16, N=4096, S=3276, sg=16, Qm=6, U=3, snr_db=25.0, seed=17, iq_dtype="int16"),
    dict(M=32, K=8, N=4096, S=3276, sg=16, Qm=8, U=2, snr_db=32.0, seed=18),
    # the bench's slot shape: the combined pilot + uplink FFT launch with
    # about 13 units per CTA
    dict(M=256, K=32, N=4096, S=3276, sg=16, Qm=6, U=12, snr_db=25.0, seed=19, channel="tdl", rho=0.5,
         n_taps=8, tap_decay=2.0),
    # the same shape on int8 samples, the reference's production format
    dict(M=256, K=32, N=4096, S=3276, sg=16, Qm=6, U=12, snr_db=25.0, seed=20, channel="tdl", rho=0.5,
         n_taps=8, tap_decay=2.0, iq_dtype="int8"),
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c['M']}x{c['K']}Q{c['Qm']}N{c['N']}{c.get('iq_dtype', '')}"
                                             for c in CASES])
def test_slot_uplink_mixed_vs_oracle(mb, case):
    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(**case)
    d = datagen.make_slot(cfg)
    run = slot.UplinkSlot(cfg, precision="mixed", sym_batch=12 if cfg.U == 12 else 4, use_graph=True)
    iq = torch.from_numpy(d["iq"]).cuda()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        run(iq, stream=s)
        llr, hard = run(iq, stream=s)
    s.synchronize()
    assert mb.ops.device_error() == 0
    assert (run.status.cpu().numpy() == 0).all()
    llr, hard = llr.cpu().numpy(), hard.cpu().numpy()
    cb, zeros, stride = cfg.ldpc()
    n_valid = min(cb, cfg.S * cfg.Qm)
    ps = orc.pilot_sign(cfg.S)
    csi = np.zeros((cfg.G, cfg.M, cfg.K), np.complex64)
    for p in range(cfg.P):
        orc.pilot_fft(d["iq"][p], cfg.N, cfg.S, cfg.start, cfg.K, cfg.sg, p * cfg.sg, ps, csi)
    W = orc.zf(csi, S=cfg.S, sg=cfg.sg)
    for l in range(cfg.U):
        y = orc.uplink_fft(d["iq"][cfg.P + l], cfg.N, cfg.S, cfg.start)
        llr_r, _, hard_r = orc.equalize(W, y, cfg.sg, cfg.Qm, cb, stride, zeros, seq=d["seq"][0])
        lr = llr_r.astype(np.float32)
        sure = np.abs(lr[:, zeros:zeros + n_valid]) > 4.0
        bg = np.unpackbits(hard[l], axis=1)[:, :n_valid]
        br = np.unpackbits(hard_r, axis=1)[:, :n_valid]
        assert (bg[sure] == br[sure]).all()
        assert np.abs(llr[l].astype(np.float32) - lr).max() <= 1.0 + 0.02 * np.abs(lr).max()


def test_slot_fuses_zf_and_equalize(mb):
    # with every uplink symbol in one batch (and the FFT of pilots and
    # symbols in one launch) the ZF kernel equalizes itself: no equalize
    # launch of its own in the stage record; split batches keep two kernels
    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(M=64, K=16, N=4096, S=3276, sg=16, Qm=6, U=3, snr_db=25.0, seed=31)
    iq = torch.from_numpy(datagen.make_slot(cfg)["iq"]).cuda()
    for sym_batch, n_eq in ((3, 0), (2, 2)):
        run = slot.UplinkSlot(cfg, precision="mixed", sym_batch=sym_batch)
        run.timing(1)
        run(iq)
        st = run.stage_ms()
        assert st["n_eq"] == n_eq, (sym_batch, st)
    assert mb.ops.device_error() == 0


def test_fused_slot_fp64_groups_vs_oracle(mb):
    # a condition threshold below 1 sends every group down the FP64 path,
    # whose detector image the fused equalize reads from shared memory
    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(M=64, K=16, N=4096, S=3276, sg=16, Qm=4, U=3, snr_db=25.0, seed=32)
    d = datagen.make_slot(cfg)
    run = slot.UplinkSlot(cfg, precision="mixed", sym_batch=cfg.U, cond_threshold=0.5)
    llr, hard = run(torch.from_numpy(d["iq"]).cuda())
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    assert (run.status.cpu().numpy() == 2).all()
    llr, hard = llr.cpu().numpy(), hard.cpu().numpy()
    cb, zeros, stride = cfg.ldpc()
    n_valid = min(cb, cfg.S * cfg.Qm)
    ps = orc.pilot_sign(cfg.S)
    csi = np.zeros((cfg.G, cfg.M, cfg.K), np.complex64)
    for p in range(cfg.P):
        orc.pilot_fft(d["iq"][p], cfg.N, cfg.S, cfg.start, cfg.K, cfg.sg, p * cfg.sg, ps, csi)
    W = orc.zf(csi, S=cfg.S, sg=cfg.sg)
    for l in range(cfg.U):
        y = orc.uplink_fft(d["iq"][cfg.P + l], cfg.N, cfg.S, cfg.start)
        llr_r, _, hard_r = orc.equalize(W, y, cfg.sg, cfg.Qm, cb, stride, zeros, seq=d["seq"][0])
        lr = llr_r.astype(np.float32)
        sure = np.abs(lr[:, zeros:zeros + n_valid]) > 4.0
        bg = np.unpackbits(hard[l], axis=1)[:, :n_valid]
        br = np.unpackbits(hard_r, axis=1)[:, :n_valid]
        assert (bg[sure] == br[sure]).all()
        assert np.abs(llr[l].astype(np.float32) - lr).max() <= 1.0 + 0.02 * np.abs(lr).max()


def test_zf_mixed_forced_fp64_path(mb):
    # a condition threshold below 1 sends every group down the FP64 path
    M, K, G = 96, 16, 4
    rng = np.random.default_rng(5)
    csi = ((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K))) / np.sqrt(2)).astype(np.complex64)
    d = dev(csi)
    status = torch.full((G,), -1, dtype=torch.int32, device="cuda")
    mb.Beamform(M, K, G, precision=1, cond_threshold=0.5).beamform_uplink(d, S=G * 16, sc_group=16,
                                                                         status=status)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    assert (status.cpu().numpy() == 2).all(), status.cpu().numpy()
    W = orc.zf(csi, S=G * 16, sg=16)
    np.testing.assert_allclose(d.cpu().numpy(), W, atol=2e-6 * np.abs(W).max())


@pytest.mark.parametrize("cond_threshold", [1e4, 0.5], ids=["ns", "fp64"])
def test_slot_mixed_precoder(mb, cond_threshold):
    # the mixed slot with a downlink: W from the fused ZF kernel (its FP32
    # copy) and P = W^T / max|W| per group from the kernel's own max |W|
    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(M=128, K=32, N=1024, S=600, sg=16, Qm=4, U=2, snr_db=25.0, seed=16)
    d = datagen.make_slot(cfg)
    run = slot.UplinkSlot(cfg, precision="mixed", sym_batch=2, use_graph=True, D=2,
                          cond_threshold=cond_threshold)
    iq = torch.from_numpy(d["iq"]).cuda()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        run(iq, stream=s)
    s.synchronize()
    assert mb.ops.device_error() == 0
    assert (run.status.cpu().numpy() == (0 if cond_threshold > 1 else 2)).all()
    W, P = run.buffers()
    W = W.cpu().numpy()
    P = P.cpu().numpy()
    ps = orc.pilot_sign(cfg.S)
    csi = np.zeros((cfg.G, cfg.M, cfg.K), np.complex64)
    for p in range(cfg.P):
        orc.pilot_fft(d["iq"][p], cfg.N, cfg.S, cfg.start, cfg.K, cfg.sg, p * cfg.sg, ps, csi)
    Wr = orc.zf(csi, S=cfg.S, sg=cfg.sg)
    assert np.abs(W - Wr).max() <= 0.01 * np.abs(Wr).max()
    mx = np.abs(W).max(axis=(1, 2))
    Pr = np.transpose(W, (0, 2, 1)) / mx[:, None, None]
    np.testing.assert_allclose(P, Pr, rtol=0, atol=1e-6)


@pytest.mark.parametrize("iq_dtype", ["int8", "int16"])
def test_mixed_hard_bits_match_plain_path(mb, iq_dtype):
    """The headline accuracy target: on the bench's slot shape (256x32,
    N = 4096, 64-QAM, 25 dB, 8-tap rho = 0.5) the mixed path's descrambled
    hard bits equal the plain FP32 path's wherever the plain path's
    |LLR| > 4, and its uncoded BER is no worse than the plain path's by more
    than the bits that lie under that tolerance."""
    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(M=256, K=32, N=4096, S=3276, sg=16, Qm=6, U=12, snr_db=25.0, channel="tdl",
                             rho=0.5, n_taps=8, tap_decay=2.0, iq_dtype=iq_dtype, seed=2024)
    d = datagen.make_slot(cfg)
    cb, zeros, _ = cfg.ldpc()
    n_valid = min(cb, cfg.S * cfg.Qm)
    iq = torch.from_numpy(d["iq"]).cuda()
    res = {}
    for prec in ("fp32", "mixed"):
        run = slot.UplinkSlot(cfg, precision=prec, sym_batch=12)
        llr, hard = run(iq)
        torch.cuda.synchronize()
        res[prec] = (llr.cpu().numpy().astype(np.float32)[..., zeros:zeros + n_valid],
                     np.unpackbits(hard.cpu().numpy(), axis=-1)[..., :n_valid])
    assert mb.ops.device_error() == 0
    lp, bp = res["fp32"]
    _, bm = res["mixed"]
    sure = np.abs(lp) > 4.0
    assert sure.mean() > 0.9
    assert int((bm != bp)[sure].sum()) == 0
    sent = d["bits"][..., :n_valid]
    ber_p, ber_m = np.mean(bp != sent), np.mean(bm != sent)
    assert ber_m <= ber_p + np.mean(~sure)

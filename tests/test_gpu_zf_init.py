"""The learned initial iterate of the mixed ZF on the GPU, against the FP64
restatement (oracle/zf_init.py) and the ZF oracle.

The network is trained here by the library's own forward, backward and Adam
kernels on the quadratic residual targets of mb_zf_init_targets; the mixed
ZF then starts Newton-Schulz from its polynomial and must give the same
detector as the exact path (1% of max |W|, the mixed tests' tolerance),
accept the learned start (status 3) on nearly every group of the
256 x 32 correlated channel, agree with the restatement on which groups it
accepts, and fall back to the exact inverse where the start is poor (the
untrained network's Neumann polynomial)."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from oracle import zf_init as zi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from megastation_b200 import learned
    data = learned.zf_init_training_set([(256, 32), (128, 16)], n_real=160, seed=11)
    net = learned.make_zf_init_net(width=64, seed=3)
    learned.train(net, data, steps=1500, batch=4096, lr=2e-3, seed=5)
    return net, data


def _held_out(M, K, n, seed, rho=(0.5, 0.5)):
    from megastation_b200 import learned
    return learned.group_csi(M, K, n, seed, rho=rho, tap_decay=(2.0, 2.0), snr_db=(25.0, 25.0))


@pytest.mark.parametrize("M,K", [(64, 16), (256, 32), (128, 64)])
def test_targets_match_restatement(M, K):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from megastation_b200 import learned
    csi = _held_out(M, K, 1, 21)[0][:12].contiguous()
    F, A, b = learned.zf_init_targets(csi)
    F, A, b = F.cpu().numpy(), A.cpu().numpy(), b.cpu().numpy()
    c = csi.cpu().numpy()
    for g in range(c.shape[0]):
        f_r, A_r, b_r = zi.features_targets(zi.gram(c[g]), M)
        np.testing.assert_allclose(F[g], f_r, rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(A[g], A_r, rtol=1e-5)
        np.testing.assert_allclose(b[g], b_r, rtol=1e-5)


def test_training_beats_neumann(trained):
    from megastation_b200 import learned
    net, data = trained
    r_learned, r_neumann = learned.poly_residual(net, data)
    assert r_learned < 0.05 * r_neumann and r_learned < 5e-3, (r_learned, r_neumann)


def test_mixed_zf_from_learned_iterate(trained):
    import megastation_b200 as mb
    from megastation_b200 import learned
    net, _ = trained
    M, K = 256, 32
    csi = _held_out(M, K, 1, 99)[0].contiguous()
    G = csi.shape[0]
    c = csi.cpu().numpy()
    W_r = orc.zf(c, S=G * 16, sg=16)
    d = csi.clone()
    status = torch.full((G,), -1, dtype=torch.int32, device="cuda")
    bf = mb.Beamform(M, K, G, precision=1, init_net=net)
    bf.beamform_uplink(d, S=G * 16, sc_group=16, status=status)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    st = status.cpu().numpy()
    assert np.isin(st, (0, 3)).all(), st
    assert (st == 3).mean() >= 0.9, (st == 3).mean()
    W = d.cpu().numpy()
    assert np.abs(W - W_r).max() <= 0.01 * np.abs(W_r).max()
    # the kernel's accept decisions against the restatement's, with the
    # coefficients the network gives for the GPU's own features
    F, _, _ = learned.zf_init_targets(csi)
    alpha = net.forward(F).cpu().numpy().astype(np.float64)
    agree = np.mean([zi.poly_ns(zi.gram(c[g]), alpha[g])[1] == (st[g] == 3) for g in range(G)])
    assert agree >= 0.97, agree


def test_poor_start_falls_back_to_exact_inverse():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import megastation_b200 as mb
    from megastation_b200 import learned
    net = learned.make_zf_init_net(width=64, seed=4)  # untrained: the Neumann polynomial
    M, K = 256, 32
    csi = _held_out(M, K, 1, 7)[0][:40].contiguous()
    G = csi.shape[0]
    W_r = orc.zf(csi.cpu().numpy(), S=G * 16, sg=16)
    d = csi.clone()
    status = torch.full((G,), -1, dtype=torch.int32, device="cuda")
    mb.Beamform(M, K, G, precision=1, init_net=net).beamform_uplink(d, S=G * 16, sc_group=16, status=status)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    assert (status.cpu().numpy() == 0).all()
    assert np.abs(d.cpu().numpy() - W_r).max() <= 0.01 * np.abs(W_r).max()


@pytest.mark.parametrize("iq_dtype", ["int8", "int16"])
def test_slot_with_learned_iterate_vs_oracle(trained, iq_dtype):
    """The bench's slot (256 x 32, N = 4096, 64-QAM, 25 dB, 8-tap rho = 0.5)
    with the learned initial iterate: LLRs and hard bits against the FP64
    oracle with the mixed path's tolerance, and the same hard bits as the
    plain FP32 slot wherever its |LLR| > 4."""
    import megastation_b200 as mb
    from megastation_b200 import datagen, slot

    from slot_oracle import check_uplink, oracle_uplink
    net, _ = trained
    cfg = datagen.CellConfig(M=256, K=32, N=4096, S=3276, sg=16, Qm=6, U=12, snr_db=25.0, channel="tdl", rho=0.5,
                             n_taps=8, tap_decay=2.0, iq_dtype=iq_dtype, seed=31)
    d = datagen.make_slot(cfg)
    iq = torch.from_numpy(d["iq"]).cuda()
    run = slot.UplinkSlot(cfg, precision="mixed", sym_batch=12, use_graph=True)
    run.set_zf_init(net)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        run(iq, stream=s)
        llr, hard = run(iq, stream=s)
    s.synchronize()
    assert mb.ops.device_error() == 0
    st = run.status.cpu().numpy()
    assert np.isin(st, (0, 3)).all() and (st == 3).mean() >= 0.9, st
    _, ref = oracle_uplink(cfg, d)
    llr, hard = llr.cpu().numpy(), hard.cpu().numpy()
    check_uplink(cfg, ref, llr, hard, "mixed", "learned")
    plain = slot.UplinkSlot(cfg, precision="fp32", sym_batch=12)
    lp, hp = plain(iq)
    torch.cuda.synchronize()
    cb, zeros, _ = cfg.ldpc()
    n_valid = min(cb, cfg.S * cfg.Qm)
    sure = np.abs(lp.cpu().numpy().astype(np.float32)[..., zeros:zeros + n_valid]) > 4.0
    bp = np.unpackbits(hp.cpu().numpy(), axis=-1)[..., :n_valid]
    bm = np.unpackbits(hard, axis=-1)[..., :n_valid]
    assert int((bm != bp)[sure].sum()) == 0

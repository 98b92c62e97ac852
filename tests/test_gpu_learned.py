"""The learned ZF initialiser on the GPU against its FP64 restatement
(oracle/mlp.py) and the FP64 ZF oracle, and the ablation: what the trained
network gains over the same method without it."""
import numpy as np
import pytest
import torch

from oracle import mlp as om
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mb():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import megastation_b200 as mb
    return mb


def _rand_net(learned, n_in, width, n_out, seed):
    net = learned.MLP(n_in, width, n_out, max_batch=512, seed=seed)
    rng = np.random.default_rng(seed)
    p = (rng.standard_normal(net.num_params()) * 0.3).astype(np.float32)
    net.set_params(p)
    return net, p


def test_mlp_forward_matches_oracle(mb):
    from megastation_b200 import learned
    n_in, width, n_out, B = 22, 256, 4, 300
    net, p = _rand_net(learned, n_in, width, n_out, 1)
    x = np.random.default_rng(2).standard_normal((B, n_in)).astype(np.float32)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    yr, _ = om.mlp_forward(p, x, n_in, width, n_out)
    # BF16 weights and activations on both sides, FP32 accumulation over 256
    # terms here; a hidden activation whose FP32 and FP64 pre-activations
    # fall on either side of a BF16 rounding boundary moves by one BF16 ulp
    # (2^-8), which bounds the band
    assert np.abs(y - yr).max() <= 1e-3 * np.abs(yr).max()


def test_mlp_gradients_match_oracle(mb):
    from megastation_b200 import learned
    n_in, width, n_out, B = 22, 256, 4, 384
    net, p = _rand_net(learned, n_in, width, n_out, 3)
    rng = np.random.default_rng(4)
    x = rng.standard_normal((B, n_in)).astype(np.float32)
    Mx = rng.standard_normal((B, n_out, n_out))
    A = (np.einsum("bij,bkj->bik", Mx, Mx) / n_out).astype(np.float32)
    b = rng.standard_normal((B, n_out)).astype(np.float32)
    c = rng.standard_normal(B).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    loss = net.loss_grad(dev(x), dev(A), dev(b), dev(c))
    g = net.grads()
    lr, gr = om.mlp_loss_grad(p, x, A, b, c, n_in, width, n_out)
    assert abs(float(loss.item()) - lr) <= 1e-4 * max(1.0, abs(lr))
    # per parameter block, relative to the block's largest gradient
    sizes = [n_in * width, width, width * width, width, width * n_out, n_out]
    o = 0
    for s in sizes:
        blk, ref = g[o:o + s], gr[o:o + s]
        # the backward products on the tensor cores take BF16 activations and
        # upstream gradients, rounded at the same places in the restatement;
        # the band covers the one-ulp rounding flips of the forward pass
        assert np.abs(blk - ref).max() <= 1e-3 * np.abs(ref).max() + 1e-7, (o, s)
        o += s


def test_mlp_adam_reduces_loss(mb):
    from megastation_b200 import learned
    n_in, width, n_out, B = 8, 64, 4, 256
    net = learned.MLP(n_in, width, n_out, max_batch=B, seed=5)
    rng = np.random.default_rng(6)
    x = torch.from_numpy(rng.standard_normal((B, n_in)).astype(np.float32)).cuda()
    A = torch.eye(n_out).repeat(B, 1, 1).cuda()
    b = torch.from_numpy(rng.standard_normal((B, n_out)).astype(np.float32) * 0.1).cuda()
    first = float(net.loss_grad(x, A, b).item())
    for _ in range(200):
        net.loss_grad(x, A, b)
        net.adam_step(3e-3)
    last = float(net.loss_grad(x, A, b).item())
    assert last < 0.2 * first


def _small_cell():
    from megastation_b200 import datagen
    return datagen.CellConfig(M=32, K=8, N=256, S=96, sg=16, Qm=4, U=2, snr_db=25.0, channel="tdl_ds",
                              delay_spread_ns=200.0, seed=7)


def test_lzf_exact_matches_zf_oracle(mb):
    from megastation_b200 import learned
    cfg = _small_cell()
    csi = learned.pilot_csi(cfg, 1, seed=8)[0]
    lz = learned.LearnedZF(cfg.M, cfg.K, cfg.S, cfg.sg)
    W = lz.run(csi, init=learned.EXACT, ns_iters=0).cpu().numpy()
    c = om.interp_csi(csi.cpu().numpy(), cfg.S, cfg.sg)
    Wr = orc.zf(c.astype(np.complex64), S=cfg.S, sg=1)
    assert np.abs(W - Wr).max() <= 2e-3 * np.abs(Wr).max()
    # Newton-Schulz from the exact inverse stays there; the residual is small
    lz.run(csi, init=learned.EXACT, ns_iters=2)
    assert float(lz.residual().max()) < 1e-3


def test_lzf_features_and_targets_match_oracle(mb):
    from megastation_b200 import learned
    cfg = _small_cell()
    csi = learned.pilot_csi(cfg, 1, seed=9)[0]
    lz = learned.LearnedZF(cfg.M, cfg.K, cfg.S, cfg.sg)
    F = lz.features(csi).cpu().numpy()
    A, b = lz.targets(csi)
    c = om.interp_csi(csi.cpu().numpy(), cfg.S, cfg.sg)
    Gs = om.gram(c)
    Fr = om.features(Gs, cfg.S, cfg.sg)
    Ar, br = om.targets(Gs, cfg.S, cfg.sg)
    assert np.abs(F - Fr).max() <= 1e-4 * max(1.0, np.abs(Fr).max())
    assert np.abs(A.cpu().numpy() - Ar).max() <= 1e-4 * np.abs(Ar).max()
    assert np.abs(b.cpu().numpy() - br).max() <= 1e-4 * np.abs(br).max()


@pytest.fixture(scope="module")
def trained(mb):
    """A network trained on the GPU for the 128x16, N = 2048, S = 1200 cell
    with delay spreads of 50-300 ns (a short run: 48 realisations)."""
    from megastation_b200 import datagen, learned
    cfg = datagen.CellConfig(M=128, K=16, N=2048, S=1200, sg=16, Qm=4, U=13, snr_db=25.0, channel="tdl_ds",
                             seed=10)
    lz = learned.LearnedZF(cfg.M, cfg.K, cfg.S, cfg.sg)
    train = learned.training_set(lz, learned.pilot_csi(cfg, 48, seed=11))
    held = learned.training_set(lz, learned.pilot_csi(cfg, 8, seed=12))
    net = learned.make_mlp(cfg.sg, seed=13)
    before = learned.blend_loss(net, held)
    hist = learned.train(net, train, steps=600, batch=4096, lr=1e-3, seed=14, log_every=100)
    after = learned.blend_loss(net, held)
    return cfg, lz, net, before, after, hist


def test_training_reduces_blend_error(trained):
    cfg, lz, net, before, after, hist = trained
    # the untrained network is exactly the coarse blend
    assert abs(before[0] - before[1]) <= 1e-3 * before[1]
    # ablation on held-out channels: the learned blend is much closer to the
    # exact per-subcarrier inverse than the group's own inverse
    assert after[0] < 0.5 * after[1], (after, hist)


def test_learned_init_lowers_newton_schulz_residual(trained):
    from megastation_b200 import learned
    cfg, lz, net, _, _, _ = trained
    csi = learned.pilot_csi(cfg, 1, seed=15)[0]
    res = {}
    for name, init in (("coarse", learned.COARSE), ("learned", learned.LEARNED)):
        for it in (0, 1, 2):
            lz.run(csi, init=init, ns_iters=it, mlp=net)
            res[(name, it)] = float(lz.residual().median())
    for it in (0, 1, 2):
        assert res[("learned", it)] < res[("coarse", it)], res


def test_learned_slot_evm(trained):
    """End to end on one slot of the tdl_ds channel (250 ns): exact
    per-subcarrier ZF beats the per-group ZF of the plain path; the learned
    iterate reaches exact ZF's EVM with 2 Newton-Schulz steps and, with none,
    is clearly better than the group's own inverse."""
    import megastation_b200 as mb
    from megastation_b200 import datagen, learned
    cfg0, lz, net, _, _, _ = trained
    cfg = datagen.CellConfig(**{**cfg0.__dict__, "delay_spread_ns": 250.0, "seed": 16})
    d = datagen.make_slot(cfg)
    iq = torch.from_numpy(d["iq"]).cuda()
    csi = torch.zeros(cfg.G, cfg.M, cfg.K, dtype=torch.complex64, device="cuda")
    mb.PilotFFT(cfg.start, cfg.N, cfg.S, cfg.M, cfg.K, cfg.sg)(iq[:cfg.P], csi)
    y = torch.zeros(cfg.U, cfg.M, cfg.S, dtype=torch.complex64, device="cuda")
    mb.UplinkFFT(cfg.start, cfg.N, cfg.S, cfg.M)(iq[cfg.P:], y)
    cb, zeros, stride = cfg.ldpc()

    def evm(W, sg):
        llr = torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda")
        x = torch.zeros(cfg.U, cfg.K, cfg.S, dtype=torch.complex64, device="cuda")
        mb.Equalize.equalize(W, y, llr, sg, cfg.Qm, cb, zeros, 1, x=x)
        xs = x.cpu().numpy()
        return 10 * np.log10(np.mean(np.abs(xs - d["x"]) ** 2) / np.mean(np.abs(d["x"]) ** 2))

    Wg = csi.clone()
    mb.Beamform(cfg.M, cfg.K, cfg.G).beamform_uplink(Wg, S=cfg.S, sc_group=cfg.sg)
    e_group = evm(Wg, cfg.sg)
    e_exact = evm(lz.run(csi, init=learned.EXACT, ns_iters=0), 1)
    e = {(name, it): evm(lz.run(csi, init=init, ns_iters=it, mlp=net), 1)
         for name, init in (("learned", learned.LEARNED), ("coarse", learned.COARSE)) for it in (0, 1, 2)}
    print("EVM dB: group", e_group, "exact", e_exact, e)
    assert e_exact < e_group - 1.0, (e_exact, e_group)
    # with 2 Newton-Schulz steps the learned iterate reaches exact ZF
    assert e[("learned", 2)] <= e_exact + 0.1, (e, e_exact)
    # without refinement the learned iterate is the better detector; one
    # Newton-Schulz step brings either start to within a tenth of a dB
    assert e[("learned", 0)] < e[("coarse", 0)] - 0.5, e
    assert abs(e[("learned", 1)] - e[("coarse", 1)]) <= 0.1, e


def test_lzf_exact_at_headline_shape(mb):
    """The per-subcarrier path at 256 antennas x 32 users (its CSI staged in
    shared memory beyond the default 48 KB): exact per-subcarrier ZF against
    the ZF oracle on the interpolated CSI, for a sample of subcarriers."""
    from megastation_b200 import datagen, learned
    cfg = datagen.CellConfig(M=256, K=32, N=4096, S=3276, sg=16, Qm=6, U=2, snr_db=25.0, channel="tdl_ds",
                             delay_spread_ns=150.0, seed=21)
    csi = learned.pilot_csi(cfg, 1, seed=22)[0]
    lz = learned.LearnedZF(cfg.M, cfg.K, cfg.S, cfg.sg)
    W = lz.run(csi, init=learned.EXACT, ns_iters=0).cpu().numpy()
    c = om.interp_csi(csi.cpu().numpy(), cfg.S, cfg.sg)
    pick = np.arange(0, cfg.S, 97)
    Wr = orc.zf(c[pick].astype(np.complex64), S=len(pick), sg=1)
    assert np.abs(W[pick] - Wr).max() <= 2e-3 * np.abs(Wr).max()


def test_lzf_far_start_takes_exact_inverse(mb):
    """On a channel that changes fast across the band (256 x 32, 300 ns), the
    group-centre start of many subcarriers is too far off for Newton-Schulz
    (||I - G X0||_F >= 1): those subcarriers are flagged 2 and take the exact
    inverse, so the iteration never diverges; the others converge."""
    from megastation_b200 import datagen, learned
    cfg = datagen.CellConfig(M=256, K=32, N=4096, S=3276, sg=16, Qm=6, U=2, snr_db=25.0, channel="tdl_ds",
                             delay_spread_ns=300.0, seed=23)
    csi = learned.pilot_csi(cfg, 1, seed=24, delay_spread_ns=(300.0, 300.0))[0]
    lz = learned.LearnedZF(cfg.M, cfg.K, cfg.S, cfg.sg)
    W_ex = lz.run(csi, init=learned.EXACT, ns_iters=0).clone()
    W = lz.run(csi, init=learned.COARSE, ns_iters=2)
    fl = lz.flags().cpu().numpy()
    res = lz.residual().cpu().numpy()
    torch.cuda.synchronize()
    assert np.isin(fl, (0, 2)).all()
    assert (fl == 2).any()
    assert np.isfinite(res).all() and res.max() < 1.0
    far = np.nonzero(fl == 2)[0]
    Wn, We = W.cpu().numpy(), W_ex.cpu().numpy()
    assert np.abs(Wn[far] - We[far]).max() <= 1e-5 * np.abs(We).max()

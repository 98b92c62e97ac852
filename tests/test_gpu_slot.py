"""End-to-end uplink slot on the GPU (mb_slot_uplink through the C ABI) against
the CPU oracle on seeded synthetic slots: hard bits bit-exact where the
oracle's |LLR| > 0.5, LLRs within FP16 tolerance, and the decoded bits
against what was transmitted."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from megastation_b200 import datagen, slot
    return datagen, slot


def oracle_slot(cfg, d):
    cb, zeros, stride = cfg.ldpc()
    ps = orc.pilot_sign(cfg.S)
    csi = np.zeros((cfg.G, cfg.M, cfg.K), np.complex64)
    for p in range(cfg.P):
        orc.pilot_fft(d["iq"][p], cfg.N, cfg.S, cfg.start, cfg.K, cfg.sg, p * cfg.sg, ps, csi)
    W = orc.zf(csi, S=cfg.S, sg=cfg.sg)
    out = []
    seq = d["seq"] if cfg.scrambler == "gold" else d["seq"][0]
    stride_u = d["seq"].shape[1] if cfg.scrambler == "gold" else 0
    for l in range(cfg.U):
        y = orc.uplink_fft(d["iq"][cfg.P + l], cfg.N, cfg.S, cfg.start)
        out.append(orc.equalize(W, y, cfg.sg, cfg.Qm, cb, stride, zeros, seq=seq.ravel(),
                                seq_user_stride=stride_u))
    return W, out


CASES = [
    dict(M=16, K=8, N=256, S=192, sg=16, Qm=4, U=3, snr_db=25.0, seed=1),
    dict(M=32, K=20, N=512, S=300, sg=16, Qm=6, U=5, snr_db=28.0, seed=2, iq_dtype="int16"),
    dict(M=64, K=16, N=2048, S=1200, sg=16, Qm=4, U=2, snr_db=20.0, seed=3),
    dict(M=24, K=4, N=128, S=100, sg=8, Qm=2, U=4, snr_db=15.0, seed=4, iq_dtype="int8",
         scrambler="gold"),
    dict(M=48, K=32, N=1024, S=600, sg=16, Qm=8, U=2, snr_db=35.0, seed=5, channel="tdl", rho=0.5,
         n_taps=4, tap_decay=1.0),
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c['M']}x{c['K']}N{c['N']}Q{c['Qm']}" for c in CASES])
@pytest.mark.parametrize("use_graph", [False, True])
def test_slot_uplink_vs_oracle(mods, case, use_graph):
    datagen, slot = mods
    cfg = datagen.CellConfig(**case)
    d = datagen.make_slot(cfg)
    run = slot.UplinkSlot(cfg, precision="fp32", sym_batch=2, use_graph=use_graph)
    iq = torch.from_numpy(d["iq"]).cuda()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        llr, hard = run(iq, stream=stream)
        llr, hard = run(iq, stream=stream)  # second call replays the graph
    stream.synchronize()
    llr, hard = llr.cpu().numpy(), hard.cpu().numpy()
    assert (run.status.cpu().numpy() == 0).all()
    W_r, ref = oracle_slot(cfg, d)
    cb, zeros, _ = cfg.ldpc()
    n_valid = min(cb, cfg.S * cfg.Qm)
    for l in range(cfg.U):
        llr_r, x_r, hard_r = ref[l]
        lr = llr_r.astype(np.float32)
        lg = llr[l].astype(np.float32)
        assert np.abs(lg - lr).max() <= 0.25 + 5e-3 * np.abs(lr).max()
        sure = np.abs(lr[:, zeros:zeros + n_valid]) > 0.5
        bg = np.unpackbits(hard[l], axis=1)[:, :n_valid]
        br = np.unpackbits(hard_r, axis=1)[:, :n_valid]
        assert (bg[sure] == br[sure]).all()
        # decoded (descrambled) hard bits against the transmitted bits
        if cfg.channel == "iid_group":
            assert (bg != d["bits"][l][:, :n_valid]).mean() < 1e-3

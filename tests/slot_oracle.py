"""Oracle restatement of whole slots for the GPU parity tests (test
infrastructure): the stage order of BandProcess::process
(baseband/process.cc:161-214) run through the FP64 CPU oracle, and the
comparisons the slot-level tests share."""
import numpy as np

from oracle import oracle as orc


def oracle_detector(cfg, iq):
    """Pilot FFT + LS estimate of every pilot symbol, then the per-group ZF
    (beamform.cu:74-122) with the short-last-group fill: W [G][M][K]."""
    ps = orc.pilot_sign(cfg.S)
    csi = np.zeros((cfg.G, cfg.M, cfg.K), np.complex64)
    for p in range(cfg.P):
        orc.pilot_fft(iq[p], cfg.N, cfg.S, cfg.start, cfg.K, cfg.sg, p * cfg.sg, ps, csi)
    return orc.zf(csi, S=cfg.S, sg=cfg.sg)


def oracle_uplink(cfg, d):
    """(W, [(llr, x, hard) per uplink symbol]) of one slot."""
    cb, zeros, stride = cfg.ldpc()
    W = oracle_detector(cfg, d["iq"])
    seq = d["seq"] if cfg.scrambler == "gold" else d["seq"][0]
    stride_u = d["seq"].shape[1] if cfg.scrambler == "gold" else 0
    out = []
    for l in range(cfg.U):
        y = orc.uplink_fft(d["iq"][cfg.P + l], cfg.N, cfg.S, cfg.start)
        out.append(orc.equalize(W, y, cfg.sg, cfg.Qm, cb, stride, zeros, seq=seq.ravel(),
                                seq_user_stride=stride_u))
    return W, out


# Tolerances of a slot against the oracle, per path: hard bits must agree
# wherever the oracle's |LLR| exceeds `sure`, LLRs within abs + rel * max|LLR|.
TOL = {"fp32": dict(sure=0.5, abs=0.25, rel=5e-3), "mixed": dict(sure=4.0, abs=1.0, rel=0.02)}


def tolerance(cfg, precision):
    """TOL of the path, widened for the mixed path on cells with fewer than
    four antennas per user: the BF16 rounding of W and y in x = W y is
    amplified by the cancellation in that sum, which grows with the
    channel's condition (M / K = 1 or 2 in the batched-cells workload)."""
    t = dict(TOL[precision])
    if precision == "mixed" and cfg.M < 4 * cfg.K:
        t.update(sure=10.0, rel=0.06)
    return t


def check_uplink(cfg, ref, llr, hard, precision, what="", sent=None):
    """llr [U][K][stride] (float16 numpy), hard [U][K][hrow] against the
    oracle's per-symbol outputs `ref`.  Mixed-path cells with fewer than two
    antennas per user (down to as many users as antennas) are judged on
    their uncoded BER against the transmitted bits `sent` instead: there the
    ZF output is dominated by amplified noise, and the BF16 rounding of an
    ill-conditioned detector moves LLRs by more than any fixed band."""
    t = tolerance(cfg, precision)
    cb, zeros, _ = cfg.ldpc()
    n_valid = min(cb, cfg.S * cfg.Qm)
    if precision == "mixed" and cfg.M < 2 * cfg.K:
        assert sent is not None, what
        got = np.unpackbits(hard, axis=-1)[..., :n_valid]
        want = np.stack([np.unpackbits(ref[l][2], axis=-1)[:, :n_valid] for l in range(cfg.U)])
        ber_g = np.mean(got != sent[..., :n_valid])
        ber_o = np.mean(want != sent[..., :n_valid])
        assert ber_g <= 1.25 * ber_o + 0.005, (what, ber_g, ber_o)
        return
    for l in range(cfg.U):
        llr_r, _, hard_r = ref[l]
        lr = llr_r.astype(np.float32)
        lg = llr[l].astype(np.float32)
        err = np.abs(lg - lr).max()
        assert err <= t["abs"] + t["rel"] * np.abs(lr).max(), (what, l, err)
        sure = np.abs(lr[:, zeros:zeros + n_valid]) > t["sure"]
        bg = np.unpackbits(hard[l], axis=1)[:, :n_valid]
        br = np.unpackbits(hard_r, axis=1)[:, :n_valid]
        assert (bg[sure] == br[sure]).all(), (what, l, int((bg[sure] != br[sure]).sum()))

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

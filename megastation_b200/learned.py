"""Learned ZF initialiser over the C ABI (mb_mlp_*, mb_lzf_*).

Per-subcarrier zero forcing from interpolated comb-pilot CSI, where the
initial iterate of each subcarrier is a blend of the exact inverses at the
neighbouring group centres with weights predicted by a 3-layer MLP (width
256, BF16 weights, FP32 accumulation), followed by Newton-Schulz steps.
The network is trained on the GPU by the library's own forward, backward
and Adam kernels, on pilot CSI of seeded channel realisations whose exact
FP64 per-subcarrier inverse is the label (mb_lzf_targets).  No counterpart
in the reference, whose ZF is per subcarrier group
(beamform/beamform.cu:74-122).
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._lib import LIB, check
from .ops import _dev, _stream

COARSE, LEARNED, EXACT = 0, 1, 2
N_BLEND = 4


def num_features(sg):
    return sg + 6


class MLP:
    """3-layer ReLU MLP n_in -> width -> width -> n_out (mb_mlp)."""

    def __init__(self, n_in, width=256, n_out=N_BLEND, max_batch=8192, seed=0, out_bias=None):
        h = ctypes.c_void_p()
        check(LIB.mb_mlp_create(n_in, width, n_out, max_batch, seed, ctypes.byref(h)), "mb_mlp_create")
        self._h = h
        self.n_in, self.width, self.n_out, self.max_batch = n_in, width, n_out, max_batch
        if out_bias is not None:
            p = self.params()
            p[-n_out:] = np.asarray(out_bias, np.float32)
            self.set_params(p)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and LIB is not None:  # LIB is None once the interpreter is shutting down
            LIB.mb_mlp_destroy(h)
            self._h = None

    def num_params(self):
        n = _lib.U64()
        check(LIB.mb_mlp_num_params(self._h, ctypes.byref(n)), "mb_mlp_num_params")
        return n.value

    def params(self):
        out = np.zeros(self.num_params(), np.float32)
        check(LIB.mb_mlp_get_params(self._h, out.ctypes.data_as(ctypes.c_void_p)), "mb_mlp_get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.num_params():
            raise ValueError("parameter count mismatch")
        check(LIB.mb_mlp_set_params(self._h, p.ctypes.data_as(ctypes.c_void_p)), "mb_mlp_set_params")

    def grads(self):
        out = np.zeros(self.num_params(), np.float32)
        check(LIB.mb_mlp_get_grads(self._h, out.ctypes.data_as(ctypes.c_void_p)), "mb_mlp_get_grads")
        return out

    def forward(self, x, out=None, stream=None):
        B = x.shape[0]
        out = torch.empty(B, self.n_out, dtype=torch.float32, device=x.device) if out is None else out
        check(LIB.mb_mlp_forward(self._h, _dev(x, "x", torch.float32), B, _dev(out, "y", torch.float32),
                                 _stream(stream)), "mb_mlp_forward")
        return out

    def loss_grad(self, x, A, b, c=None, loss=None, stream=None):
        """Gradients of the batch-mean quadratic loss into the object; the
        loss lands in the 1-element device tensor `loss` (returned)."""
        B = x.shape[0]
        loss = torch.zeros(1, dtype=torch.float32, device=x.device) if loss is None else loss
        check(LIB.mb_mlp_loss_grad(self._h, _dev(x, "x", torch.float32), _dev(A, "A", torch.float32),
                                   _dev(b, "b", torch.float32),
                                   None if c is None else _dev(c, "c", torch.float32), B,
                                   _dev(loss, "loss", torch.float32), _stream(stream)), "mb_mlp_loss_grad")
        return loss

    def adam_step(self, lr, stream=None):
        check(LIB.mb_mlp_adam_step(self._h, ctypes.c_float(lr), _stream(stream)), "mb_mlp_adam_step")


class LearnedZF:
    """Per-subcarrier ZF workspace for one cell shape (mb_lzf)."""

    def __init__(self, M, K, S, sg=16):
        h = ctypes.c_void_p()
        check(LIB.mb_lzf_create(M, K, S, sg, ctypes.byref(h)), "mb_lzf_create")
        self._h = h
        self.M, self.K, self.S, self.sg = M, K, S, sg
        self.G = (S + sg - 1) // sg
        self.n_features = num_features(sg)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and LIB is not None:  # LIB is None once the interpreter is shutting down
            LIB.mb_lzf_destroy(h)
            self._h = None

    def features(self, csi, out=None, stream=None):
        out = torch.empty(self.S, self.n_features, dtype=torch.float32, device=csi.device) if out is None else out
        check(LIB.mb_lzf_features(self._h, _dev(csi, "csi", torch.complex64), _dev(out, "features"),
                                  _stream(stream)), "mb_lzf_features")
        return out

    def targets(self, csi, A=None, b=None, stream=None):
        A = torch.empty(self.S, N_BLEND, N_BLEND, dtype=torch.float32, device=csi.device) if A is None else A
        b = torch.empty(self.S, N_BLEND, dtype=torch.float32, device=csi.device) if b is None else b
        check(LIB.mb_lzf_targets(self._h, _dev(csi, "csi", torch.complex64), _dev(A, "A"), _dev(b, "b"),
                                 _stream(stream)), "mb_lzf_targets")
        return A, b

    def run(self, csi, init=LEARNED, ns_iters=2, mlp=None, W=None, stream=None):
        """Per-subcarrier detector W [S][M][K] (use with sc_group = 1)."""
        W = torch.empty(self.S, self.M, self.K, dtype=torch.complex64, device=csi.device) if W is None else W
        check(LIB.mb_lzf_run(self._h, _dev(csi, "csi", torch.complex64), mlp._h if mlp is not None else None,
                             init, ns_iters, _dev(W, "W"), _stream(stream)), "mb_lzf_run")
        return W

    def flags(self, out=None, stream=None):
        """Per subcarrier of the last run: 0 Newton-Schulz from the chosen
        start, 1 not positive definite, 2 start too far off (exact inverse
        taken instead)."""
        out = torch.empty(self.S, dtype=torch.int32, device="cuda") if out is None else out
        check(LIB.mb_lzf_flags(self._h, _dev(out, "flags"), _stream(stream)), "mb_lzf_flags")
        return out

    def residual(self, out=None, stream=None):
        out = torch.empty(self.S, dtype=torch.float32, device="cuda") if out is None else out
        check(LIB.mb_lzf_residual(self._h, _dev(out, "res"), _stream(stream)), "mb_lzf_residual")
        return out


def pilot_csi(cfg, n, seed, delay_spread_ns=(50.0, 300.0), device="cuda"):
    """n pilot-CSI realisations [n][G][M][K] (complex64, device) of the
    'tdl_ds' channel of datagen with the delay spread drawn uniformly per
    realisation: the LS comb-pilot estimate conj(H) at user u's pilot
    subcarrier g sg + u mod sg plus CN(0, noise) estimation noise, i.e. what
    the pilot FFT returns.  Synthetic training data, generated with torch."""
    from . import datagen
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    rng = np.random.default_rng(seed)
    G, M, K, sg, S = cfg.G, cfg.M, cfg.K, cfg.sg, cfg.S
    L = cfg.n_taps
    s_pil = (np.arange(G)[:, None] * sg + (np.arange(K)[None, :] % sg))  # [G][K]
    s_pil = np.minimum(s_pil, S - 1)
    bins = (s_pil + cfg.start + cfg.N // 2) % cfg.N
    f = ((bins + cfg.N // 2) % cfg.N) - cfg.N // 2  # signed bin offsets [G][K]
    f_t = torch.from_numpy(f.astype(np.float64)).to(device)
    noise = 10.0 ** (-cfg.snr_db / 10.0)
    out = torch.empty(n, G, M, K, dtype=torch.complex64, device=device)
    for i in range(n):
        ds = float(rng.uniform(*delay_spread_ns))
        c = datagen.CellConfig(**{**cfg.__dict__, "channel": "tdl_ds", "delay_spread_ns": ds})
        tau, pdp = datagen.tap_profile(c)
        w = torch.complex(torch.randn(L, M, K, generator=g, device=device, dtype=torch.float64),
                          torch.randn(L, M, K, generator=g, device=device, dtype=torch.float64)) / math.sqrt(2)
        if cfg.rho:
            idx = np.arange(M)
            Rh = np.linalg.cholesky(cfg.rho ** np.abs(idx[:, None] - idx[None, :]))
            w = torch.einsum("ab,lbk->lak", torch.from_numpy(Rh).to(device).to(w.dtype), w)
        taps = w * torch.from_numpy(np.sqrt(pdp)).to(device)[:, None, None]
        tau_t = torch.from_numpy(tau).to(device)
        ph = torch.exp(-2j * math.pi * f_t[..., None] * tau_t / cfg.N)  # [G][K][L]
        H = torch.einsum("gkl,lbk->gbk", ph, taps)  # [G][M][K] at each user's pilot
        nz = torch.complex(torch.randn(G, M, K, generator=g, device=device, dtype=torch.float64),
                           torch.randn(G, M, K, generator=g, device=device, dtype=torch.float64))
        out[i] = (torch.conj(H) + nz * math.sqrt(noise / 2)).to(torch.complex64)
    return out


def training_set(lzf, csi_batch, stream=None):
    """Features, A, b and c = 1 of every subcarrier of every realisation."""
    n = csi_batch.shape[0]
    S, F = lzf.S, lzf.n_features
    X = torch.empty(n * S, F, dtype=torch.float32, device="cuda")
    A = torch.empty(n * S, N_BLEND, N_BLEND, dtype=torch.float32, device="cuda")
    b = torch.empty(n * S, N_BLEND, dtype=torch.float32, device="cuda")
    for i in range(n):
        lzf.features(csi_batch[i], out=X[i * S:(i + 1) * S], stream=stream)
        lzf.targets(csi_batch[i], A=A[i * S:(i + 1) * S], b=b[i * S:(i + 1) * S], stream=stream)
    return X, A, b, torch.ones(n * S, dtype=torch.float32, device="cuda")


def train(mlp, data, steps, batch=4096, lr=1e-3, seed=0, log_every=0, stream=None):
    """Adam on shuffled mini-batches of `data` (features, A, b, c); returns
    the loss history (one entry per logged step)."""
    X, A, b, c = data
    n = X.shape[0]
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    hist = []
    perm = torch.randperm(n, generator=gen, device="cuda")
    pos = 0
    for k in range(steps):
        if pos + batch > n:
            perm = torch.randperm(n, generator=gen, device="cuda")
            pos = 0
        idx = perm[pos:pos + batch]
        pos += batch
        mlp.loss_grad(X[idx].contiguous(), A[idx].contiguous(), b[idx].contiguous(), c[idx].contiguous(),
                      loss=loss, stream=stream)
        mlp.adam_step(lr, stream=stream)
        if log_every and (k % log_every == 0 or k == steps - 1):
            hist.append((k, float(loss.item())))
    return hist


def blend_loss(mlp, data, batch=8192):
    """Mean normalised squared distance of the learned blend to the exact
    inverse over `data` (and of the coarse choice alpha = (0, 1, 0, 0))."""
    X, A, b, c = data
    tot_l, tot_c, n = 0.0, 0.0, X.shape[0]
    for i in range(0, n, batch):
        xs = X[i:i + batch]
        y = mlp.forward(xs.contiguous()).double()
        Ai, bi = A[i:i + batch].double(), b[i:i + batch].double()
        q = torch.einsum("bi,bij,bj->b", y, Ai, y) - 2 * (bi * y).sum(1) + 1
        tot_l += float(q.sum())
        tot_c += float((Ai[:, 1, 1] - 2 * bi[:, 1] + 1).sum())
    return tot_l / n, tot_c / n


def make_mlp(sg=16, width=256, seed=0, max_batch=8192):
    """An untrained network whose output is the coarse blend (0, 1, 0, 0)."""
    return MLP(num_features(sg), width, N_BLEND, max_batch=max_batch, seed=seed, out_bias=[0, 1, 0, 0])


# ---------------------------------------------------------------------------
# Learned initial iterate of the group ZF (mixed precision, any cell shape):
# a network maps six spectral features of a group's Gram to the coefficients
# of a cubic polynomial X0 = p(Gn) / tau, the Newton-Schulz start that
# replaces the exact inverse (mb_zf_set_init_net, mb_slot_set_zf_init).

ZF_INIT_FEATURES, ZF_INIT_COEFFS = 6, 4
# (I - (I - Gn))^-1 to third order: the untrained network's output, and the
# fixed (not learned) polynomial the learned one is compared with
NEUMANN3 = (4.0, -6.0, 4.0, -1.0)


def make_zf_init_net(width=64, seed=0, max_batch=8192):
    """An untrained initial-iterate network (6 -> width -> width -> 4, ReLU,
    BF16 weights) whose output is the third-order Neumann polynomial."""
    return MLP(ZF_INIT_FEATURES, width, ZF_INIT_COEFFS, max_batch=max_batch, seed=seed, out_bias=NEUMANN3)


def group_csi(M, K, n, seed, G=205, sg=16, N=4096, S=3276, n_taps=8, rho=(0.3, 0.7), tap_decay=(1.0, 3.0),
              snr_db=(18.0, 30.0), batch=32, device="cuda"):
    """n comb-pilot CSI realisations [n][G][M][K] (complex64, device) of the
    'tdl' channel of datagen: n_taps taps at 0..n_taps-1 samples with PDP
    e^{-l / decay}, exponential receive correlation rho, CN(0, 1) per tap
    and link; user u's estimate conj(H) sits at its pilot subcarrier
    g sg + u mod sg, plus CN(0, 10^(-snr/10)) estimation noise.  rho, decay
    and SNR are drawn uniformly per realisation from the given ranges.
    Synthetic training data, generated with torch in batches."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    rng = np.random.default_rng(seed)
    start = (N - S) // 2
    s_pil = np.minimum(np.arange(G)[:, None] * sg + (np.arange(K)[None, :] % sg), S - 1)  # [G][K]
    bins = (s_pil + start + N // 2) % N
    f = torch.from_numpy((((bins + N // 2) % N) - N // 2).astype(np.float64)).to(device)
    tau = torch.arange(n_taps, dtype=torch.float64, device=device)
    ph = torch.exp(-2j * math.pi * f[..., None] * tau / N)  # [G][K][L]
    idx = np.arange(M)
    out = torch.empty(n, G, M, K, dtype=torch.complex64, device=device)
    for i0 in range(0, n, batch):
        B = min(batch, n - i0)
        rh = rng.uniform(*rho, B)
        dec = rng.uniform(*tap_decay, B)
        snr = rng.uniform(*snr_db, B)
        Rh = np.stack([np.linalg.cholesky(r ** np.abs(idx[:, None] - idx[None, :]) + 1e-12 * np.eye(M)) for r in rh])
        pdp = np.exp(-np.arange(n_taps)[None, :] / dec[:, None])
        pdp /= pdp.sum(1, keepdims=True)
        w = torch.complex(torch.randn(B, n_taps, M, K, generator=g, device=device, dtype=torch.float64),
                          torch.randn(B, n_taps, M, K, generator=g, device=device, dtype=torch.float64)) / math.sqrt(2)
        w = torch.einsum("nab,nlbk->nlak", torch.from_numpy(Rh).to(device).to(w.dtype), w)
        w = w * torch.from_numpy(np.sqrt(pdp)).to(device)[:, :, None, None]
        H = torch.einsum("gkl,nlbk->ngbk", ph, w)  # [B][G][M][K]
        nz = torch.complex(torch.randn(B, G, M, K, generator=g, device=device, dtype=torch.float64),
                           torch.randn(B, G, M, K, generator=g, device=device, dtype=torch.float64))
        sd = torch.from_numpy(np.sqrt(10.0 ** (-snr / 10.0) / 2)).to(device)[:, None, None, None]
        out[i0:i0 + B] = (torch.conj(H) + nz * sd).to(torch.complex64)
    return out


def zf_init_targets(csi, stream=None):
    """(features [G][6], A [G][4][4], b [G][4]) of every group of csi
    [G][M][K] (mb_zf_init_targets, FP64 on the GPU)."""
    G, M, K = csi.shape
    F = torch.empty(G, ZF_INIT_FEATURES, dtype=torch.float32, device=csi.device)
    A = torch.empty(G, ZF_INIT_COEFFS, ZF_INIT_COEFFS, dtype=torch.float32, device=csi.device)
    b = torch.empty(G, ZF_INIT_COEFFS, dtype=torch.float32, device=csi.device)
    check(LIB.mb_zf_init_targets(_dev(csi, "csi", torch.complex64), G, M, K, _dev(F, "features"), _dev(A, "A"),
                                 _dev(b, "b"), _stream(stream)), "mb_zf_init_targets")
    return F, A, b


def zf_init_training_set(shapes, n_real, seed, **channel):
    """Features, A, b and c = 1 of every group of n_real realisations per
    (M, K) shape in `shapes` (group_csi's channel model)."""
    Xs, As, bs = [], [], []
    for k, (M, K) in enumerate(shapes):
        done = 0
        while done < n_real:
            n = min(64, n_real - done)
            csi = group_csi(M, K, n, seed + 7919 * k + done, **channel)
            F, A, b = zf_init_targets(csi.view(-1, M, K))  # every group of every realisation
            Xs.append(F)
            As.append(A)
            bs.append(b)
            done += n
    X, A, b = torch.cat(Xs), torch.cat(As), torch.cat(bs)
    return X, A, b, torch.ones(X.shape[0], dtype=torch.float32, device=X.device)


def poly_residual(net, data, batch=8192):
    """Mean ||I - Gn p(Gn)||_F^2 / K over `data` for the network's
    coefficients and for the fixed Neumann polynomial."""
    X, A, b, c = data
    tot_l, tot_n, n = 0.0, 0.0, X.shape[0]
    a_n = torch.tensor(NEUMANN3, dtype=torch.float64, device=X.device)
    for i in range(0, n, batch):
        y = net.forward(X[i:i + batch].contiguous()).double()
        Ai, bi = A[i:i + batch].double(), b[i:i + batch].double()
        tot_l += float((torch.einsum("bi,bij,bj->b", y, Ai, y) - 2 * (bi * y).sum(1) + 1).sum())
        tot_n += float((torch.einsum("i,bij,j->b", a_n, Ai, a_n) - 2 * (bi * a_n).sum(1) + 1).sum())
    return tot_l / n, tot_n / n

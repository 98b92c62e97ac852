"""FP64 restatement of the learned ZF initialiser (numpy).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU
kernels in megastation_b200/csrc/mlp.cu and lzf.cu; the product package never
imports it.  The algorithms have no counterpart in the reference (the
reference ZF is per subcarrier group, beamform/beamform.cu:74-122); they are
restated here from their definitions:

- mlp_forward / mlp_loss_grad: the 3-layer ReLU MLP with both operands of
  every product rounded to BF16 (round to nearest even): the weights, the
  inputs and hidden activations, and in the backward pass the upstream
  gradients; biases and the bias gradients (column sums) in full precision,
  and the quadratic loss y^T A y - 2 b^T y + c averaged over the batch;
  gradients are taken with respect to the (FP32) master parameters through
  the rounding (straight-through), flat in the order W1, b1, W2, b2, W3, b3.
- interp_csi / gram / centre_inverses / features / targets: the
  per-subcarrier CSI interpolation, the reference-convention Gram C C^H, the
  centre inverses and the blend targets of lzf.cu.
"""
import numpy as np


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, n_in, width, n_out):
    p = np.asarray(params, dtype=np.float64)
    sizes = [n_in * width, width, width * width, width, width * n_out, n_out]
    out, o = [], 0
    for s in sizes:
        out.append(p[o:o + s])
        o += s
    W1, b1, W2, b2, W3, b3 = out
    return W1.reshape(n_in, width), b1, W2.reshape(width, width), b2, W3.reshape(width, n_out), b3


def _round_act(act_bf16):
    """The rounding of an activation or gradient entering a product: BF16, or
    none (act_bf16 False, the smooth model a finite-difference check needs)."""
    if act_bf16:
        return lambda v: bf16(np.asarray(v).astype(np.float32))
    return lambda v: np.asarray(v, np.float64)


def mlp_forward(params, x, n_in, width, n_out, act_bf16=True):
    W1, b1, W2, b2, W3, b3 = unpack(params, n_in, width, n_out)
    W1, W2, W3 = bf16(W1), bf16(W2), bf16(W3)
    r = _round_act(act_bf16)
    x = r(np.asarray(x, np.float32) if act_bf16 else x)
    z1 = x @ W1 + b1
    h1 = r(np.maximum(z1, 0))
    z2 = h1 @ W2 + b2
    h2 = r(np.maximum(z2, 0))
    return h2 @ W3 + b3, (x, z1, h1, z2, h2, W1, W2, W3)


def mlp_loss_grad(params, x, A, b, c, n_in, width, n_out, act_bf16=True):
    y, (x, z1, h1, z2, h2, W1, W2, W3) = mlp_forward(params, x, n_in, width, n_out, act_bf16)
    B = x.shape[0]
    A = np.asarray(A, np.float64).reshape(B, n_out, n_out)
    b = np.asarray(b, np.float64).reshape(B, n_out)
    c = np.zeros(B) if c is None else np.asarray(c, np.float64)
    Ay = np.einsum("bij,bj->bi", A, y)
    loss = np.mean(np.einsum("bi,bi->b", y, Ay) - 2 * np.einsum("bi,bi->b", b, y) + c)
    dy = 2 * (Ay - b) / B
    r = _round_act(act_bf16)  # an upstream gradient entering a product
    gW3 = h2.T @ r(dy)
    gb3 = dy.sum(0)
    d2 = (r(dy) @ W3.T) * (z2 > 0)
    gW2 = h1.T @ r(d2)
    gb2 = d2.sum(0)
    d1 = (r(d2) @ W2.T) * (z1 > 0)
    gW1 = x.T @ r(d1)
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def interp_csi(csi, S, sg):
    """csi [G][M][K] comb-pilot estimates -> per-subcarrier c_s [S][M][K]:
    linear interpolation of user u's pilots (subcarriers g sg + u mod sg),
    clamped at the band edges (lzf.cu interp_kernel)."""
    csi = np.asarray(csi, np.complex128)
    G, M, K = csi.shape
    out = np.zeros((S, M, K), np.complex128)
    for u in range(K):
        p = (np.arange(S) - (u % sg)) / sg
        g0 = np.clip(np.floor(p).astype(int), 0, max(G - 2, 0))
        t = np.clip(p - g0, 0, 1) if G > 1 else np.zeros(S)
        g1 = np.minimum(g0 + 1, G - 1)
        out[:, :, u] = (1 - t)[:, None] * csi[g0, :, u] + t[:, None] * csi[g1, :, u]
    return out


def gram(c):
    """G_s = C C^H with C[u][b] = c_s[b][u]: G[u][v] = sum_b c[b][u] conj(c[b][v])."""
    return np.einsum("sbu,sbv->suv", c, np.conj(c))


def centres(S, sg):
    G = (S + sg - 1) // sg
    return np.minimum(np.arange(G) * sg + sg // 2, S - 1)


def features(Gs, S, sg):
    """lzf.cu features_kernel from the per-subcarrier Grams."""
    Gc = Gs[centres(S, sg)]
    G = Gc.shape[0]
    F = np.zeros((S, sg + 6))
    for s in range(S):
        g, o = s // sg, s % sg
        F[s, o] = 1
        C0 = Gc[g]
        n0 = np.linalg.norm(C0)
        t0 = np.trace(C0).real
        for q, j in enumerate((-1, 1, 2)):
            gj = g + j
            if 0 <= gj < G:
                F[s, sg + q] = np.linalg.norm(Gc[gj] - C0) / n0 if n0 > 0 else 0
                F[s, sg + 3 + q] = np.trace(Gc[gj]).real / t0 - 1 if t0 > 0 else 0
    return F


def targets(Gs, S, sg):
    """A [S][4][4], b [S][4] of the blend of centre inverses g-1..g+2 against
    the exact inverse of G_s (lzf.cu targets_kernel)."""
    Xs = np.linalg.inv(Gs)
    Yc = Xs[centres(S, sg)]
    G = Yc.shape[0]
    A = np.zeros((S, 4, 4))
    b = np.zeros((S, 4))
    for s in range(S):
        g = s // sg
        Y = [Yc[min(max(g + j - 1, 0), G - 1)] for j in range(4)]
        nx = np.sum(np.abs(Xs[s]) ** 2)
        for j in range(4):
            b[s, j] = np.sum((np.conj(Y[j]) * Xs[s]).real) / nx
            for k in range(4):
                A[s, j, k] = np.sum((np.conj(Y[j]) * Y[k]).real) / nx
    return A, b

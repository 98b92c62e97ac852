"""FP64 restatement of the learned initial iterate of the mixed ZF.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker.  The product
(megastation_b200/csrc/zf_mixed.cu poly_init, csrc/zf_init.cu) never
imports it.  No counterpart in the reference, whose ZF solves each group's
Gram exactly (beamform/beamform.cu:74-122); this file restates the
polynomial start and its Newton-Schulz refinement so that the GPU's
features, training targets and accept decisions can be checked.
"""
import numpy as np

NEUMANN3 = np.array([4.0, -6.0, 4.0, -1.0])
ACCEPT = 0.04


def gram(csi_g):
    """G = C C^H with C[u][b] = csi_g[b][u] (beamform.cu:74-122)."""
    C = np.asarray(csi_g, np.complex128).T
    return C @ C.conj().T


def features_targets(G, M):
    """(features [6], A [4][4], b [4]) of one Gram: t_k = tr(Gn^k) / K with
    Gn = G / (tr G / K); features t2 - 1, t3 - 3 t2 + 2,
    t4 - 4 t3 + 6 t2 - 3, min / max diag(Gn) - 1, K / M; A_ij = t_(i+j+2),
    b_i = t_(i+1)."""
    K = G.shape[0]
    tau = np.trace(G).real / K
    Gn = G / tau
    t = [1.0]
    P = np.eye(K, dtype=np.complex128)
    for k in range(1, 9):
        P = P @ Gn
        t.append(np.trace(P).real / K)
    d = np.diag(Gn).real
    f = np.array([t[2] - 1, t[3] - 3 * t[2] + 2, t[4] - 4 * t[3] + 6 * t[2] - 3, d.min() - 1, d.max() - 1, K / M])
    A = np.array([[t[i + j + 2] for j in range(4)] for i in range(4)])
    b = np.array([t[i + 1] for i in range(4)])
    return f, A, b


def residual_sq(G, alpha):
    """||I - Gn p_alpha(Gn)||_F^2 / K computed directly."""
    K = G.shape[0]
    Gn = G / (np.trace(G).real / K)
    X = sum(a * np.linalg.matrix_power(Gn, i) for i, a in enumerate(alpha))
    E = np.eye(K) - Gn @ X
    return float(np.sum(np.abs(E) ** 2) / K)


def poly_ns(G, alpha, ns_iters=2):
    """The kernel's schedule in FP64: X0 = p_alpha(Gn) / tau, ns_iters
    Newton-Schulz steps plus at most two more while ACCEPT < ||E|| < 0.3;
    returns (X, accepted, residual norm before the last step)."""
    K = G.shape[0]
    tau = np.trace(G).real / K
    Gn = G / tau
    X = sum(a * np.linalg.matrix_power(Gn, i) for i, a in enumerate(alpha)) / tau
    e_last = np.inf
    for s in range(ns_iters + 2):
        if s >= ns_iters and (e_last <= ACCEPT or e_last >= 0.3):
            break
        E = np.eye(K) - G @ X
        e_last = np.linalg.norm(E)
        if not e_last < 1.0:
            return X, False, e_last
        X = X @ (np.eye(K) + E)
    return X, e_last <= ACCEPT, e_last

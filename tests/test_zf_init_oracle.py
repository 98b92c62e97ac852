"""CPU checks of the learned initial iterate's restatement (oracle/zf_init.py):
the quadratic form A, b reproduces the residual computed directly, the
Newton-Schulz schedule squares the residual, and the fixed Neumann
polynomial, which the learned coefficients replace, does not converge on a
256 x 32 Gram with correlated antennas while its least-squares optimum does."""
import numpy as np

from oracle import zf_init as zi


def _csi(M, K, rho, seed):
    rng = np.random.default_rng(seed)
    R = rho ** np.abs(np.arange(M)[:, None] - np.arange(M)[None, :])
    L = np.linalg.cholesky(R)
    h = (rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))) / np.sqrt(2)
    return L @ h


def test_quadratic_form_is_the_residual():
    G = zi.gram(_csi(64, 16, 0.3, 1))
    f, A, b = zi.features_targets(G, 64)
    for alpha in (zi.NEUMANN3, np.array([1.0, 0.5, -0.2, 0.01]), np.linalg.solve(A, b)):
        q = alpha @ A @ alpha - 2 * b @ alpha + 1
        assert abs(q - zi.residual_sq(G, alpha)) <= 1e-9 * max(1.0, q)
    assert f[5] == 16 / 64 and abs(f[0] - (np.sum(np.abs(G / (np.trace(G).real / 16)) ** 2) / 16 - 1)) < 1e-12


def test_least_squares_polynomial_converges_where_neumann_does_not():
    G = zi.gram(_csi(256, 32, 0.5, 2))
    f, A, b = zi.features_targets(G, 256)
    a = np.linalg.solve(A, b)
    X, ok, e = zi.poly_ns(G, a)
    assert ok and e <= zi.ACCEPT
    assert np.linalg.norm(np.eye(32) - G @ X) <= e * e * 1.01 + 1e-12
    assert np.abs(X - np.linalg.inv(G)).max() <= 2e-3 * np.abs(np.linalg.inv(G)).max()
    _, ok_n, _ = zi.poly_ns(G, zi.NEUMANN3)
    assert not ok_n

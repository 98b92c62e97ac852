"""The FP64 restatement of the learned initialiser (oracle/mlp.py), checked
on its own: BF16 rounding and a finite-difference gradient check."""
import numpy as np

from oracle import mlp as om


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-30], np.float32)
    r = om.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1.0); 1 + 1.5 2^-8 rounds up
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)


def test_oracle_gradient_finite_difference():
    rng = np.random.default_rng(0)
    n_in, width, n_out, B = 5, 7, 4, 6
    n = n_in * width + width + width * width + width + width * n_out + n_out
    # parameters already on the BF16 grid so the rounding is the identity
    p = om.bf16(rng.standard_normal(n).astype(np.float32) * 0.5)
    x = rng.standard_normal((B, n_in))
    M = rng.standard_normal((B, n_out, n_out))
    A = np.einsum("bij,bkj->bik", M, M) / n_out
    b = rng.standard_normal((B, n_out))
    c = rng.standard_normal(B)
    # the smooth model (activations not rounded): its gradient is what the
    # backward pass computes, with the roundings of the GPU's products
    # applied at the same places in mlp_loss_grad's default mode
    loss, g = om.mlp_loss_grad(p, x, A, b, c, n_in, width, n_out, act_bf16=False)

    def f(q):
        y, _ = om.mlp_forward(q, x, n_in, width, n_out, act_bf16=False)
        # same loss without the BF16 rounding of the perturbed weights
        return np.mean(np.einsum("bi,bij,bj->b", y, A, y) - 2 * np.einsum("bi,bi->b", b, y) + c)

    W1, b1, W2, b2, W3, b3 = om.unpack(p, n_in, width, n_out)
    # finite differences in float64 on the biases (never rounded) and on
    # weights through an exactly representable step of the BF16 grid
    for idx in list(range(n_in * width, n_in * width + width)) + [n - 1, n - 2]:
        e = np.zeros(n)
        e[idx] = 1e-6
        num = (f(p + e) - f(p - e)) / 2e-6
        assert abs(num - g[idx]) <= 1e-6 + 1e-5 * abs(num), idx
    assert np.isfinite(loss)

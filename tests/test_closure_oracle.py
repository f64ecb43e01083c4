"""The closure model's CPU oracle (oracle/closure_oracle.py), pinned by finite differences.

The reference has no closure model, so the oracle's gradients are checked against central
differences of its own float64 loss (relative error 1e-6 on every layer, a batch of two
fields); im2col and col2im are checked to be adjoint (<A x, y> = <x, A^T y> to 1e-12) and the
GELU derivative against differences of GELU.
"""
import numpy as np
import pytest

from conftest import load_oracle_module


@pytest.fixture(scope="module")
def co():
    return load_oracle_module("closure_oracle")


def _params(rng, H):
    shapes = [(H, 5), (H, H), (H, H), (1, H)]
    return [(rng.standard_normal((o, 9, i)) * np.sqrt(2.0 / (9 * i)), 0.1 * rng.standard_normal(o)) for o, i in shapes]


def test_im2col_col2im_adjoint(co):
    rng = np.random.default_rng(1)
    x = rng.standard_normal((7, 8, 3))
    y = rng.standard_normal((7, 8, 9, 3))
    assert abs((co.im2col(x) * y).sum() - (x * co.col2im(y)).sum()) < 1e-12 * np.abs(y).sum()


def test_gelu_grad(co):
    x = np.linspace(-4, 4, 41)
    fd = (co.gelu(x + 1e-6) - co.gelu(x - 1e-6)) / 2e-6
    assert np.allclose(co.gelu_grad(x), fd, atol=1e-8)


def test_gradients_match_finite_differences(co):
    rng = np.random.default_rng(2)
    Ny, Nx, H = 7, 8, 4
    params = _params(rng, H)
    samples = [tuple(rng.standard_normal((Ny, Nx)) for _ in range(5)) for _ in range(2)]
    y = np.linspace(-1, 1, Ny)
    scales = ((1.3, 0.7, 0.9, 1.1), 2.0)
    loss, grads = co.loss_and_grads(params, samples, y, scales)
    eps = 1e-6
    for layer in range(4):
        W, b = params[layer]
        for arr, g in ((W, grads[layer][0]), (b, grads[layer][1])):
            flat = arr.reshape(-1)
            idx = rng.choice(flat.size, size=min(10, flat.size), replace=False)
            for k in idx:
                old = flat[k]
                flat[k] = old + eps
                lp, _ = co.loss_and_grads(params, samples, y, scales)
                flat[k] = old - eps
                lm, _ = co.loss_and_grads(params, samples, y, scales)
                flat[k] = old
                fd = (lp - lm) / (2 * eps)
                assert abs(fd - g.reshape(-1)[k]) <= 1e-6 * max(1.0, abs(fd)), (layer, k, fd, g.reshape(-1)[k])


def test_bf16_rounding(co):
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0e-40, 65504.0, 1.0 + 2 ** -9])
    r = co.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[5] == 1.0


def test_box_filter_constant_and_linear(co):
    f = np.full((17, 16), 3.0)
    assert np.allclose(co.box_filter(f, 4, 5), 3.0)
    x = np.arange(16)[None, :] * np.ones((17, 1))
    c = co.box_filter(np.sin(2 * np.pi * x / 16), 4, 5)
    assert c.shape == (5, 4) and np.all(np.isfinite(c))

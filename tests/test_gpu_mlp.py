"""Estimator MLP kernels vs the float64 NumPy oracle (forward, loss, gradient, training)."""
import numpy as np
import pytest

import sjoin
from oracle import mlp

pytestmark = pytest.mark.gpu


def _data(m, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((m, 16)).astype(np.float32)
    t = np.stack([x[:, :4].sum(1), np.abs(x[:, 4:8]).sum(1)], 1).astype(np.float32)
    return x, t


def test_forward_matches_oracle():
    x, _ = _data(1000, 1)
    w = sjoin.mlp_init(1)
    got = sjoin.mlp_forward(x, w)
    ref = mlp.forward(x.astype(np.float64), w.astype(np.float64))
    # FP32 accumulation over 16 and 64 terms
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("m", [1, 37, 4096])
def test_gradient_matches_oracle(m):
    x, t = _data(m, 2)
    w = sjoin.mlp_init(2)
    loss, g = sjoin.mlp_loss_grad(x, t, w)
    rloss, rg = mlp.loss_grad(x, t, w.astype(np.float64))
    assert abs(loss - rloss) <= 1e-4 * max(1.0, abs(rloss))
    # tolerance: FP32 sums of up to 4096 per-sample terms
    np.testing.assert_allclose(g, rg, rtol=2e-3, atol=2e-5 * max(1.0, np.abs(rg).max()))


def test_gradient_matches_finite_differences():
    x, t = _data(64, 3)
    w = sjoin.mlp_init(3).astype(np.float64)
    _, g = mlp.loss_grad(x, t, w)
    gd, _ = sjoin.mlp_loss_grad(x, t, w.astype(np.float32))[1], None
    idx = np.random.default_rng(0).choice(w.size, 40, replace=False)
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (mlp.loss_grad(x, t, wp)[0] - mlp.loss_grad(x, t, wm)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 + 1e-4 * abs(fd)
        assert abs(gd[i] - g[i]) <= 1e-4 + 2e-3 * abs(g[i])


def test_training_reduces_loss():
    x, t = _data(20000, 4)
    w0 = sjoin.mlp_init(4)
    l0, _ = sjoin.mlp_loss_grad(x, t, w0)
    w, l1 = sjoin.mlp_train(x, t, w0, steps=600, lr=2e-3, batch=2048)
    assert l1 < 0.2 * l0
    lr_, _ = mlp.loss_grad(x, t, w.astype(np.float64))
    assert abs(lr_ - l1) <= 1e-3 * max(1.0, lr_)

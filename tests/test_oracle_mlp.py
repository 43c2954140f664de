"""The estimator MLP's float64 restatement (oracle/mlp.py), the checker of the
GPU forward/backward kernels, pinned on CPU: its gradient against central
finite differences, and its forward pass against an independent per-sample
loop over the documented parameter layout."""
import numpy as np

from oracle import mlp


def _params(seed):
    rng = np.random.default_rng(seed)
    n = mlp.F * mlp.H + mlp.H + mlp.H * mlp.H + mlp.H + mlp.H * mlp.O + mlp.O
    return rng.standard_normal(n) * 0.3


def _data(m, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((m, mlp.F))
    t = np.stack([x[:, :4].sum(1), np.abs(x[:, 4:8]).sum(1)], 1)
    return x, t


def test_gradient_matches_finite_differences():
    x, t = _data(48, 1)
    w = _params(2)
    loss, g = mlp.loss_grad(x, t, w)
    assert np.isfinite(loss) and g.shape == w.shape
    h = 1e-6
    for i in np.random.default_rng(3).choice(w.size, 60, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (mlp.loss_grad(x, t, wp)[0] - mlp.loss_grad(x, t, wm)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_forward_matches_per_sample_loop():
    x, t = _data(5, 4)
    w = _params(5)
    o = 0
    parts = {}
    for name, size in (("W1", mlp.F * mlp.H), ("b1", mlp.H), ("W2", mlp.H * mlp.H), ("b2", mlp.H),
                       ("W3", mlp.H * mlp.O), ("b3", mlp.O)):
        parts[name] = w[o:o + size]
        o += size
    out = mlp.forward(x, w)
    for s in range(len(x)):
        h1 = [max(0.0, parts["b1"][j] + sum(x[s, i] * parts["W1"][i * mlp.H + j] for i in range(mlp.F)))
              for j in range(mlp.H)]
        h2 = [max(0.0, parts["b2"][j] + sum(h1[i] * parts["W2"][i * mlp.H + j] for i in range(mlp.H)))
              for j in range(mlp.H)]
        y = [parts["b3"][j] + sum(h2[i] * parts["W3"][i * mlp.O + j] for i in range(mlp.H)) for j in range(mlp.O)]
        np.testing.assert_allclose(out[s], y, rtol=1e-12, atol=1e-12)
    loss, _ = mlp.loss_grad(x, t, w)
    assert abs(loss - ((out - t) ** 2).sum() / (2 * len(x))) <= 1e-12 * max(1.0, loss)

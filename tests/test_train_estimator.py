"""Host logic of the estimator's training script (CPU): the training-set
resampling and the output-bias calibration, with the float64 NumPy
restatement of the network standing in for the engine's forward kernel."""
import numpy as np

import oracle.mlp as omlp
import sjoin
from sjoin import train_estimator as te


def _data(m=4000, seed=3):
    rng = np.random.default_rng(seed)
    x = rng.random((m, 16)).astype(np.float32)
    # targets: log2(1 + hits) with heavy-tailed hits
    y = np.stack([x[:, 0] * 12 + rng.normal(0, 0.7, m), x[:, 1] * 10 + rng.normal(0, 0.7, m)], 1)
    return x, np.maximum(y, 0).astype(np.float32)


def test_calibration_makes_summed_predictions_match(monkeypatch):
    monkeypatch.setattr(te, "mlp_forward", lambda x, w: omlp.forward(x, w).astype(np.float32))
    x, y = _data()
    w = sjoin.mlp_init(5)
    w[-2:] += np.array([9.0, 7.0], np.float32)   # an untrained net with a plausible output scale
    wc, shift = te.calibrate(x, y, w)
    assert np.array_equal(wc[:-2], w[:-2])        # only the two output biases move
    np.testing.assert_allclose(wc[-2:] - w[-2:], shift, rtol=1e-6, atol=1e-6)
    meas = (np.exp2(y.astype(np.float64)) - 1.0).sum(0)
    before = np.maximum(np.exp2(omlp.forward(x, w)) - 1.0, 0.0).sum(0) / meas
    after = np.maximum(np.exp2(omlp.forward(x, wc)) - 1.0, 0.0).sum(0) / meas
    # the shift scales 2^p, not 2^p - 1: exact only for cells with many hits, so the
    # summed ratio lands within a small fraction of 1 rather than on it
    assert np.all(np.abs(after - 1.0) < 0.01), (before, after)
    assert np.all(np.abs(after - 1.0) < np.abs(before - 1.0)), (before, after)


def test_resampling_favours_cells_with_many_hits():
    x, y = _data(20000)
    xt, yt = te.resample(x, y, size=40000, beta=1.0, seed=2)
    assert xt.shape == (40000, 16) and yt.shape == (40000, 2)
    hits = (np.exp2(y.astype(np.float64)) - 1).sum(1)
    hits_t = (np.exp2(yt.astype(np.float64)) - 1).sum(1)
    assert hits_t.mean() > 1.5 * hits.mean()

"""The learned estimator's per-cell features against a NumPy restatement (GPU).

Features 9, 13 and 14 are the expected hits of a cell with its owned
neighbours under a locally uniform density: log2(1 + occupancy x sum over the
owned neighbours of occupancy x w_m), over all offset classes, face neighbours
(m = 1) and edge neighbours (m = 2), where w_m is the probability that two
points uniform in two eps-wide cells differing by one in m of the k indexed
coordinates lie within eps.  The weights are checked against a Monte Carlo
estimate, and the features against the same sums over the grid built here
(cells eps wide from min - eps, linear id dim 0 fastest, linear-ID Unicomp
ownership: the neighbour with the larger linear id).
"""
import itertools

import numpy as np
import pytest

import sjoin

NB = 1024


def offset_class_weights(k):
    v = np.arange(NB + 1) / NB
    p0 = np.diff(2 * np.sqrt(v) - v)
    p1 = np.diff(v / 2)

    def power(p, j):
        z = np.zeros(NB)
        z[0] = 1.0
        for _ in range(j):
            z = np.convolve(z, p)[:NB]
        return z
    return np.array([np.convolve(power(p1, m), power(p0, k - m))[:NB].sum() for m in range(k + 1)])


def test_offset_class_weights_match_monte_carlo():
    w = offset_class_weights(6)
    rng = np.random.default_rng(3)
    m_pts = 400_000
    for m in range(4):
        a = rng.random((m_pts, 6))
        b = rng.random((m_pts, 6))
        b[:, :m] += 1.0
        mc = np.mean(((a - b) ** 2).sum(1) <= 1.0)
        assert abs(w[m] - mc) < 4 * np.sqrt(mc * (1 - mc) / m_pts) + 2e-3 * mc, (m, w[m], mc)


@pytest.mark.gpu
def test_neighbour_features_match_numpy():
    D, eps = 6, 0.05
    pts = sjoin.datasets.exponential(60_000, D, 40.0, 77)
    with sjoin.SelfJoin(D, eps, mode=10, precision=sjoin.PREC_FP32_REFINE) as sj:
        sj.set_points(pts)
        sj.build_index()
        feat, _, _ = sj.cell_features(with_hits=False)
    mn = pts.min(0) - eps
    nc = np.ceil((pts.max(0) + eps - mn) / eps).astype(np.int64)
    cc = ((pts - mn) / eps).astype(np.int64)
    mult = np.concatenate([[1], np.cumprod(nc)[:-1]])
    lid = (cc * mult).sum(1)
    ul, inv, occ = np.unique(lid, return_inverse=True, return_counts=True)
    assert len(ul) == len(feat)
    coords = np.zeros((len(ul), D), np.int64)
    coords[inv] = cc
    w = offset_class_weights(D)
    tot = np.zeros(len(ul))
    cls = np.zeros((len(ul), 3))
    for o in itertools.product([-1, 0, 1], repeat=D):
        o = np.array(o)
        m = int((o != 0).sum())
        if m == 0 or (o * mult).sum() < 0:   # home, or a neighbour with a smaller linear id
            continue
        nb = coords + o
        ok = np.all((nb >= 0) & (nb < nc), 1)
        nl = (nb * mult).sum(1)
        j = np.minimum(np.searchsorted(ul, nl), len(ul) - 1)
        v = np.where(ok & (ul[j] == nl), occ[j], 0) * w[m]
        tot += v
        if m <= 2:
            cls[:, m] += v
    np.testing.assert_allclose(feat[:, 0], np.log2(1.0 + occ), atol=1e-5)
    np.testing.assert_allclose(feat[:, 9], np.log2(1.0 + occ * tot), atol=1e-4, rtol=1e-5)
    np.testing.assert_allclose(feat[:, 13], np.log2(1.0 + occ * cls[:, 1]), atol=1e-4, rtol=1e-5)
    np.testing.assert_allclose(feat[:, 14], np.log2(1.0 + occ * cls[:, 2]), atol=1e-4, rtol=1e-5)

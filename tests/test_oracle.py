"""CPU oracle self-consistency: grid join vs brute force, predicate threshold, hashing."""
import math

import numpy as np
import pytest

import oracle
import sjoin
from conftest import exp_points, lattice_points, shell_points


def _pairset(k, v):
    return set(zip(k.tolist(), v.tolist()))


@pytest.mark.parametrize("n,d,k,eps,kind", [
    (1500, 2, 2, 0.03, "uniform"),
    (1500, 3, 3, 0.08, "uniform"),
    (1200, 5, 3, 0.15, "uniform"),
    (1500, 2, 2, 0.004, "exp"),
    (800, 6, 6, 0.06, "exp"),
    (600, 1, 1, 0.001, "uniform"),
])
def test_grid_join_equals_brute_force(n, d, k, eps, kind):
    pts = np.random.default_rng(n + d).random((n, d)) if kind == "uniform" else exp_points(n, d, n + d)
    ix = oracle.OracleIndex(pts, eps, k)
    gk, gv = ix.pairs()
    bk, bv = oracle.brute_pairs(pts, eps)
    assert np.array_equal(gk, bk) and np.array_equal(gv, bv)
    P, H, E = ix.stats()
    assert P == len(gk) and H == oracle.hash_pairs(gk, gv)
    assert E == int(ix.cell_candidates().sum())


def test_grid_join_subset_on_borderline_lattice():
    # pairs at distance ~eps may straddle a rounded cell boundary; the grid
    # restriction (shared with the reference) may only drop pairs, never add.
    pts = lattice_points(25, 2, 0.1)
    ix = oracle.OracleIndex(pts, 0.1, 2)
    g = _pairset(*ix.pairs())
    b = _pairset(*oracle.brute_pairs(pts, 0.1))
    assert g <= b
    assert len(g) >= 0.99 * len(b)


def test_symmetry_and_self_pairs():
    pts = exp_points(1000, 3, 7)
    ix = oracle.OracleIndex(pts, 0.02, 3)
    k, v = ix.pairs()
    s = _pairset(k, v)
    assert all((b, a) in s for a, b in s)
    assert all((i, i) in s for i in range(len(pts)))


def test_threshold_matches_sqrt_predicate():
    for eps in [0.01, 0.0015, 0.03, 0.05, 1e-7, 3.0, 0.1]:
        t = oracle.threshold(eps)
        assert math.sqrt(t) <= eps
        assert math.sqrt(np.nextafter(t, np.inf)) > eps


def test_fma_contraction_changes_borderline_pairs():
    # the golden fixtures can only discriminate the two predicate variants if
    # they differ on borderline data
    pts = shell_points(3000, 3, 0.05, 3)
    ix = oracle.OracleIndex(pts, 0.05, 3)
    a = _pairset(*ix.pairs(fma_mode=1))
    b = _pairset(*ix.pairs(fma_mode=0))
    assert a != b
    assert len(a ^ b) < 0.01 * len(a)


def test_python_hash_matches_oracle():
    pts = exp_points(700, 2, 11)
    ix = oracle.OracleIndex(pts, 0.01, 2)
    k, v = ix.pairs()
    assert sjoin.pair_hash(k, v) == oracle.hash_pairs(k, v)
    perm = np.random.default_rng(0).permutation(len(k))
    assert sjoin.pair_hash(k[perm], v[perm]) == oracle.hash_pairs(k, v)


def test_index_layout_invariants():
    pts = exp_points(3000, 3, 5)
    ix = oracle.OracleIndex(pts, 0.01, 3)
    ex = ix.export()
    lid = ex["gridLinearID"]
    g = ex["grid"]
    assert np.all(np.diff(lid.astype(np.float64)) > 0)
    assert g[0, 0] == 0 and g[-1, 1] == len(pts) - 1
    assert np.all(g[1:, 0] == g[:-1, 1] + 1)
    lookup = ex["indexLookupArr"]
    assert sorted(lookup.tolist()) == list(range(len(pts)))
    for c in range(len(g)):                       # ids ascend inside a cell
        seg = lookup[g[c, 0]:g[c, 1] + 1]
        assert np.all(np.diff(seg.astype(np.int64)) > 0)
    off = ex["gridCellNDMaskOffsets"]
    m = ex["gridCellNDMask"]
    for j in range(3):
        seg = m[off[2 * j]:off[2 * j + 1] + 1]
        assert np.all(np.diff(seg.astype(np.int64)) > 0)


def test_degrees_sum_to_pairs():
    pts = exp_points(2000, 2, 9)
    ix = oracle.OracleIndex(pts, 0.005, 2)
    deg = ix.degrees()
    k, _ = ix.pairs()
    assert int(deg.sum()) == len(k)
    assert np.array_equal(np.bincount(k, minlength=len(pts)), deg)


@pytest.mark.parametrize("n,d,k,eps,kind", [
    (3000, 2, 2, 0.02, "uniform"),
    (2000, 6, 6, 0.08, "exp"),
    (1500, 8, 4, 0.2, "uniform"),
])
def test_unicomp_stats_equal_full_stencil_stats(n, d, k, eps, kind):
    """The CPU baseline's linear-ID Unicomp join: over all points the same pair
    count and set hash as the full-stencil join, with about half its candidate
    evaluations (each unordered pair once, plus the diagonal)."""
    pts = np.random.default_rng(n + 7 * d).random((n, d)) if kind == "uniform" else exp_points(n, d, n + d)
    ix = oracle.OracleIndex(pts, eps, k)
    P, H, E = ix.stats()
    Pu, Hu, Eu = ix.stats(unicomp=True)
    assert (Pu, Hu) == (P, H)
    assert Eu == (E + n) // 2

"""GPU engine vs the CPU oracle at the benchmark configurations' own sizes.

The five configurations (2-D uniform n = 1e5; 2-D exponential n = 2e6; 4-D
exponential n = 5e6; 6-D exponential n = 1e7; 16-D Gaussian mixture n = 1e6
indexed on 6 dims) are checked at full size, each as far as the oracle
finishes in seconds:

  * c1, c5: the exact sorted pair list (c5 in both precisions, with the
    sampling and the learned estimator);
  * c2: every 1000th query's row of the on-device CSR neighbour table against
    the oracle's row (exact sorted values);
  * c3, c4: every 5000th query's degree (sj_degrees, the mixed-precision count
    pass) against the oracle's, and the mixed-precision join's pair count and
    set hash against the plain FP64 join's.

The predicate is the reference's (kernel.cu:344-349): emit (p, q) iff
sqrt(acc) <= eps, acc in the reference build's FP64 rounding order.
"""
import numpy as np
import pytest

import oracle
import sjoin

pytestmark = pytest.mark.gpu

WEIGHTS = sjoin.PKG + "/estimator_c4.bin"


def _make(name):
    pts, eps, k, spec = sjoin.datasets.make(name)
    return pts, eps, k, spec


def _join_pairs(pts, eps, k, spec, prec, learned=False):
    with sjoin.SelfJoin(spec["D"], eps, indexed_dims=k, mode=spec["mode"], precision=prec,
                        scheduler=sjoin.SCHED_LEARNED if learned else sjoin.SCHED_SAMPLING,
                        capacity=spec["capacity"]) as sj:
        if learned:
            sj.load_estimator(WEIGHTS)
        sj.set_points(pts)
        sj.build_index()
        ks, vs = [], []

        def cb(_i, key, val):
            assert np.all(np.diff(key.astype(np.int64)) >= 0)
            ks.append(key.copy())
            vs.append(val.copy())

        st = sj.join(sjoin.DELIVER_HOST, cb)
    key = np.concatenate(ks) if ks else np.zeros(0, np.int32)
    val = np.concatenate(vs) if vs else np.zeros(0, np.int32)
    assert st.total_pairs == len(key)
    return sjoin.canonical(key, val), st


def _oracle_all_rows(pts, eps, k):
    """Every query's sorted row as one canonical (key, value) list."""
    ix = oracle.OracleIndex(pts, eps, k)
    q = np.arange(len(pts), dtype=np.int64)
    deg, _, rows = ix.query_rows(q, values=True)
    key = np.repeat(q.astype(np.int32), deg.astype(np.int64))
    val = np.concatenate(rows) if len(rows) else np.zeros(0, np.int32)
    return key, val


def test_c1_full_size_exact_pairs():
    pts, eps, k, spec = _make("c1")
    ok, ov = oracle.OracleIndex(pts, eps, k).pairs()
    for prec in (sjoin.PREC_FP64, sjoin.PREC_FP32_REFINE):
        (key, val), st = _join_pairs(pts, eps, k, spec, prec)
        assert len(key) == len(ok) == 3_213_752
        assert np.array_equal(key, ok) and np.array_equal(val, ov)


def test_c5_full_size_exact_pairs_both_precisions_and_estimators():
    pts, eps, k, spec = _make("c5")
    ok, ov = _oracle_all_rows(pts, eps, k)
    assert len(ok) == 1_105_638
    for prec, learned in ((sjoin.PREC_FP64, False), (sjoin.PREC_FP32_REFINE, False),
                          (sjoin.PREC_FP32_REFINE, True)):
        (key, val), st = _join_pairs(pts, eps, k, spec, prec, learned)
        assert np.array_equal(key, ok) and np.array_equal(val, ov), (prec, learned)
        if prec == sjoin.PREC_FP32_REFINE:
            assert st.refined_pairs > 0


def test_c2_full_size_sampled_csr_rows():
    torch = pytest.importorskip("torch")
    pts, eps, k, spec = _make("c2")
    n = len(pts)
    with sjoin.SelfJoin(spec["D"], eps, indexed_dims=k, mode=spec["mode"], precision=0,
                        capacity=spec["capacity"]) as sj:
        sj.set_points(pts)
        sj.build_index()
        row = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
        total = sj.neighbor_csr(row.data_ptr())
        cols = torch.empty(total, dtype=torch.int32, device="cuda")
        assert sj.neighbor_csr(row.data_ptr(), cols.data_ptr(), total) == total
        st = sj.stats()
    assert total == st.total_pairs == 10_758_070_116
    q = np.arange(0, n, 1000, dtype=np.int64)
    rp = row.cpu().numpy()
    deg, hs, rows = oracle.OracleIndex(pts, eps, k).query_rows(q, values=True)
    assert np.array_equal(rp[q + 1] - rp[q], deg.astype(np.int64))
    lo, hi = torch.from_numpy(rp[q]), torch.from_numpy(rp[q + 1])
    for i in range(len(q)):
        got = np.sort(cols[int(lo[i]):int(hi[i])].cpu().numpy())
        assert np.array_equal(got, rows[i]), f"row of point {q[i]}"
    del cols


def _degrees_and_hash_check(name, stride):
    pts, eps, k, spec = _make(name)
    n = len(pts)
    q = np.arange(0, n, stride, dtype=np.int64)
    odeg, _ = oracle.OracleIndex(pts, eps, k).query_rows(q)
    learned = name == "c4"
    res = {}
    for prec in (sjoin.PREC_FP32_REFINE, sjoin.PREC_FP64):
        use_learned = learned and prec == sjoin.PREC_FP32_REFINE
        with sjoin.SelfJoin(spec["D"], eps, indexed_dims=k, mode=spec["mode"], precision=prec,
                            scheduler=sjoin.SCHED_LEARNED if use_learned else sjoin.SCHED_SAMPLING,
                            capacity=spec["capacity"]) as sj:
            if use_learned:
                sj.load_estimator(WEIGHTS)
            sj.set_points(pts)
            sj.build_index()
            if prec == sjoin.PREC_FP32_REFINE:
                deg = sj.degrees()
                assert np.array_equal(deg[q], odeg), f"{name}: sampled degrees differ from the oracle"
                dsum = int(deg.sum(dtype=np.uint64))
            st = sj.join(sjoin.DELIVER_NONE)
            res[prec] = (int(st.total_pairs), int(st.pair_hash))
    assert res[sjoin.PREC_FP32_REFINE][0] == dsum
    assert res[sjoin.PREC_FP32_REFINE] == res[sjoin.PREC_FP64], f"{name}: mixed and FP64 pair sets differ"
    return res


def test_c3_full_size_sampled_degrees_and_mixed_equals_fp64():
    res = _degrees_and_hash_check("c3", 5000)
    assert res[sjoin.PREC_FP64][0] == 115_473_826_618


def test_c4_full_size_sampled_degrees_and_mixed_equals_fp64():
    res = _degrees_and_hash_check("c4", 5000)
    assert res[sjoin.PREC_FP64][0] == 3_176_142_773_964

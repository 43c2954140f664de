"""GPU engine vs the CPU oracle: bit-exact pair sets for every traversal mode and precision."""
import os

import numpy as np
import pytest

import oracle
import sjoin
from conftest import exp_points, lattice_points, shell_points

pytestmark = pytest.mark.gpu


def _gauss16(n, seed):
    return sjoin.datasets.gaussian_mixture(n, 16, seed)


# name -> (points, eps, k)
def _cases():
    r = np.random.default_rng
    dup = np.repeat(r(3).random((5, 2)), 700, axis=0)          # five heavy cells, exact duplicates
    # far outlier in a non-indexed dimension: the FP32 filter's error band grows
    # with the data's extent there, so nearly every evaluation is refined in FP64
    outlier = r(11).random((3000, 5))
    outlier[17, 4] = 3.0e5
    return {
        "uniform2d": (r(1).random((20000, 2)), 0.01, 2),
        "exp2d_dense": (exp_points(30000, 2, 2), 0.002, 2),
        "uniform3d": (r(3).random((8000, 3)), 0.05, 3),
        "exp4d": (exp_points(10000, 4, 4), 0.02, 4),
        "exp6d": (exp_points(6000, 6, 6), 0.05, 6),
        "gauss16_k6": (_gauss16(4000, 5), 0.25, 6),
        "uniform5d_k3": (r(6).random((5000, 5)), 0.12, 3),
        "exp8d_k4": (exp_points(4000, 8, 9), 0.06, 4),          # padded width 8
        "uniform12d_k3": (r(10).random((3000, 12)) * 0.4, 0.3, 3),  # padded width 12
        "line1d": (r(7).random((5000, 1)), 0.0005, 1),
        "shell3d": (shell_points(3000, 3, 0.05, 8), 0.05, 3),
        "lattice2d": (lattice_points(60, 2, 0.1), 0.1, 2),
        "duplicates": (dup, 0.01, 2),
        "single": (np.array([[0.25, 0.5]]), 0.1, 2),
        # coordinates far from zero (FP32 ulp there exceeds eps / 10)
        "offset3d": (r(12).random((6000, 3)) * 0.5 + np.array([1.0e4, -2.5e4, 7.0e3]), 0.04, 3),
        "outlier5d_k2": (outlier, 0.15, 2),
    }


_ORACLE = {}


def _oracle_pairs(name):
    if name not in _ORACLE:
        pts, eps, k = _cases()[name]
        ix = oracle.OracleIndex(pts, eps, k)
        _ORACLE[name] = (pts, eps, k, ix, ix.pairs())
    return _ORACLE[name]


def _run(pts, eps, k, mode, prec, **kw):
    with sjoin.SelfJoin(pts.shape[1], eps, indexed_dims=k, mode=mode, precision=prec, **kw) as sj:
        sj.set_points(pts)
        sj.build_index()
        batches = []

        def cb(i, key, val):
            batches.append((key.copy(), val.copy()))

        st = sj.join(sjoin.DELIVER_HOST, cb)
        return batches, st


def _check_batches(batches, cap=None):
    for key, val in batches:
        assert np.all(np.diff(key.astype(np.int64)) >= 0), "keys must ascend inside a batch"
        if cap:
            assert len(key) <= cap


def _modes_for(k):
    return [3, 4, 5, 6, 7, 8, 9, 10] if k in (2, 3) else [3, 4, 6, 7, 8, 9, 10]


@pytest.mark.parametrize("name", sorted(_cases()))
@pytest.mark.parametrize("prec", [sjoin.PREC_FP64, sjoin.PREC_FP32_REFINE])
def test_all_modes_match_oracle(name, prec):
    pts, eps, k, ix, (ok, ov) = _oracle_pairs(name)
    for mode in _modes_for(k):
        batches, st = _run(pts, eps, k, mode, prec)
        _check_batches(batches)
        gk = np.concatenate([b[0] for b in batches]) if batches else np.zeros(0, np.int32)
        gv = np.concatenate([b[1] for b in batches]) if batches else np.zeros(0, np.int32)
        ck, cv = sjoin.canonical(gk, gv)
        assert len(ck) == len(ok), (name, mode, prec)
        assert np.array_equal(ck, ok) and np.array_equal(cv, ov), (name, mode, prec)
        assert st.total_pairs == len(ok)
        assert st.pair_hash == oracle.hash_pairs(ok, ov)
        assert st.full_stencil_calcs == int(ix.cell_candidates().sum())


@pytest.mark.parametrize("prec", [sjoin.PREC_FP64, sjoin.PREC_FP32_REFINE])
@pytest.mark.parametrize("mode", [3, 5, 6, 10])
def test_multi_batch_with_overflow_retries(mode, prec):
    pts, eps, k, ix, (ok, ov) = _oracle_pairs("exp2d_dense")
    cap = 65536
    # alpha 0 and a tiny sample make underestimates (and so retries) likely
    batches, st = _run(pts, eps, k, mode, prec, capacity=cap, alpha=0.0, sample_rate=0.002)
    _check_batches(batches, cap)
    assert len(batches) >= len(ok) // cap
    ck, cv = sjoin.canonical(np.concatenate([b[0] for b in batches]), np.concatenate([b[1] for b in batches]))
    assert np.array_equal(ck, ok) and np.array_equal(cv, ov)
    assert st.num_batches == len(batches)


@pytest.mark.parametrize("prec", [sjoin.PREC_FP64, sjoin.PREC_FP32_REFINE])
@pytest.mark.parametrize("mode", [5, 10])
def test_device_fold_pipeline_with_overflow_retries(mode, prec):
    # on-device delivery runs every batch back to back on two streams and
    # re-plans the batches whose count exceeds the buffer: an untrained
    # estimator network under-predicts by orders of magnitude, so batches
    # overflow for certain at this capacity
    pts, eps, k, ix, (ok, ov) = _oracle_pairs("exp2d_dense")
    with sjoin.SelfJoin(2, eps, mode=mode, precision=prec, capacity=65536, alpha=0.0,
                        scheduler=sjoin.SCHED_LEARNED) as sj:
        sj.set_estimator(sjoin.mlp_init(3))
        sj.set_points(pts)
        sj.build_index()
        st = sj.join(sjoin.DELIVER_NONE)
    assert st.num_batches >= 2 and st.overflow_retries > 0
    assert st.total_pairs == len(ok) and st.pair_hash == oracle.hash_pairs(ok, ov)


def test_mode8_splits_streams_by_thirds_of_the_work():
    # mode 8 (the reference's dynamic threads per point): each query tile's
    # candidate stream is shared by 16, 8 or 2 tasks by the third of the work
    # its cell falls in; mode 9 chunks streams by predicted pairs instead
    pts, eps, k, ix, (ok, ov) = _oracle_pairs("exp4d")
    st = {}
    for mode in (8, 9):
        with sjoin.SelfJoin(4, eps, mode=mode) as sj:
            sj.set_points(pts)
            sj.build_index()
            st[mode] = sj.join(sjoin.DELIVER_NONE)
    h = oracle.hash_pairs(ok, ov)
    for mode in (8, 9):
        assert st[mode].total_pairs == len(ok) and st[mode].pair_hash == h
    assert st[8].num_tasks > st[9].num_tasks


def test_full_stencil_batches_hold_complete_rows():
    # with the full stencil every key is produced by one task's query tile, and
    # the count pass places all of a key's values together
    pts, eps, k, ix, (ok, ov) = _oracle_pairs("uniform2d")
    batches, _ = _run(pts, eps, k, 3, sjoin.PREC_FP64, capacity=65536)
    seen = set()
    for key, val in batches:
        ks = set(np.unique(key).tolist())
        assert not (ks & seen)
        seen |= ks


def test_mixed_precision_refines_only_borderline():
    pts, eps, k, ix, (ok, ov) = _oracle_pairs("exp4d")
    _, st = _run(pts, eps, k, 10, sjoin.PREC_FP32_REFINE)
    assert 0 <= st.refined_pairs < 0.01 * st.distance_calcs
    _, st64 = _run(pts, eps, k, 10, sjoin.PREC_FP64)
    assert st64.refined_pairs == 0 and st.pair_hash == st64.pair_hash


@pytest.mark.parametrize("mode", [3, 6, 10])
def test_degrees_match_oracle(mode):
    pts, eps, k, ix, _ = _oracle_pairs("exp4d")
    with sjoin.SelfJoin(pts.shape[1], eps, indexed_dims=k, mode=mode) as sj:
        sj.set_points(pts)
        sj.build_index()
        assert np.array_equal(sj.degrees(), ix.degrees())


def test_neighbor_table_rows():
    pts, eps, k, ix, (ok, ov) = _oracle_pairs("exp2d_dense")
    with sjoin.SelfJoin(2, eps, mode=10, capacity=65536) as sj:
        sj.set_points(pts)
        sj.build_index()
        rows, vals = sj.neighbor_table()
    deg = ix.degrees()
    assert np.array_equal(rows[:, 1] - rows[:, 0] + 1, deg)
    starts = np.concatenate([[0], np.cumsum(deg)[:-1]])
    for p in np.random.default_rng(0).choice(len(pts), 300, replace=False):
        got = np.sort(vals[rows[p, 0]:rows[p, 1] + 1])
        s0 = int(starts[p])
        assert np.array_equal(got, ov[s0:s0 + int(deg[p])])


@pytest.mark.parametrize("name", ["exp4d", "gauss16_k6", "duplicates", "uniform5d_k3"])
def test_index_export_matches_oracle(name):
    pts, eps, k, ix, _ = _oracle_pairs(name)
    ref = ix.export()
    mn, nc = ix.grid()
    with sjoin.SelfJoin(pts.shape[1], eps, indexed_dims=k) as sj:
        sj.set_points(pts)
        sj.build_index()
        got = sj.index_export()
    assert np.array_equal(got["indexLookupArr"], ref["indexLookupArr"])
    assert np.array_equal(got["grid"], ref["grid"])
    assert np.array_equal(got["gridLinearID"], ref["gridLinearID"])
    assert np.array_equal(got["gridIdx"], np.arange(len(ref["grid"])))
    assert np.array_equal(got["minArr"].view(np.uint64), mn.view(np.uint64))
    assert np.array_equal(got["nCells"], nc)
    assert np.array_equal(got["gridCellNDMask"], ref["gridCellNDMask"])
    assert np.array_equal(got["gridCellNDMaskOffsets"], ref["gridCellNDMaskOffsets"])


def test_device_input_and_delivery():
    torch = pytest.importorskip("torch")
    pts, eps, k, ix, (ok, ov) = _oracle_pairs("uniform3d")
    t = torch.from_numpy(pts).cuda()
    counts = []
    with sjoin.SelfJoin(3, eps, mode=6) as sj:
        sj.set_points_device(t.data_ptr(), t.shape[0])
        sj.build_index()

        def cb(i, kptr, vptr, cnt):
            counts.append(int(cnt))

        st = sj.join(sjoin.DELIVER_DEVICE, cb)
    assert sum(counts) == len(ok) and st.pair_hash == oracle.hash_pairs(ok, ov)


def test_csv_import_path(tmp_path):
    pts, eps, k, ix, _ = _oracle_pairs("exp2d_dense")
    f = tmp_path / "d.csv"
    sjoin.datasets.write_csv(str(f), pts)
    imported = sjoin.read_csv(str(f), 2)          # the reference's point order
    ref = oracle.OracleIndex(imported, eps, 2)
    rk, rv = ref.pairs()
    with sjoin.SelfJoin(2, eps, mode=6) as sj:
        sj.import_csv(str(f))
        sj.build_index()
        st = sj.join(sjoin.DELIVER_NONE)
    assert st.total_pairs == len(rk) and st.pair_hash == oracle.hash_pairs(rk, rv)


def test_shards_partition_the_pairs():
    pts, eps, k, ix, (ok, ov) = _oracle_pairs("exp4d")
    total, h = 0, 0
    for s in range(3):
        with sjoin.SelfJoin(4, eps, mode=10, shard_index=s, shard_count=3) as sj:
            sj.set_points(pts)
            sj.build_index()
            st = sj.join(sjoin.DELIVER_NONE)
            total += st.total_pairs
            h = (h + st.pair_hash) % (1 << 64)
    assert total == len(ok) and h == oracle.hash_pairs(ok, ov)


def test_learned_scheduler_never_changes_pairs():
    pts, eps, k, ix, (ok, ov) = _oracle_pairs("exp6d")
    w = sjoin.mlp_init(3)
    with sjoin.SelfJoin(6, eps, mode=10, precision=sjoin.PREC_FP32_REFINE, scheduler=sjoin.SCHED_LEARNED,
                        capacity=200000) as sj:
        sj.set_estimator(w)
        sj.set_points(pts)
        sj.build_index()
        st = sj.join(sjoin.DELIVER_NONE)
    assert st.total_pairs == len(ok) and st.pair_hash == oracle.hash_pairs(ok, ov)


def test_bad_input_and_call_order():
    with sjoin.SelfJoin(2, 0.01) as sj:
        with pytest.raises(sjoin.SJError) as e:
            sj.join()
        assert e.value.status == sjoin.SJ_ERR_STATE
        with pytest.raises(sjoin.SJError) as e:
            sj.set_points(np.array([[0.1, np.nan], [0.2, 0.3]]))
            sj.build_index()
        assert e.value.status == sjoin.SJ_ERR_BAD_INPUT


@pytest.mark.parametrize("name,mode,prec", [("exp2d_dense", 5, 0), ("exp4d", 10, 1), ("gauss16_k6", 3, 1)])
def test_neighbor_csr_on_device(name, mode, prec):
    # the device CSR table holds exactly the oracle's rows, with several batches
    import torch
    pts, eps, k, ix, (ok, ov) = _oracle_pairs(name)
    n = len(pts)
    deg = np.bincount(ok, minlength=n)
    with sjoin.SelfJoin(pts.shape[1], eps, indexed_dims=k, mode=mode, precision=prec,
                        capacity=max(65536, len(ok) // 3)) as sj:
        sj.set_points(pts)
        sj.build_index()
        row_ptr = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
        total = sj.neighbor_csr(row_ptr.data_ptr())
        assert total == len(ok)
        assert np.array_equal(row_ptr.cpu().numpy(), np.concatenate([[0], np.cumsum(deg)]))
        with pytest.raises(sjoin.SJError):
            small = torch.empty(max(total - 1, 1), dtype=torch.int32, device="cuda")
            sj.neighbor_csr(row_ptr.data_ptr(), small.data_ptr(), max(total - 1, 1))
        with pytest.raises(sjoin.SJError) as e:   # host memory is refused before any kernel runs
            host_cols = np.zeros(total, np.int32)
            sj.neighbor_csr(row_ptr.data_ptr(), host_cols.ctypes.data, total)
        assert e.value.status == sjoin.SJ_ERR_BAD_INPUT
        cols = torch.full((total,), -1, dtype=torch.int32, device="cuda")
        assert sj.neighbor_csr(row_ptr.data_ptr(), cols.data_ptr(), total) == total
        st = sj.stats()
    v = cols.cpu().numpy()
    keys = np.repeat(np.arange(n, dtype=np.int32), deg)
    order = np.lexsort((v, keys))
    assert np.array_equal(v[order], ov)
    assert st.num_batches >= 2 or len(ok) < 65536

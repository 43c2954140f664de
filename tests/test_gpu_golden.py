"""GPU engine vs the reference's own outputs (golden fixtures), with no oracle in between.

Each fixture in tests/golden/ holds the points in the reference's id order, the
pair set of the reference's full-stencil kernel (mode 3) as per-key degrees +
values, and the count and set hash of its other modes (made by
tests/golden/make_golden.py from the reference built by oracle/build_ref.py).
Every traversal mode of the engine, in both precisions, must emit exactly the
mode-3 set: sorted (key, value) lists compared element by element.
"""
import glob
import os

import numpy as np
import pytest

import sjoin

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def _load(path):
    d = np.load(path)
    return {k: d[k] for k in d.files}


def _join(pts, eps, k, mode, prec, capacity=0):
    with sjoin.SelfJoin(pts.shape[1], eps, indexed_dims=k, mode=mode, precision=prec, capacity=capacity) as sj:
        sj.set_points(pts)
        sj.build_index()
        ks, vs = [], []

        def take(i, kk, vv):
            ks.append(kk.copy())
            vs.append(vv.copy())

        st = sj.join(sjoin.DELIVER_HOST, take)
    key = np.concatenate(ks) if ks else np.zeros(0, np.int32)
    val = np.concatenate(vs) if vs else np.zeros(0, np.int32)
    order = np.lexsort((val, key))
    return key[order], val[order], st


@pytest.mark.parametrize("prec", [sjoin.PREC_FP64, sjoin.PREC_FP32_REFINE])
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_engine_matches_reference_pairs(path, prec):
    f = _load(path)
    pts, eps, k = f["pts"], float(f["eps"]), int(f["k"])
    ref_key = np.repeat(np.arange(len(pts), dtype=np.int32), f["deg"])
    ref_val = f["val"]
    modes = [3, 4, 5, 6, 7, 8, 9, 10] if k in (2, 3) else [3, 4, 6, 7, 8, 9, 10]
    for mode in modes:
        key, val, st = _join(pts, eps, k, mode, prec)
        assert st.total_pairs == len(ref_key), (mode, st.total_pairs, len(ref_key))
        assert np.array_equal(key, ref_key), f"mode {mode}: keys differ from the reference"
        assert np.array_equal(val, ref_val), f"mode {mode}: values differ from the reference"
        assert st.pair_hash == int(f["mode3_hash"])


@pytest.mark.parametrize("mode", [3, 6, 10])
@pytest.mark.parametrize("prec", [sjoin.PREC_FP64, sjoin.PREC_FP32_REFINE])
def test_engine_matches_reference_in_several_batches(mode, prec):
    # the smallest batch capacity the engine accepts (65536 pairs) splits the
    # largest fixture (72,448 pairs) into at least two batches
    f = _load(os.path.join(HERE, "golden", "exp4d.npz"))
    pts, eps, k = f["pts"], float(f["eps"]), int(f["k"])
    ref_key = np.repeat(np.arange(len(pts), dtype=np.int32), f["deg"])
    key, val, st = _join(pts, eps, k, mode, prec, capacity=65536)
    assert st.num_batches >= 2
    assert np.array_equal(key, ref_key) and np.array_equal(val, f["val"])

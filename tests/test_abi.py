"""The C ABI library: loads, exports every declared symbol, validates input without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import sjoin
from conftest import REPO, has_gpu


def _declared():
    text = open(os.path.join(REPO, "include", "sj.h")).read()
    return sorted(set(re.findall(r"^\s*(?:sj_status|void|uint32_t|uint64_t|const char \*)\s*\*?\s*(sj_[a-z0-9_]+)\s*\(",
                                 text, re.M)))


def test_library_exports_every_declared_symbol():
    L = sjoin.load()
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(sjoin.EXPORTS)


def test_params_default_follow_params_h():
    L = sjoin.load()
    p = sjoin.Params()
    L.sj_params_default(C.byref(p))
    assert p.blocksize == 256 and p.threadperpoint == 1 and p.sort_by_workload == 1
    assert p.gpunumdim == 2 and p.numindexeddim == 2
    assert abs(p.sample_rate - 0.01) < 1e-12 and abs(p.alpha - 0.05) < 1e-12
    assert p.shard_count == 1


@pytest.mark.parametrize("field,value", [
    ("gpunumdim", 0), ("gpunumdim", 17), ("numindexeddim", 3), ("epsilon", 0.0), ("epsilon", float("nan")),
    ("search_mode", 11), ("search_mode", 2), ("precision", 5), ("scheduler", 9), ("sample_rate", 0.0),
    ("shard_count", 0), ("batch_capacity_pairs", 1000),
])
def test_bad_params_rejected_before_device(field, value):
    L = sjoin.load()
    p = sjoin.Params()
    L.sj_params_default(C.byref(p))
    setattr(p, field, value)
    h = C.c_void_p()
    st = L.sj_create(C.byref(p), C.byref(h))
    assert st == sjoin.SJ_ERR_BAD_INPUT
    assert L.sj_last_error()


def test_bunicomp_needs_two_or_three_indexed_dims():
    L = sjoin.load()
    p = sjoin.Params()
    L.sj_params_default(C.byref(p))
    p.gpunumdim, p.numindexeddim, p.search_mode = 4, 4, 5
    assert L.sj_create(C.byref(p), C.byref(C.c_void_p())) == sjoin.SJ_ERR_BAD_INPUT


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly():
    with pytest.raises(sjoin.SJError) as e:
        sjoin.SelfJoin(2, 0.01)
    assert e.value.status == sjoin.SJ_ERR_CUDA


def test_status_strings_and_version():
    L = sjoin.load()
    assert L.sj_version().startswith(b"sj-b200")
    for s in range(10):
        assert L.sj_status_string(s)


def test_read_csv_values_roundtrip(tmp_path):
    # the reference's bin sort (an unstable std::sort) reorders rows once n > 16;
    # values must survive the text round trip exactly
    pts = np.random.default_rng(1).random((257, 3))
    f = tmp_path / "d.csv"
    sjoin.datasets.write_csv(str(f), pts)
    got = sjoin.read_csv(str(f), 3)
    key = lambda a: a[np.lexsort(a.T[::-1])]
    assert np.array_equal(key(got), key(pts))
    small = pts[:16]
    sjoin.datasets.write_csv(str(f), small)
    assert np.array_equal(sjoin.read_csv(str(f), 3), small)


def test_read_csv_missing_file():
    with pytest.raises(sjoin.SJError) as e:
        sjoin.read_csv("/nonexistent/x.csv", 2)
    assert e.value.status == sjoin.SJ_ERR_IO

"""The dataset import matches the reference's own importNDDataset + sortInNDBins.

The reference's import_dataset.cpp is compiled by oracle/build_ref.py into a
CPU-only binary (oracle/_ref/ref_import_D{D}); these tests run it here and
compare point order and values bit for bit with sj_read_csv.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

import sjoin
from oracle import build_ref


def _ref_import(path, d):
    exe = build_ref.binary("import", d, d)
    if not os.path.exists(exe):
        pytest.skip("reference import binary not built (reference sources absent)")
    out = path + ".bin"
    subprocess.check_call([exe, path, out], stdout=subprocess.DEVNULL)
    raw = open(out, "rb").read()
    n = struct.unpack("<Q", raw[:8])[0]
    return np.frombuffer(raw[8:], dtype=np.float64).reshape(n, d)


CASES = {
    "plain": "0.5,0.25\n0.125,0.75\n0.3,0.9\n",
    "spaces": " 0.5 , 0.25 \n\t0.125,0.75\r\n0.3,   0.9",
    "newline_only": "0.5\n0.25\n0.125\n0.75\n",
    "partial_last": "0.5,0.25\n0.125,0.75\n0.3\n",
    "exponents": "1e-3,2.5E-2\n-1.5e+0,3.\n.5,-.25\n",
    "bins": "1.5,0.2\n0.3,2.7\n-0.5,0.1\n2.0,2.0\n0.9,0.9\n1.0,0.0\n",
    "bad_token": "0.5,abc\n0.25,0.75\n0.1x,0.2\n0.3,0.4\n",
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_import_matches_reference(tmp_path, name):
    f = tmp_path / f"{name}.csv"
    f.write_text(CASES[name])
    ref = _ref_import(str(f), 2)
    got = sjoin.read_csv(str(f), 2)
    assert got.shape == ref.shape
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))


@pytest.mark.parametrize("d,seed", [(2, 1), (5, 2)])
def test_import_bin_sort_permutation_matches_reference(tmp_path, d, seed):
    # coordinates >= 1 give non-zero int() bins, so the reference's unstable
    # std::sort permutes the points; the ids must follow the same permutation
    pts = np.random.default_rng(seed).normal(0.5, 0.6, (3000, d))
    f = tmp_path / "mix.csv"
    sjoin.datasets.write_csv(str(f), pts)
    ref = _ref_import(str(f), d)
    got = sjoin.read_csv(str(f), d)
    assert not np.array_equal(ref, pts)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("n", [10, 16, 17, 5000])
def test_import_order_for_unit_cube_data(tmp_path, n):
    # every bin key is 0 for [0,1) data, yet std::sort's introsort still moves
    # rows once n > 16 (its insertion-sort cutoff); ids follow the reference
    pts = sjoin.datasets.exponential(n, 2, 40.0, 3)
    f = tmp_path / "exp.csv"
    sjoin.datasets.write_csv(str(f), pts)
    ref = _ref_import(str(f), 2)
    assert np.array_equal(sjoin.read_csv(str(f), 2), ref)
    assert np.array_equal(ref, pts) == (n <= 16)


def test_import_parallel_ranges_match_reference(tmp_path):
    # a file of several MB is parsed in one range per thread, cut after commas;
    # the concatenated values and the replayed bin sort must still equal the
    # reference's own import (mixed spacing and a trailing partial point)
    rng = np.random.default_rng(9)
    pts = rng.normal(0.5, 0.7, (250_000, 3))
    lines = [f"{a!r}, {b!r},{c!r}" if i % 7 else f" {a!r} ,\t{b!r} , {c!r} "
             for i, (a, b, c) in enumerate(pts.tolist())]
    f = tmp_path / "big.csv"
    f.write_text("\n".join(lines) + "\n0.25,0.5\n")
    assert os.path.getsize(f) > 4 << 20
    ref = _ref_import(str(f), 3)
    got = sjoin.read_csv(str(f), 3)
    assert got.shape == ref.shape == (250_000, 3)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))

"""Generates the golden fixtures from the reference itself (run on a GPU machine).

For each small seeded case this writes the dataset as CSV, runs the reference's
own import (oracle/_ref/ref_import_D*) to get its point order, then runs the
reference's own join kernels (oracle/_ref/ref_dump_*_hd; modes 3 full stencil,
4 Unicomp, 5 B-Unicomp, 6 linear-ID Unicomp, single batch, SORT_BY_WORKLOAD 0;
the _hd build is the reference with its cell comparison operator made callable
on the device, see oracle/build_ref.py)
and stores, per case, an .npz with
    pts      the points in the reference's id order (float64)
    eps, k   search radius and indexed dimensions
    deg, val the mode-3 pair set in CSR form (neighbour count per key, then the
             sorted neighbour ids of key 0, 1, ...)
    mode{m}_count, mode{m}_hash  pair count and set hash of every mode's raw output
The cases lean on borderline distances (points on shells of radius eps and on
lattices of pitch eps) so that the fixtures pin the FP64 predicate, including
nvcc's fused multiply-add contraction of the distance accumulation.

usage: python tests/golden/make_golden.py [out_dir]     (default: tests/golden)
"""
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "self-join-hpbdc2019_b200"))

from oracle import build_ref  # noqa: E402
from sjoin import datasets, pair_hash  # noqa: E402


def shell(n, d, eps, seed):
    rng = np.random.default_rng(seed)
    base = rng.random((n, d))
    u = rng.standard_normal((n, d))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    return np.vstack([base, base + eps * u])


def lattice(m, d, step):
    g = np.stack(np.meshgrid(*([np.arange(m) * step] * d), indexing="ij"), -1).reshape(-1, d)
    return g.astype(np.float64)


# name -> (points, eps, D, k, modes)
CASES = {
    "uni2d": (lambda: np.random.default_rng(11).random((3000, 2)), 0.02, 2, 2, [3, 4, 5, 6]),
    "exp2d": (lambda: datasets.exponential(3000, 2, 40.0, 12), 0.002, 2, 2, [3, 4, 5, 6]),
    "shell2d": (lambda: shell(8000, 2, 0.005, 13), 0.005, 2, 2, [3, 5, 6]),
    "lattice2d": (lambda: lattice(45, 2, 0.1), 0.1, 2, 2, [3, 5, 6]),
    "shell3d": (lambda: shell(6000, 3, 0.03, 14), 0.03, 3, 3, [3, 4, 5, 6]),
    "exp4d": (lambda: datasets.exponential(3000, 4, 40.0, 15), 0.012, 4, 4, [3, 4, 6]),
    "shell6d": (lambda: shell(3000, 6, 0.1, 16), 0.1, 6, 6, [3, 6]),
    "gauss16": (lambda: datasets.gaussian_mixture(2000, 16, 17), 0.3, 16, 6, [3, 6]),
    "uni5d_k3": (lambda: np.random.default_rng(18).random((2000, 5)), 0.12, 5, 3, [3, 5, 6]),
    "shell4d": (lambda: shell(4000, 4, 0.05, 19), 0.05, 4, 4, [3, 6]),
    "shell5d_k3": (lambda: shell(4000, 5, 0.08, 20), 0.08, 5, 3, [3, 5, 6]),
    "shell16d_k6": (lambda: shell(3000, 16, 0.3, 21), 0.3, 16, 6, [3, 6]),
}


def run_case(name, out_dir, tmp):
    make, eps, D, k, modes = CASES[name]
    pts = make()
    csv = os.path.join(tmp, f"{name}.csv")
    datasets.write_csv(csv, pts)
    imp = build_ref.binary("import", D, k)
    subprocess.check_call([imp, csv, csv + ".imp"], stdout=subprocess.DEVNULL)
    raw = open(csv + ".imp", "rb").read()
    n = struct.unpack("<Q", raw[:8])[0]
    ref_pts = np.frombuffer(raw[8:], np.float64).reshape(n, D).copy()
    rec = dict(pts=ref_pts, eps=np.float64(eps), k=np.int64(k))
    if D == 2 and k == 2:
        # the reference exactly as shipped: record what it emits (zero pairs
        # with nvcc 12.9, its device cell lookups never match)
        exe = build_ref.binary("dump", D, k, 0, variant="")
        out = os.path.join(tmp, f"{name}_asis.bin")
        subprocess.check_call([exe, csv, repr(eps), "3", out], stdout=subprocess.DEVNULL)
        rec["asis_mode3_count"] = np.int64(struct.unpack("<Q", open(out, "rb").read()[:8])[0])
    for m in modes:
        exe = build_ref.binary("dump", D, k, 0)
        out = os.path.join(tmp, f"{name}_{m}.bin")
        subprocess.check_call([exe, csv, repr(eps), str(m), out], stdout=subprocess.DEVNULL)
        b = open(out, "rb").read()
        cnt = struct.unpack("<Q", b[:8])[0]
        keys = np.frombuffer(b[8:8 + 4 * cnt], np.int32)
        vals = np.frombuffer(b[8 + 4 * cnt:8 + 8 * cnt], np.int32)
        rec[f"mode{m}_count"] = np.int64(cnt)
        rec[f"mode{m}_hash"] = np.uint64(pair_hash(keys, vals))
        if m == 3:
            o = np.lexsort((vals, keys))
            k_, v_ = keys[o], vals[o]
            rec["deg"] = np.bincount(k_, minlength=n).astype(np.int32)
            rec["val"] = v_.astype(np.int32)
    path = os.path.join(out_dir, f"{name}.npz")
    np.savez_compressed(path, **rec)
    return path, {m: int(rec[f"mode{m}_count"]) for m in modes}


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out_dir, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        for name in CASES:
            path, counts = run_case(name, out_dir, tmp)
            print(name, os.path.getsize(path), counts, flush=True)


if __name__ == "__main__":
    main()

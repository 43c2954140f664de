"""CPU oracle for the epsilon self-join (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
bench.py import this package, and only as the checker.  The product library
never routes through it.

``liboracle.so`` is built from ``sj_oracle.c`` (a C restatement of the
reference's host grid build, candidate stencil and FP64 predicate; see the
header of that file for the file:line map into the reference project).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so (gcc, OpenMP, no FP contraction)."""
    src = os.path.join(HERE, "sj_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(
            ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
             "-std=c11", "-o", LIB_PATH, src, "-lm"])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        vp, i64, u64p = C.c_void_p, C.c_int64, C.POINTER(C.c_uint64)
        L.orc_index_build.restype = vp
        L.orc_index_build.argtypes = [vp, i64, C.c_int, C.c_int, C.c_double]
        L.orc_index_free.argtypes = [vp]
        L.orc_index_sizes.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), u64p]
        L.orc_index_grid.argtypes = [vp, vp, vp]
        L.orc_index_export.argtypes = [vp, vp, vp, vp, vp, vp]
        L.orc_join_stats.argtypes = [vp, C.c_int, i64, i64, i64, C.c_int, u64p, u64p, u64p]
        L.orc_join_stats_unicomp.argtypes = [vp, C.c_int, i64, i64, i64, C.c_int, u64p, u64p, u64p]
        L.orc_join_degrees.argtypes = [vp, C.c_int, C.c_int, vp]
        L.orc_query_rows.argtypes = [vp, C.c_int, vp, i64, C.c_int, vp, vp, vp, vp, i64]
        L.orc_join_pairs.restype = i64
        L.orc_join_pairs.argtypes = [vp, C.c_int, vp, vp, i64]
        L.orc_brute_pairs.restype = i64
        L.orc_brute_pairs.argtypes = [vp, i64, C.c_int, C.c_double, C.c_int, vp, vp, i64]
        L.orc_threshold.restype = C.c_double
        L.orc_threshold.argtypes = [C.c_double]
        L.orc_pair_hash.restype = C.c_uint64
        L.orc_pair_hash.argtypes = [C.c_int32, C.c_int32]
        L.orc_hash_pairs.restype = C.c_uint64
        L.orc_hash_pairs.argtypes = [vp, vp, i64]
        L.orc_cell_candidates.argtypes = [vp, vp]
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def threshold(eps: float) -> float:
    """Largest T with sqrt(T) <= eps (round-to-nearest)."""
    return lib().orc_threshold(float(eps))


def hash_pairs(keys: np.ndarray, vals: np.ndarray) -> int:
    k = np.ascontiguousarray(keys, dtype=np.int32)
    v = np.ascontiguousarray(vals, dtype=np.int32)
    return int(lib().orc_hash_pairs(_ptr(k), _ptr(v), len(k)))


def num_threads() -> int:
    return int(lib().orc_num_threads())


class OracleIndex:
    """Grid index over an (n, D) float64 point array, indexed on the first k dims."""

    def __init__(self, pts: np.ndarray, eps: float, k: int):
        self.pts = np.ascontiguousarray(pts, dtype=np.float64)
        self.n, self.D = self.pts.shape
        self.k = int(k)
        self.eps = float(eps)
        self._h = lib().orc_index_build(_ptr(self.pts), self.n, self.D, self.k, self.eps)
        if not self._h:
            raise ValueError("oracle index build rejected the input")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_index_free(h)
            self._h = None

    def sizes(self):
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint64()
        lib().orc_index_sizes(self._h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def grid(self):
        mn = np.zeros(self.k, np.float64)
        nc = np.zeros(self.k, np.uint32)
        lib().orc_index_grid(self._h, _ptr(mn), _ptr(nc))
        return mn, nc

    def export(self):
        nne, nmask, _ = self.sizes()
        lookup = np.zeros(self.n, np.uint32)
        grid = np.zeros((nne, 2), np.int32)
        lid = np.zeros(nne, np.uint64)
        mask = np.zeros(max(nmask, 1), np.uint32)
        moff = np.zeros(2 * self.k, np.uint32)
        lib().orc_index_export(self._h, _ptr(lookup), _ptr(grid), _ptr(lid), _ptr(mask), _ptr(moff))
        return dict(indexLookupArr=lookup, grid=grid, gridLinearID=lid,
                    gridCellNDMask=mask[:nmask], gridCellNDMaskOffsets=moff)

    def stats(self, fma_mode=1, q0=0, q1=None, qstride=1, threads=0, unicomp=False):
        """(pair count, set hash, candidate evaluations) for sampled query ids.
        unicomp=True: each sampled point evaluates only the candidates it owns
        under the linear-ID Unicomp rule and counts both directions of a hit
        (over all points: the same pairs and hash, half the evaluations)."""
        P, H, E = C.c_uint64(), C.c_uint64(), C.c_uint64()
        q1 = self.n if q1 is None else q1
        fn = lib().orc_join_stats_unicomp if unicomp else lib().orc_join_stats
        fn(self._h, fma_mode, q0, q1, qstride, threads, C.byref(P), C.byref(H), C.byref(E))
        return P.value, H.value, E.value

    def degrees(self, fma_mode=1, threads=0) -> np.ndarray:
        deg = np.zeros(self.n, np.uint32)
        lib().orc_join_degrees(self._h, fma_mode, threads, _ptr(deg))
        return deg

    def query_rows(self, qids, fma_mode=1, threads=0, values=False):
        """Neighbour-table rows of the query ids `qids`: (degrees uint32, row set
        hashes uint64) and, with values=True, the rows' values as a list of
        sorted int32 arrays."""
        q = np.ascontiguousarray(qids, dtype=np.int64)
        deg = np.zeros(len(q), np.uint32)
        hs = np.zeros(len(q), np.uint64)
        lib().orc_query_rows(self._h, fma_mode, _ptr(q), len(q), threads, _ptr(deg), _ptr(hs), None, None, 0)
        if not values:
            return deg, hs
        off = np.zeros(len(q) + 1, np.int64)
        off[1:] = np.cumsum(deg, dtype=np.int64)
        vals = np.zeros(max(int(off[-1]), 1), np.int32)
        deg2 = np.zeros(len(q), np.uint32)
        r = lib().orc_query_rows(self._h, fma_mode, _ptr(q), len(q), threads, _ptr(deg2), None, _ptr(off),
                                 _ptr(vals), len(vals))
        assert r == 0 and np.array_equal(deg, deg2)
        return deg, hs, [np.sort(vals[off[i]:off[i + 1]]) for i in range(len(q))]

    def pairs(self, fma_mode=1):
        """All pairs sorted by (key, value) as two int32 arrays."""
        m = lib().orc_join_pairs(self._h, fma_mode, None, None, 0)
        keys = np.zeros(max(m, 1), np.int32)
        vals = np.zeros(max(m, 1), np.int32)
        r = lib().orc_join_pairs(self._h, fma_mode, _ptr(keys), _ptr(vals), m)
        assert r == m
        return keys[:m], vals[:m]

    def cell_candidates(self) -> np.ndarray:
        nne, _, _ = self.sizes()
        out = np.zeros(nne, np.uint64)
        lib().orc_cell_candidates(self._h, _ptr(out))
        return out


def brute_pairs(pts: np.ndarray, eps: float, fma_mode=1):
    """O(n^2) pairs with the reference predicate and no grid restriction."""
    p = np.ascontiguousarray(pts, dtype=np.float64)
    n, D = p.shape
    m = lib().orc_brute_pairs(_ptr(p), n, D, float(eps), fma_mode, None, None, 0)
    keys = np.zeros(max(m, 1), np.int32)
    vals = np.zeros(max(m, 1), np.int32)
    lib().orc_brute_pairs(_ptr(p), n, D, float(eps), fma_mode, _ptr(keys), _ptr(vals), m)
    return keys[:m], vals[:m]

"""Python mirror of the self-join engine's C ABI (include/sj.h), over ctypes.

The reference drives its GPU join from C++ (main.cu -> distanceTableNDGridBatches,
GPU.h:37-40).  This module exposes the same steps -- import / set points, build
the grid index, run the batched join, read the neighbour table -- through
``libsj.so``.  There is no CPU fallback: if the library or a CUDA device is
missing, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Callable, Optional

import numpy as np

from . import datasets  # noqa: F401  (re-exported)

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libsj.so")

SJ_OK, SJ_ERR_OOM, SJ_OVERFLOW_RETRIED, SJ_ERR_BAD_INPUT, SJ_ERR_CUDA = 0, 1, 2, 3, 4
SJ_ERR_TIMEOUT, SJ_ERR_STATE, SJ_ERR_IO, SJ_ERR_ABORTED, SJ_ERR_INTERNAL = 5, 6, 7, 8, 9
PREC_FP64, PREC_FP32_REFINE = 0, 1
SCHED_SAMPLING, SCHED_LEARNED = 0, 1
DELIVER_DEVICE, DELIVER_HOST, DELIVER_NONE = 0, 1, 2

# Symbols declared in include/sj.h (checked by the tests against the library).
EXPORTS = [
    "sj_params_default", "sj_create", "sj_destroy", "sj_import_csv", "sj_read_csv", "sj_set_points", "sj_build_index",
    "sj_index_sizes", "sj_index_export", "sj_join", "sj_degrees", "sj_neighbor_table", "sj_neighbor_csr", "sj_free",
    "sj_get_stats", "sj_get_stream", "sj_mlp_num_params", "sj_set_estimator_weights", "sj_load_estimator",
    "sj_cell_features", "sj_cell_samples", "sj_mlp_train", "sj_mlp_loss_grad", "sj_mlp_forward", "sj_mlp_loss_grad_noalloc",
    "sj_status_string",
    "sj_last_error", "sj_version", "sj_kernel_launch_count",
]


class Params(C.Structure):
    _fields_ = [
        ("gpunumdim", C.c_int), ("numindexeddim", C.c_int), ("epsilon", C.c_double),
        ("blocksize", C.c_int), ("threadperpoint", C.c_int), ("search_mode", C.c_int),
        ("sort_by_workload", C.c_int), ("precision", C.c_int), ("scheduler", C.c_int),
        ("batch_capacity_pairs", C.c_uint64), ("sample_rate", C.c_double), ("alpha", C.c_double),
        ("device", C.c_int), ("shard_index", C.c_int), ("shard_count", C.c_int), ("verbose", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("total_pairs", C.c_uint64), ("pair_hash", C.c_uint64), ("distance_calcs", C.c_uint64),
        ("full_stencil_calcs", C.c_uint64), ("refined_pairs", C.c_uint64), ("num_batches", C.c_uint64),
        ("overflow_retries", C.c_uint64), ("num_tasks", C.c_uint64), ("total_cells", C.c_uint64),
        ("n_points", C.c_uint32), ("n_nonempty_cells", C.c_uint32),
        ("estimated_pairs", C.c_double), ("estimator_mean_abs_rel_err", C.c_double),
        ("estimator_task_rel_err", C.c_double),
        ("ms_upload", C.c_float), ("ms_index", C.c_float), ("ms_tasks", C.c_float), ("ms_estimate", C.c_float),
        ("ms_count", C.c_float), ("ms_scan", C.c_float), ("ms_fill", C.c_float), ("ms_deliver", C.c_float),
        ("ms_total", C.c_float), ("ms_join_kernels", C.c_float), ("ms_fill_kernel", C.c_float),
        ("kernel_launches", C.c_uint64), ("ms_expand", C.c_float), ("exact_plan_batches", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class Batch(C.Structure):
    _fields_ = [("batch_index", C.c_uint64), ("count", C.c_uint64), ("key", C.c_void_p),
                ("val", C.c_void_p), ("on_device", C.c_int)]


class GridCell(C.Structure):
    _fields_ = [("indexmin", C.c_int), ("indexmax", C.c_int)]


class GridCellLookup(C.Structure):
    _fields_ = [("idx", C.c_uint), ("gridLinearID", C.c_uint64)]


class NeighborTableLookup(C.Structure):
    _fields_ = [("pointID", C.c_int), ("indexmin", C.c_int), ("indexmax", C.c_int),
                ("dataPtr", C.POINTER(C.c_int))]


BATCH_CB = C.CFUNCTYPE(C.c_int, C.POINTER(Batch), C.c_void_p)

_lib = None


class SJError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"sj status {status}: {msg}")
        self.status = status


def load() -> C.CDLL:
    """Loads libsj.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} missing: build it with `python -m sjoin.build`")
    L = C.CDLL(LIB_PATH)
    vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
    L.sj_params_default.argtypes = [C.POINTER(Params)]
    L.sj_params_default.restype = None
    L.sj_create.argtypes = [C.POINTER(Params), C.POINTER(vp)]
    L.sj_destroy.argtypes = [vp]
    L.sj_import_csv.argtypes = [vp, C.c_char_p]
    L.sj_set_points.argtypes = [vp, vp, u64, i32]
    L.sj_read_csv.argtypes = [C.c_char_p, i32, vp, u64, C.POINTER(u64)]
    L.sj_build_index.argtypes = [vp]
    L.sj_index_sizes.argtypes = [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u64)]
    L.sj_index_export.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    L.sj_join.argtypes = [vp, i32, BATCH_CB, vp]
    L.sj_degrees.argtypes = [vp, vp]
    L.sj_neighbor_table.argtypes = [vp, vp, C.POINTER(C.POINTER(C.c_int)), C.POINTER(u64)]
    L.sj_neighbor_csr.argtypes = [vp, vp, vp, u64, C.POINTER(u64)]
    L.sj_free.argtypes = [vp]
    L.sj_free.restype = None
    L.sj_get_stats.argtypes = [vp, C.POINTER(Stats)]
    L.sj_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.sj_mlp_num_params.restype = u32
    L.sj_set_estimator_weights.argtypes = [vp, vp, u32]
    L.sj_load_estimator.argtypes = [vp, C.c_char_p]
    L.sj_cell_features.argtypes = [vp, vp, vp, vp]
    L.sj_cell_samples.argtypes = [vp, vp, vp, vp, vp]
    L.sj_mlp_train.argtypes = [vp, vp, u32, vp, i32, C.c_float, u32, u64, C.POINTER(C.c_float), i32]
    L.sj_mlp_loss_grad.argtypes = [vp, vp, u32, vp, C.POINTER(C.c_float), vp, i32]
    L.sj_mlp_forward.argtypes = [vp, u32, vp, vp, i32]
    L.sj_mlp_loss_grad_noalloc.argtypes = [vp, vp, u32, vp, vp, vp, vp]
    L.sj_status_string.restype = C.c_char_p
    L.sj_status_string.argtypes = [i32]
    L.sj_last_error.restype = C.c_char_p
    L.sj_version.restype = C.c_char_p
    L.sj_kernel_launch_count.restype = C.c_uint64
    for name in EXPORTS:
        if not hasattr(L, name):
            raise RuntimeError(f"libsj.so lacks {name}")
    _lib = L
    return L


def _check(st: int):
    if st != SJ_OK:
        L = load()
        raise SJError(st, f"{L.sj_status_string(st).decode()}: {L.sj_last_error().decode()}")


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def read_csv(path: str, dim: int) -> np.ndarray:
    """Parses a dataset file with the reference's rules and point order (no device needed)."""
    L = load()
    n = C.c_uint64()
    _check(L.sj_read_csv(path.encode(), int(dim), None, 0, C.byref(n)))
    out = np.zeros((n.value, dim), np.float64)
    _check(L.sj_read_csv(path.encode(), int(dim), _ptr(out), n.value, C.byref(n)))
    return out


def kernel_launch_count() -> int:
    """Kernels libsj has launched since it was loaded."""
    return int(load().sj_kernel_launch_count())


def mlp_num_params() -> int:
    return int(load().sj_mlp_num_params())


MODE_NAMES = {3: "full stencil", 4: "Unicomp", 5: "B-Unicomp", 6: "linear-ID Unicomp",
              7: "full stencil, workload order", 8: "full stencil, work split by workload", 9: "work queue",
              10: "work queue + linear-ID Unicomp"}


class SelfJoin:
    """One engine context (one device).  Mirrors the reference call sequence:
    import / set_points -> build_index -> join."""

    def __init__(self, dim: int, eps: float, indexed_dims: Optional[int] = None, mode: int = 10,
                 precision: int = PREC_FP64, scheduler: int = SCHED_SAMPLING, capacity: int = 0,
                 sort_by_workload: int = 1, sample_rate: float = 0.01, alpha: float = 0.05,
                 device: int = 0, shard_index: int = 0, shard_count: int = 1):
        L = load()
        p = Params()
        L.sj_params_default(C.byref(p))
        p.gpunumdim = int(dim)
        p.numindexeddim = int(indexed_dims if indexed_dims is not None else dim)
        p.epsilon = float(eps)
        p.search_mode = int(mode)
        p.precision = int(precision)
        p.scheduler = int(scheduler)
        p.batch_capacity_pairs = int(capacity)
        p.sort_by_workload = int(sort_by_workload)
        p.sample_rate = float(sample_rate)
        p.alpha = float(alpha)
        p.device = int(device)
        p.shard_index = int(shard_index)
        p.shard_count = int(shard_count)
        self.params = p
        self._h = C.c_void_p()
        _check(L.sj_create(C.byref(p), C.byref(self._h)))
        self.n = 0

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            load().sj_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- input
    def set_points(self, pts: np.ndarray):
        a = np.ascontiguousarray(pts, dtype=np.float64)
        assert a.ndim == 2 and a.shape[1] == self.params.gpunumdim
        _check(load().sj_set_points(self._h, _ptr(a), a.shape[0], 0))
        self.n = a.shape[0]

    def set_points_device(self, ptr: int, n: int):
        _check(load().sj_set_points(self._h, C.c_void_p(ptr), int(n), 1))
        self.n = int(n)

    def import_csv(self, path: str):
        _check(load().sj_import_csv(self._h, path.encode()))
        self.n = None

    # ---- index
    def build_index(self):
        _check(load().sj_build_index(self._h))
        if self.n is None:
            self.n = int(self.stats().n_points)

    def index_export(self) -> dict:
        L = load()
        nne, nmask, tot = C.c_uint32(), C.c_uint32(), C.c_uint64()
        _check(L.sj_index_sizes(self._h, C.byref(nne), C.byref(nmask), C.byref(tot)))
        k = self.params.numindexeddim
        lookup = np.zeros(self.n, np.uint32)
        grid = (GridCell * max(nne.value, 1))()
        gcl = (GridCellLookup * max(nne.value, 1))()
        mn = np.zeros(k, np.float64)
        nc = np.zeros(k, np.uint32)
        mask = np.zeros(max(nmask.value, 1), np.uint32)
        moff = np.zeros(2 * k, np.uint32)
        _check(L.sj_index_export(self._h, _ptr(lookup), C.cast(grid, C.c_void_p), C.cast(gcl, C.c_void_p),
                                 _ptr(mn), _ptr(nc), _ptr(mask), _ptr(moff)))
        g = np.array([(c.indexmin, c.indexmax) for c in grid[:nne.value]], dtype=np.int32).reshape(-1, 2)
        lid = np.array([c.gridLinearID for c in gcl[:nne.value]], dtype=np.uint64)
        idx = np.array([c.idx for c in gcl[:nne.value]], dtype=np.uint32)
        return dict(indexLookupArr=lookup, grid=g, gridLinearID=lid, gridIdx=idx, minArr=mn, nCells=nc,
                    gridCellNDMask=mask[:nmask.value], gridCellNDMaskOffsets=moff, totalCells=tot.value)

    # ---- join
    def join(self, delivery: int = DELIVER_NONE, callback: Optional[Callable] = None):
        """Runs the join.  `callback(batch_index, key, val)` receives numpy
        arrays (host delivery) or (batch_index, key_ptr, val_ptr, count)
        (device delivery); return True to stop."""
        L = load()
        err = []

        def _cb(bp, _user):
            b = bp.contents
            try:
                if callback is None:
                    return 0
                if b.on_device:
                    r = callback(b.batch_index, b.key, b.val, b.count)
                else:
                    cnt = int(b.count)
                    if cnt:
                        key = np.ctypeslib.as_array(C.cast(b.key, C.POINTER(C.c_int32)), (cnt,))
                        val = np.ctypeslib.as_array(C.cast(b.val, C.POINTER(C.c_int32)), (cnt,))
                    else:
                        key = val = np.zeros(0, np.int32)
                    r = callback(b.batch_index, key, val)
                return 1 if r else 0
            except Exception as e:  # surface Python errors after the join returns
                err.append(e)
                return 1

        cb = BATCH_CB(_cb)
        st = L.sj_join(self._h, int(delivery), cb, None)
        if err:
            raise err[0]
        _check(st)
        return self.stats()

    def pairs(self):
        """All pairs on the host, in delivery order (sorted by key inside each batch)."""
        ks, vs = [], []

        def cb(_i, k, v):
            ks.append(k.copy())
            vs.append(v.copy())

        self.join(DELIVER_HOST, cb)
        if not ks:
            return np.zeros(0, np.int32), np.zeros(0, np.int32)
        return np.concatenate(ks), np.concatenate(vs)

    def degrees(self) -> np.ndarray:
        d = np.zeros(self.n, np.uint32)
        _check(load().sj_degrees(self._h, _ptr(d)))
        return d

    def neighbor_table(self):
        """(table rows [(indexmin, indexmax)], values) as numpy arrays."""
        L = load()
        n = self.n
        tab = (NeighborTableLookup * n)()
        vals = C.POINTER(C.c_int)()
        tot = C.c_uint64()
        _check(L.sj_neighbor_table(self._h, C.cast(tab, C.c_void_p), C.byref(vals), C.byref(tot)))
        try:
            v = np.ctypeslib.as_array(vals, (max(int(tot.value), 1),))[: int(tot.value)].copy()
            rows = np.array([(t.indexmin, t.indexmax) for t in tab], dtype=np.int64).reshape(-1, 2)
        finally:
            L.sj_free(C.cast(vals, C.c_void_p))
        return rows, v

    def neighbor_csr(self, row_ptr: int, cols: int = 0, capacity: int = 0) -> int:
        """Device CSR neighbour table: row_ptr / cols are device addresses
        (n+1 uint64 and `capacity` int32, e.g. torch tensors' data_ptr());
        cols = 0 only fills row_ptr.  Returns the number of values."""
        tot = C.c_uint64()
        _check(load().sj_neighbor_csr(self._h, C.c_void_p(row_ptr), C.c_void_p(cols or None), int(capacity),
                                      C.byref(tot)))
        return int(tot.value)

    def stream(self) -> int:
        """cudaStream_t of this context (for CUDA events around its work)."""
        s = C.c_void_p()
        _check(load().sj_get_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def stats(self) -> Stats:
        s = Stats()
        _check(load().sj_get_stats(self._h, C.byref(s)))
        return s

    # ---- learned estimator
    def set_estimator(self, weights: np.ndarray):
        w = np.ascontiguousarray(weights, dtype=np.float32)
        _check(load().sj_set_estimator_weights(self._h, _ptr(w), w.size))

    def load_estimator(self, path: str):
        _check(load().sj_load_estimator(self._h, path.encode()))

    def cell_samples(self):
        """(home hits, home evaluations, owned-neighbour hits, owned-neighbour
        evaluations) per cell from the sampling estimator (exact with
        sample_rate=1)."""
        return _cell_samples(self)

    def cell_features(self, with_hits: bool = True):
        nne = int(self.stats().n_nonempty_cells)
        f = np.zeros((nne, 16), np.float32)
        h = np.zeros(nne, np.float64)
        c = np.zeros(nne, np.float64)
        _check(load().sj_cell_features(self._h, _ptr(f), _ptr(h) if with_hits else None, _ptr(c)))
        return f, (h if with_hits else None), c


def _cell_samples(sj: "SelfJoin"):
    nne = int(sj.stats().n_nonempty_cells)
    out = [np.zeros(nne, np.float64) for _ in range(4)]
    _check(load().sj_cell_samples(sj._h, *[_ptr(a) for a in out]))
    return tuple(out)


def mlp_loss_grad(x: np.ndarray, y: np.ndarray, w: np.ndarray, device: int = 0):
    L = load()
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    g = np.zeros_like(w)
    loss = C.c_float()
    _check(L.sj_mlp_loss_grad(_ptr(x), _ptr(y), x.shape[0], _ptr(w), C.byref(loss), _ptr(g), device))
    return float(loss.value), g


MLP_NOALLOC_MAX_SAMPLES = 8192


def mlp_loss_grad_noalloc(x_ptr: int, y_ptr: int, m: int, w_ptr: int, loss_ptr: int, grad_ptr: int,
                          stream: int = 0):
    """Allocation-free loss/gradient on caller-owned device buffers (see sj.h).
    Queues the work on `stream` and returns without synchronising."""
    _check(load().sj_mlp_loss_grad_noalloc(C.c_void_p(x_ptr), C.c_void_p(y_ptr), int(m), C.c_void_p(w_ptr),
                                           C.c_void_p(loss_ptr), C.c_void_p(grad_ptr), C.c_void_p(stream or None)))


def mlp_forward(x: np.ndarray, w: np.ndarray, device: int = 0) -> np.ndarray:
    L = load()
    x = np.ascontiguousarray(x, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    out = np.zeros((x.shape[0], 2), np.float32)
    _check(L.sj_mlp_forward(_ptr(x), x.shape[0], _ptr(w), _ptr(out), device))
    return out


def mlp_train(x: np.ndarray, y: np.ndarray, w: np.ndarray, steps: int, lr: float = 1e-3, batch: int = 4096,
              seed: int = 1, device: int = 0):
    L = load()
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    w = np.ascontiguousarray(w, np.float32).copy()
    loss = C.c_float()
    _check(L.sj_mlp_train(_ptr(x), _ptr(y), x.shape[0], _ptr(w), int(steps), float(lr), int(batch), int(seed),
                          C.byref(loss), device))
    return w, float(loss.value)


def mlp_init(seed: int = 0) -> np.ndarray:
    """He-initialised parameters in the engine's layout."""
    rng = np.random.default_rng(seed)
    F, H, O = 16, 64, 2
    parts = [rng.standard_normal((F, H)) * np.sqrt(2.0 / F), np.zeros(H),
             rng.standard_normal((H, H)) * np.sqrt(2.0 / H), np.zeros(H),
             rng.standard_normal((H, O)) * np.sqrt(1.0 / H), np.zeros(O)]
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)


def canonical(keys: np.ndarray, vals: np.ndarray):
    """Pairs sorted by (key, value)."""
    k = np.asarray(keys, np.int64)
    v = np.asarray(vals, np.int64)
    o = np.lexsort((v, k))
    return k[o].astype(np.int32), v[o].astype(np.int32)


def pair_hash(keys: np.ndarray, vals: np.ndarray) -> int:
    """Order-independent set hash: wrapping sum of splitmix64(key << 32 | val)."""
    z = (np.asarray(keys, np.int64).astype(np.uint64) << np.uint64(32)) | \
        (np.asarray(vals, np.int64).astype(np.uint64) & np.uint64(0xffffffff))
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9e3779b97f4a7c15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
        z = z ^ (z >> np.uint64(31))
        return int(np.sum(z, dtype=np.uint64))

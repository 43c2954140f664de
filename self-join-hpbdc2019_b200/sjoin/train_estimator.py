"""Trains the learned batch estimator on counts the engine itself measures.

Data: seeded runs of the 6-D exponential(40) generator (the c4 workload's
distribution) with eps drawn uniformly from [0.01, 0.05] and the point count
drawn log-uniformly up to 1e7, the c4 workload's size.  For each run the
engine builds its index and computes every cell's 16 features; its count
pass then measures, with the sampling estimator at sample rate 1 (every
point, sj_cell_samples), each cell's hits among its own points and among its
owned neighbours' points under the linear-ID Unicomp traversal (search mode
10).  A cell's targets are (log2(1 + home hits), log2(1 + neighbour hits)):
the engine divides them by the cell's exactly known evaluation counts to get
the two hit rates that predict every task's pairs.  The point count of a run
is shrunk until the run's full-stencil work stays under a budget (by default
a little above the c4 workload's 4.06e13), so the heaviest runs reach the
cell sizes of that workload.

Training: the 16 -> 64 -> 64 -> 2 MLP is trained with the engine's own FP32
forward / backward / Adam kernels (sj_mlp_train).  The batch planner sums the
predictions over many cells, so what matters is the error on the cells that
hold the pairs: the training set is drawn from the collected cells with
probability proportional to (1 + hits)^beta (beta = 0.5 by default), which
keeps every cell size represented while the heavy cells that dominate a
batch's total are seen far more often than their number alone would give.
Last, the two output biases are shifted so that the summed predictions over
every collected cell equal the measured sums (a log-space fit predicts typical
values, while a batch's size is a sum).  Weights are written as raw float32 in
the engine's layout (sj_mlp_num_params() values).

usage: python -m sjoin.train_estimator [--runs 50] [--out sjoin/estimator_c4.bin]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import PREC_FP32_REFINE, SCHED_SAMPLING, SelfJoin, datasets, mlp_forward, mlp_init, mlp_loss_grad, mlp_train

PKG = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(PKG, "estimator_c4.bin")


def cell_table(pts: np.ndarray, eps: float, k: int, with_hits: bool = True):
    """(features, full-stencil calcs, targets or None) of every non-empty cell, measured by the engine."""
    D = pts.shape[1]
    with SelfJoin(D, eps, indexed_dims=k, mode=10, precision=PREC_FP32_REFINE, scheduler=SCHED_SAMPLING,
                  sample_rate=1.0) as sj:
        sj.set_points(pts)
        sj.build_index()
        feat, _, calcs = sj.cell_features(with_hits=False)
        y = None
        if with_hits:
            home, _, nbr, _ = sj.cell_samples()
            y = targets(home, nbr)
    return feat, calcs, y


def targets(home_hits: np.ndarray, nbr_hits: np.ndarray) -> np.ndarray:
    return np.stack([np.log2(1.0 + home_hits), np.log2(1.0 + nbr_hits)], 1).astype(np.float32)


def collect(runs: int = 50, seed0: int = 7000, n_max: int = 10_000_000, n_min: int = 50_000,
            work_budget: float = 4.5e13, D: int = 6, log=print):
    rng = np.random.default_rng(seed0)
    xs, ys, meta = [], [], []
    for r in range(runs):
        eps = float(rng.uniform(0.01, 0.05))
        n = int(10 ** rng.uniform(math.log10(n_min), math.log10(n_max)))
        seed = seed0 + r
        while True:
            pts = datasets.exponential(n, D, 40.0, seed)
            feat, calcs, _ = cell_table(pts, eps, D, with_hits=False)
            work = float(calcs.sum())
            if work <= work_budget or n <= n_min:
                break
            n = max(n_min, int(n * math.sqrt(work_budget / work) * 0.9))
        t0 = time.time()
        feat, calcs, y = cell_table(pts, eps, D, with_hits=True)
        xs.append(feat)
        ys.append(y)
        meta.append(dict(run=r, seed=seed, n=n, eps=eps, cells=len(feat), calcs=float(calcs.sum()),
                         hits=float((np.exp2(y.astype(np.float64)) - 1.0).sum()), s=round(time.time() - t0, 2)))
        log(json.dumps(meta[-1]))
    return np.concatenate(xs), np.concatenate(ys), meta


def resample(x: np.ndarray, y: np.ndarray, size: int = 4_000_000, beta: float = 0.5, seed: int = 1):
    """Training set drawn with probability proportional to (1 + hits)^beta (home + neighbour hits)."""
    hits = (np.exp2(y.astype(np.float64)) - 1.0).sum(1)
    p = np.power(1.0 + hits, beta)
    p /= p.sum()
    idx = np.random.default_rng(seed).choice(len(x), size=min(size, 4 * len(x)), replace=True, p=p)
    return x[idx], y[idx]


def train(x: np.ndarray, y: np.ndarray, steps: int = 6000, lr: float = 2e-3, batch: int = 4096, seed: int = 1):
    w0 = mlp_init(seed)
    # step-wise learning-rate decay: three stages
    w = w0
    for frac, scale in ((0.5, 1.0), (0.3, 0.3), (0.2, 0.1)):
        w, loss = mlp_train(x, y, w, steps=max(1, int(steps * frac)), lr=lr * scale, batch=batch, seed=seed)
    return w, loss


def calibrate(x: np.ndarray, y: np.ndarray, w: np.ndarray):
    """Shifts the two output biases so that the network's hits, summed over every collected cell,
    equal the measured sums.  A fit in log space predicts a typical value rather than the mean,
    while a batch's size is a sum of predictions: the shift removes that bias from the sums."""
    pred = mlp_forward(x, w).astype(np.float64)
    meas = np.exp2(y.astype(np.float64)) - 1.0
    shift = np.log2(meas.sum(0) / np.maximum(np.exp2(pred) - 1.0, 0.0).sum(0))
    w = w.astype(np.float32).copy()
    w[-2:] += shift.astype(np.float32)
    return w, [round(float(v), 6) for v in shift]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=50)
    ap.add_argument("--steps", type=int, default=12000)
    ap.add_argument("--beta", type=float, default=0.5, help="resampling exponent (0: every cell alike)")
    ap.add_argument("--data-in", default=None, help="train on a saved .npz instead of collecting")
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--data-out", default=None, help="optional .npz of the collected training set")
    args = ap.parse_args()
    t0 = time.time()
    if args.data_in:
        d = np.load(args.data_in)
        x, y = d["x"], d["y"]
    else:
        x, y, meta = collect(args.runs)
        print(f"collected {len(x)} cells from {len(meta)} runs in {time.time() - t0:.1f} s", flush=True)
    if args.data_out:
        np.savez_compressed(args.data_out, x=x, y=y)
    xt, yt = resample(x, y, beta=args.beta) if args.beta > 0 else (x, y)
    w, loss = train(xt, yt, steps=args.steps)
    w, shift = calibrate(x, y, w)
    full, _ = mlp_loss_grad(x, y, w)
    w.astype(np.float32).tofile(args.out)
    print(json.dumps({"cells": int(len(x)), "final_loss": full, "output_shift": shift, "out": args.out,
                      "seconds": round(time.time() - t0, 1)}), flush=True)


if __name__ == "__main__":
    main()

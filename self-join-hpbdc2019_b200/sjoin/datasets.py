"""Seeded synthetic point sets with the shapes of the five benchmark workloads.

No dataset ships with the reference; these generators stand in for them.
Exponential coordinates are drawn as -ln(1-U)/lambda and clipped to [0, 1].
"""
from __future__ import annotations

import numpy as np

# name -> (n, D, k, eps, kind, search mode, precision, batch capacity)
WORKLOADS = {
    "c1": dict(n=100_000, D=2, k=2, eps=0.01, kind="uniform", mode=3, precision=0, capacity=0),
    "c2": dict(n=2_000_000, D=2, k=2, eps=0.0015, kind="exp40", mode=5, precision=0, capacity=50_000_000),
    "c3": dict(n=5_000_000, D=4, k=4, eps=0.01, kind="exp40", mode=6, precision=1, capacity=100_000_000),
    "c4": dict(n=10_000_000, D=6, k=6, eps=0.03, kind="exp40", mode=10, precision=1, capacity=2_000_000_000),
    "c5": dict(n=1_000_000, D=16, k=6, eps=0.05, kind="gauss64", mode=10, precision=1, capacity=0),
}

SEEDS = {"c1": 101, "c2": 202, "c3": 303, "c4": 404, "c5": 505}


def uniform(n: int, D: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).random((n, D))


def exponential(n: int, D: int, lam: float, seed: int) -> np.ndarray:
    u = np.random.default_rng(seed).random((n, D))
    return np.clip(-np.log1p(-u) / lam, 0.0, 1.0)


def gaussian_mixture(n: int, D: int, seed: int, centres: int = 64, background: float = 0.10,
                     sigma=(0.02, 0.08)) -> np.ndarray:
    rng = np.random.default_rng(seed)
    nb = int(round(n * background))
    ng = n - nb
    c = rng.random((centres, D))
    s = rng.uniform(sigma[0], sigma[1], centres)
    lab = rng.integers(0, centres, ng)
    g = c[lab] + rng.standard_normal((ng, D)) * s[lab, None]
    pts = np.vstack([g, rng.random((nb, D))])
    return pts[rng.permutation(n)]


def make(name: str, n: int | None = None, seed: int | None = None, eps: float | None = None):
    """(points, eps, k, spec) for a named workload, optionally resized."""
    spec = dict(WORKLOADS[name])
    n = spec["n"] if n is None else int(n)
    seed = SEEDS[name] if seed is None else int(seed)
    if spec["kind"] == "uniform":
        pts = uniform(n, spec["D"], seed)
    elif spec["kind"] == "exp40":
        pts = exponential(n, spec["D"], 40.0, seed)
    else:
        pts = gaussian_mixture(n, spec["D"], seed)
    spec["n"] = n
    if eps is not None:
        spec["eps"] = float(eps)
    return pts, spec["eps"], spec["k"], spec


def write_csv(path: str, pts: np.ndarray):
    """Comma-separated, one point per line, 17 significant digits (exact round trip)."""
    np.savetxt(path, pts, delimiter=",", fmt="%.17g")

"""Shared test setup: import paths, the `gpu` marker and dataset helpers."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(REPO, "self-join-hpbdc2019_b200")
for p in (REPO, PKG_DIR):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def rng():
    return np.random.default_rng(12345)


def exp_points(n, d, seed, lam=40.0):
    u = np.random.default_rng(seed).random((n, d))
    return np.clip(-np.log1p(-u) / lam, 0.0, 1.0)


def shell_points(n, d, eps, seed):
    """Pairs of points at distance ~eps (borderline for the predicate)."""
    rng = np.random.default_rng(seed)
    base = rng.random((n, d))
    u = rng.standard_normal((n, d))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    other = base + eps * u
    return np.vstack([base, other])


def lattice_points(m, d, step):
    g = np.stack(np.meshgrid(*([np.arange(m) * step] * d), indexing="ij"), -1).reshape(-1, d)
    return g.astype(np.float64)

"""The FP32 filter's error bound, checked on CPU by exact emulation.

The count pass's mixed-precision path (sj_join.cu: query setup, eval_block_f32)
computes, per (query a, candidate b) in FP32,
    y = RN(RN(nb32 - tLo) + sum_l fma(-2 a~_l, b~_l, .))     (one rounding per op)
with a~ = RN32(a - o), b~ = RN32(b - o) local coordinates (o: the home cell's
centre on indexed dims, the data centre elsewhere), nb32 = RN32(sum b~^2),
tLo = RD32(T - sum a~^2 - M), and calls the pair a hit when y's sign bit is set,
borderline (re-evaluated in FP64) when RN32(y - delta) is negative too.  The
bound (filter_bounds in sj_api.cpp, restated below) must make
  * every FP32 hit a hit of the pinned FP64 predicate, and
  * every pair outside the band a miss of it,
so the emitted set is the FP64 set.  Here every FP32 operation is emulated
exactly (rational arithmetic, one round-to-nearest-even per operation) on
random stencil pairs and on pairs within 1e-6 relative of the threshold.
"""
import math
from fractions import Fraction

import numpy as np
import pytest

U = 2.0 ** -24


def rn32(x: Fraction) -> Fraction:
    """x rounded to the nearest binary32 value, ties to even (normal range)."""
    if x == 0:
        return Fraction(0)
    s = -1 if x < 0 else 1
    x = abs(x)
    e = math.floor(math.log2(x.numerator) - math.log2(x.denominator))
    while Fraction(2) ** e > x:
        e -= 1
    while Fraction(2) ** (e + 1) <= x:
        e += 1
    assert e >= -126, "subnormal range"
    scaled = x / Fraction(2) ** (e - 23)          # in [2^23, 2^24)
    q, r = divmod(scaled.numerator, scaled.denominator)
    twice = 2 * r
    if twice > scaled.denominator or (twice == scaled.denominator and q & 1):
        q += 1
    return s * Fraction(q) * Fraction(2) ** (e - 23)


def f32(x: float) -> Fraction:
    return Fraction(float(np.float32(x)))


def rd32(x: float) -> Fraction:
    f = np.float32(x)
    if float(f) > x:
        f = np.nextafter(f, np.float32(-np.inf))
    return Fraction(float(f))


def threshold(eps):
    t = eps * eps
    while math.sqrt(t) > eps:
        t = math.nextafter(t, -math.inf)
    while math.sqrt(math.nextafter(t, math.inf)) <= eps:
        t = math.nextafter(t, math.inf)
    return t


def bounds(D, k, eps, lo, hi):
    """margin M and band delta exactly as filter_bounds computes them."""
    ra2 = rb2 = 0.0
    for j in range(D):
        if j < k:
            ra2 += (0.5 * eps * 1.01) * (0.5 * eps * 1.01)
            rb2 += (1.5 * eps * 1.01) * (1.5 * eps * 1.01)
        else:
            h = 0.5 * (hi[j] - lo[j]) * 1.01 + 1e-300
            ra2 += h * h
            rb2 += h * h
    r = math.sqrt(ra2) + math.sqrt(rb2)
    T = threshold(eps)
    margin = 2.0 * (D + 4) * U * (r * r + T) + math.ldexp(r * r + T, -39)
    d = (2.0 * margin + 2.0 * U * (T + ra2 + margin)) * (1.0 + math.ldexp(1.0, -20))
    df = float(np.float32(d))
    if df < d:
        df = float(np.nextafter(np.float32(d), np.float32(np.inf)))
    return T, margin, df


def pinned_d2(a, b):
    """The reference's FP64 rounding order: fma(d0, d0, d1*d1), then fma(dl, dl, acc)."""
    d = [bb - aa for aa, bb in zip(a, b)]
    if len(d) == 1:
        return d[0] * d[0]
    acc = float(Fraction(d[0]) * Fraction(d[0]) + Fraction(d[1] * d[1]))
    for x in d[2:]:
        acc = float(Fraction(x) * Fraction(x) + Fraction(acc))
    return acc


def filter32(a, b, o, T, margin, delta):
    """(hit, borderline) of the FP32 filter for query a and candidate b."""
    at = [f32(x - y) for x, y in zip(a, o)]
    bt = [f32(x - y) for x, y in zip(b, o)]
    na = 0.0
    for x in at:
        na += float(x) * float(x)
    nb = 0.0
    for x in bt:
        nb += float(x) * float(x)
    tlo = rd32(T - na - margin)
    y = rn32(f32(nb) - tlo)
    for x, z in zip(at, bt):
        y = rn32(-2 * x * z + y)
    hit = y < 0
    near = rn32(y - Fraction(delta)) < 0
    return hit, near


CONFIGS = {
    # name: (D, k, eps, per-dim data extent lo, hi)
    "2d": (2, 2, 0.01, 0.0, 1.0),
    "6d": (6, 6, 0.03, 0.0, 1.0),
    "16d_k6": (16, 6, 0.05, 0.0, 1.0),
    "12d_k3": (12, 3, 0.3, 0.0, 0.4),
    "3d_offset": (3, 3, 0.04, 1.0e4, 1.0e4 + 0.5),
    "5d_k2_wide": (5, 2, 0.15, 0.0, 3.0e5),
}


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_fp32_filter_never_disagrees_outside_its_band(name):
    D, k, eps, lo0, hi0 = CONFIGS[name]
    rng = np.random.default_rng(sorted(CONFIGS).index(name) + 7)
    lo, hi = np.full(D, lo0), np.full(D, hi0)
    if name == "5d_k2_wide":
        hi[:k] = 1.0                                # the wide extent is in non-indexed dims
    T, margin, delta = bounds(D, k, eps, lo, hi)
    min_arr = lo - eps
    centre = 0.5 * (lo + hi)
    checked = 0
    border = [0, 0]     # borderline pairs among [near-threshold, random stencil] pairs
    drawn = [0, 0]
    for trial in range(1500):
        a = lo + (hi - lo) * (0.1 + 0.8 * rng.random(D))
        if trial % 2 == 0:                          # within 1e-6 relative of the threshold
            u = rng.standard_normal(D)
            u /= np.linalg.norm(u)
            b = a + u * math.sqrt(T) * (1.0 + 1e-6 * (2 * rng.random() - 1))
        else:                                       # anywhere in the stencil
            b = a.copy()
            b[:k] += eps * (3 * rng.random(k) - 1.5)
            b[k:] = lo[k:] + (hi[k:] - lo[k:]) * rng.random(D - k)
        b = np.clip(b, lo, hi)
        ca = np.floor((a[:k] - min_arr[:k]) / eps)
        cb = np.floor((b[:k] - min_arr[:k]) / eps)
        if np.any(np.abs(ca - cb) > 1):
            continue                                # not a stencil candidate
        o = np.concatenate([min_arr[:k] + (ca + 0.5) * eps, centre[k:]])
        a_l, b_l, o_l = a.tolist(), b.tolist(), o.tolist()
        exact = pinned_d2(a_l, b_l) <= T
        hit, near = filter32(a_l, b_l, o_l, T, margin, delta)
        if hit:
            assert exact, (name, a_l, b_l)
        elif not near:
            assert not exact, (name, a_l, b_l)
        else:
            border[trial % 2] += 1
        drawn[trial % 2] += 1
        checked += 1
    assert checked > 1000
    if name != "5d_k2_wide":                        # the band is narrow outside the wide case
        assert border[1] <= 0.02 * drawn[1], (border, drawn)


def test_the_check_catches_a_filter_without_margin():
    # the same emulation with no margin and no band must meet disagreements
    # near the threshold (so the test above can fail)
    D, k, eps, lo0, hi0 = CONFIGS["6d"]
    lo, hi = np.full(D, lo0), np.full(D, hi0)
    T, _, _ = bounds(D, k, eps, lo, hi)
    rng = np.random.default_rng(1)
    min_arr, centre = lo - eps, 0.5 * (lo + hi)
    wrong = 0
    for _ in range(1500):
        a = lo + (hi - lo) * (0.1 + 0.8 * rng.random(D))
        u = rng.standard_normal(D)
        u /= np.linalg.norm(u)
        b = a + u * math.sqrt(T) * (1.0 + 1e-6 * (2 * rng.random() - 1))
        ca = np.floor((a[:k] - min_arr[:k]) / eps)
        o = np.concatenate([min_arr[:k] + (ca + 0.5) * eps, centre[k:]])
        exact = pinned_d2(a.tolist(), b.tolist()) <= T
        hit, near = filter32(a.tolist(), b.tolist(), o.tolist(), T, 0.0, 1e-30)
        wrong += (hit and not exact) or (not hit and not near and exact)
    assert wrong > 0

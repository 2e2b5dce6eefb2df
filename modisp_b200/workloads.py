"""Seeded synthetic layered-model batches of the benchmark configurations.

No public dataset is named for this path; these generators stand in for it with
the shapes, sizes and value distributions the benchmark configurations state.
Each batch is [B, L] (h, vp, vs, rho), ragged models padded the modisp way: the
real layers, then zero-thickness copies of the half-space, then the half-space
(python/modisp/models.py:224-270).
"""
from __future__ import annotations

import numpy as np

SEED = 20261203


def _gardner(vp):
    return 1.74 * vp ** 0.25


def _pad(rows, L):
    """Pack a list of (h, vp, vs, rho) row arrays into padded [B, L] arrays."""
    B = len(rows)
    out = {k: np.zeros((B, L)) for k in ("thickness", "vp", "vs", "rho")}
    for i, (h, vp, vs, rho) in enumerate(rows):
        n = h.size - 1  # finite layers
        for key, src in zip(("thickness", "vp", "vs", "rho"), (h, vp, vs, rho)):
            out[key][i, :n] = src[:n]
            out[key][i, n:] = src[n]
        out["thickness"][i, n:] = 0.
    return out


def quickstart():
    """One layer over a half-space (the reference quickstart model)."""
    return dict(thickness=np.array([0.3, 0.]), vp=np.array([2.0, 5.0]), vs=np.array([0.8, 2.8]),
                rho=np.array([2.0, 2.6])), np.geomspace(0.1, 10., 30)


def crustal_batch(B, seed=SEED + 2, nmin=8, nmax=20, lvz_fraction=0.0, layers=None):
    """Random crustal models: n ~ U{nmin..nmax} finite layers (or exactly `layers`),
    h ~ U(0.2, 3) km, Vs rising linearly from U(0.3, 1.0) to U(3.5, 4.7) km/s with
    +-10 % row noise, Vp = Vs U(1.7, 2.0), rho = 1.74 Vp^0.25.  A fraction
    `lvz_fraction` of the models get one interior low-velocity layer whose Vs is
    20-40 % below the layer above it."""
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(B):
        n = int(layers) if layers else int(rng.integers(nmin, nmax + 1))
        top, bottom = rng.uniform(0.3, 1.0), rng.uniform(3.5, 4.7)
        vs = (top + (bottom - top) * np.arange(n + 1) / n) * rng.uniform(0.9, 1.1, n + 1)
        vs[-1] = max(vs[-1], vs[:-1].max() * 1.02)  # the half-space stays the fastest
        ratio = rng.uniform(1.7, 2.0, n + 1)
        if lvz_fraction and rng.uniform() < lvz_fraction and n >= 3:
            j = int(rng.integers(1, n))
            vs[j] = vs[j - 1] * (1. - rng.uniform(0.2, 0.4))
        vp = vs * ratio
        h = rng.uniform(0.2, 3.0, n + 1)
        h[-1] = 0.
        rows.append((h, vp, vs, _gardner(vp)))
    L = max(r[0].size for r in rows)
    return _pad(rows, L)


def config2(B=10_000):
    """Batched FP64: 8-20 layers, 60 periods 0.5-50 s, 5 modes."""
    return crustal_batch(B, SEED + 2), np.geomspace(0.5, 50., 60), 5


def config3(B=100_000):
    """Mixed precision: as config 2 with 30 % low-velocity-layer models."""
    return crustal_batch(B, SEED + 3, lvz_fraction=0.3), np.geomspace(0.5, 50., 60), 5


def config4(B=4096):
    """Differentiation: 12 layers each, 40 periods 1-40 s, 3 modes, Rayleigh."""
    return crustal_batch(B, SEED + 4, layers=12), np.geomspace(1., 40., 40), 3


def deep_batch(B, seed=SEED + 6):
    """Deep slow-over-fast models whose short periods carry hundreds of modes:
    n ~ U{3..5} finite layers of h ~ U(15, 80) km, Vs rising from U(0.4, 0.9) to
    U(2.5, 3.5) km/s over the stack, a half-space of Vs ~ U(4.2, 4.7) km/s,
    Vp = Vs U(1.75, 2.2), rho = 1.74 Vp^0.25."""
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(B):
        n = int(rng.integers(3, 6))
        top, bottom = rng.uniform(0.4, 0.9), rng.uniform(2.5, 3.5)
        vs = np.append(top + (bottom - top) * np.arange(n) / (n - 1), rng.uniform(4.2, 4.7))
        vp = vs * rng.uniform(1.75, 2.2, n + 1)
        h = np.append(rng.uniform(15., 80., n), 0.)
        rows.append((h, vp, vs, _gardner(vp)))
    return _pad(rows, max(r[0].size for r in rows))


def gradient_batch(B, seed=SEED + 5):
    """Smooth-gradient models: n ~ U{30..100} layers of h = 80/n km, Vs(z) = 0.2 + 4.3 z/80
    with +-5 % noise, Vp/rho as above; per-model periods (50-120 geomspaced in a random
    sub-window of 0.2-100 s) and mode counts 1-10.  Returns (batch, periods list, modes)."""
    rng = np.random.default_rng(seed)
    rows, periods, modes = [], [], []
    for _ in range(B):
        n = int(rng.integers(30, 101))
        z = (np.arange(n + 1) + 0.5) * 80. / n
        vs = (0.2 + 4.3 * np.minimum(z, 80.) / 80.) * rng.uniform(0.95, 1.05, n + 1)
        vs[-1] = max(vs[-1], vs[:-1].max() * 1.02)
        vp = vs * rng.uniform(1.7, 2.0, n + 1)
        h = np.full(n + 1, 80. / n)
        h[-1] = 0.
        rows.append((h, vp, vs, _gardner(vp)))
        a, b = np.sort(np.exp(rng.uniform(np.log(0.2), np.log(100.), 2)))
        if b / a < 1.5:
            b = min(100., a * 1.5)
        periods.append(np.geomspace(a, b, int(rng.integers(50, 121))))
        modes.append(int(rng.integers(1, 11)))
    return _pad(rows, max(r[0].size for r in rows)), periods, modes

"""Seeded synthetic workloads (stand-ins for the reference's SIFT files).

``mixture`` draws an isotropic Gaussian mixture: centres uniform in [0, 255],
sigma 20, rounded and clipped to [0, 255] (integer-valued FP32, the shape of
SIFT data), or unit-norm centres with small sigma for the float configuration.
All draws use numpy's default_rng so any machine reproduces them bit for bit.
"""
from __future__ import annotations

import numpy as np


def mixture(n: int, dim: int, clusters: int, seed: int, sigma: float = 20.0, centres_seed: int = 1234,
            integer: bool = True, unit_norm: bool = False, chunk: int = 1 << 18) -> np.ndarray:
    crng = np.random.default_rng(centres_seed)
    if unit_norm:
        centres = crng.standard_normal((clusters, dim)).astype(np.float64)
        centres /= np.linalg.norm(centres, axis=1, keepdims=True)
    else:
        centres = crng.uniform(0.0, 255.0, (clusters, dim))
    rng = np.random.default_rng(seed)
    out = np.empty((n, dim), np.float32)
    for s in range(0, n, chunk):
        m = min(chunk, n - s)
        lab = rng.integers(0, clusters, m)
        x = centres[lab] + sigma * rng.standard_normal((m, dim))
        if integer:
            x = np.clip(np.rint(x), 0.0, 255.0)
        out[s:s + m] = x
    return out


def config1(seed_base: int = 1, seed_query: int = 2):
    """10,000 x 128 integer-valued base, 100 queries, 100 clusters."""
    base = mixture(10_000, 128, 100, seed_base)
    q = mixture(100, 128, 100, seed_query)
    return base, q


def config2(n: int = 1_000_000, nq: int = 10_000, seed_base: int = 1, seed_query: int = 2):
    """1M x 128 integer-valued base, 10k queries, 1,000 clusters."""
    base = mixture(n, 128, 1000, seed_base)
    q = mixture(nq, 128, 1000, seed_query)
    return base, q

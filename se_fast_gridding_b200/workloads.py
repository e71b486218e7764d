"""Seeded synthetic particle systems and the error measure of the benchmarks.

The same counter-based (Philox) streams as the systems the test fixtures were
generated from, so a benchmark input equals the fixture's input bit for bit.
"""
from __future__ import annotations

import numpy as np


def synthetic_system(N: int, L: float = 1.0, seed: int = 0, charges="pm1",
                     clusters: int = 0, sigma: float = 0.02):
    """Positions in [0, L)^3 as SoA (x[n], x[n+N], x[n+2N]) and charges.

    charges: 'pm1' -- +-1 with zero sum (one charge 0 when N is odd), shuffled;
             'uniform' -- uniform in [-1, 1], minus their mean.
    clusters > 0: positions from that many isotropic Gaussians of width
    sigma*L around uniform centres, wrapped into the box."""
    rng = np.random.Generator(np.random.Philox(seed))
    if clusters > 0:
        centres = rng.random((clusters, 3)) * L
        which = rng.integers(0, clusters, size=N)
        pos = np.mod(centres[which] + rng.normal(0.0, sigma * L, size=(N, 3)), L)
    else:
        pos = rng.random((N, 3)) * L
    pos[pos >= L] = 0.0
    if charges == "pm1":
        q = np.ones(N)
        q[N // 2:] = -1.0
        if N % 2:
            q[-1] = 0.0
        rng.shuffle(q)
    elif charges == "uniform":
        q = rng.uniform(-1.0, 1.0, size=N)
        q -= q.mean()
    else:
        raise ValueError(charges)
    return np.ascontiguousarray(pos.T.reshape(-1)), np.ascontiguousarray(q)


def rel_rms(a, b) -> float:
    """||a - b||_2 / ||b||_2 over all entries."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))

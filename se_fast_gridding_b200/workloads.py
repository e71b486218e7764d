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


def c3_systems(seed: int = 3):
    """The batched workload: 256 independent POTENTIAL systems, N log-uniform
    in [1e3, 6.4e4], L uniform in [1, 4], M = 64 (h = L/64), P from
    {8, 12, 16}, xi = 8/L, charges +-1 (each system seeded 1000 + i)."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for i in range(256):
        N = int(round(np.exp(rng.uniform(np.log(1e3), np.log(6.4e4)))))
        L = float(rng.uniform(1.0, 4.0))
        P = int(rng.choice([8, 12, 16]))
        out.append(dict(N=N, M=64, P=P, L=L, xi=8.0 / L, seed=1000 + i))
    return out


# The large clustered FORCE system (16M particles in 64 Gaussian clusters of
# width 0.02 L, M = 512, P = 12, xi = 60) and its scaled-down shape for the
# parity tests: the same clusters and stencil with N and M reduced so that
# N / M^3 and xi h stay those of the full size.
C5 = dict(N=16_000_000, M=512, P=12, xi=60.0, L=1.0, clusters=64, sigma=0.02, seed=5)
C5_SCALED = dict(N=2_000_000, M=256, P=12, xi=30.0, L=1.0, clusters=64, sigma=0.02, seed=5)

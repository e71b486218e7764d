"""Request traces of the serving benchmark (host logic, no GPU)."""
import math

import numpy as np

from se_fast_gridding_b200 import serve


def test_grid_reading():
    assert serve.grid_for(500) == 64
    assert serve.grid_for(16000) == 64
    assert serve.grid_for(16001) == 128
    assert serve.grid_for(128000) == 128
    assert serve.grid_for(128001) == 256
    assert serve.grid_for(2_000_000) == 256     # capped at 256^3


def test_poisson_trace_statistics():
    tr = serve.poisson_trace(2000.0, 5.0, seed=4)
    assert tr == serve.poisson_trace(2000.0, 5.0, seed=4)          # deterministic
    n = len(tr)
    assert abs(n - 10000) < 4 * math.sqrt(10000)                    # Poisson count
    t = np.array([r.t for r in tr])
    assert np.all(np.diff(t) > 0) and t[-1] < 5.0
    gaps = np.diff(t)
    assert abs(gaps.mean() - 1 / 2000) < 0.05 / 2000
    N = np.array([r.system.N for r in tr])
    assert N.min() >= 500 and N.max() <= 2_000_000
    # log-uniform: the median sits at the geometric mean of the range
    assert abs(np.log(np.median(N)) - 0.5 * (np.log(500) + np.log(2e6))) < 0.15
    modes = [r.system.mode for r in tr]
    assert abs(modes.count("force") / n - 0.5) < 0.03
    assert {r.system.P for r in tr} == {8, 12, 16}
    for r in tr[:500]:
        s = r.system
        assert s.M == serve.grid_for(s.N)
        assert math.isclose(s.xi * s.L / s.M, 8.0 / 64)
        assert 0 <= r.offset and r.offset + 3 * s.N <= 6_000_000


def test_literal_grid_trace():
    tr = serve.poisson_trace(2000.0, 0.5, seed=5, literal_grid=True)
    assert {r.system.M for r in tr} == {64}
    assert all(math.isclose(r.system.xi, 8.0) for r in tr)

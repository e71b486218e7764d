"""The benchmark's seeded inputs are the fixtures' inputs, bit for bit."""
import numpy as np
import pytest

from se_fast_gridding_b200 import workloads as W


@pytest.mark.parametrize("kw", [dict(N=1001, seed=1, charges="uniform"),
                                dict(N=1000, L=3.0, seed=7),
                                dict(N=777, seed=5, clusters=8, sigma=0.02)])
def test_generator_matches_oracle(oracle_mod, kw):
    x0, q0 = oracle_mod.synthetic_system(**kw)
    x1, q1 = W.synthetic_system(**kw)
    np.testing.assert_array_equal(x0, x1)
    np.testing.assert_array_equal(q0, q1)
    L = kw.get("L", 1.0)
    assert x1.min() >= 0 and x1.max() < L
    assert abs(q1.sum()) < 1e-12 * len(q1)


def test_rel_rms(oracle_mod):
    rng = np.random.Generator(np.random.Philox(2))
    a, b = rng.random(100), rng.random(100)
    assert W.rel_rms(a, b) == oracle_mod.rel_rms(a, b)
    assert W.rel_rms(b, b) == 0.0

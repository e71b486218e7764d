"""Accuracy-driven parameter choice (se_choose_params): host code, no GPU."""
import math

import numpy as np
import pytest

from se_fast_gridding_b200 import solver


def bound(P, L, xi, Q, mode):
    # SE_init_params' printed estimates (SE_general.c:531-549), c = 0.95
    c = 0.95
    g = math.exp(-math.pi * P * c * c / 2)
    if mode == "force":
        return Q * math.sqrt(xi * L) / L / L * g * 2 * math.pi * c * c * P
    return math.sqrt(Q * xi * L) / L * g


@pytest.mark.parametrize("mode", ["potential", "force"])
@pytest.mark.parametrize("eps", [1e-4, 1e-7, 1e-10])
@pytest.mark.parametrize("L,xi", [(1.0, 8.0), (3.1814, 8.0), (1.0, 20.0)])
def test_choose_params(mode, eps, L, xi):
    Q = 100.0
    M, P, m = solver.choose_params(eps, L, xi, Q, mode)
    assert solver.error_estimate(P, L, xi, Q, mode) == pytest.approx(bound(P, L, xi, Q, mode),
                                                                      rel=1e-12)
    assert bound(P, L, xi, Q, mode) <= eps < bound(P - 1, L, xi, Q, mode)
    assert m == pytest.approx(0.95 * math.sqrt(math.pi * P))
    assert M >= max(math.ceil(4 * xi * L + 1) + 2, P)
    assert (M % 16 == 0) if M >= 32 else (M % 2 == 0)


def test_choose_params_from_charges_and_limits():
    q = np.array([1.0, -1.0, 0.5, -0.5])
    assert solver.choose_params(1e-6, 1.0, 8.0, q) == solver.choose_params(1e-6, 1.0, 8.0, 2.5)
    from se_fast_gridding_b200 import _lib
    with pytest.raises(_lib.SEError):
        solver.choose_params(1e-300, 1.0, 8.0, 1.0)     # no P <= 32 reaches it
    with pytest.raises(_lib.SEError):
        solver.choose_params(-1.0, 1.0, 8.0, 1.0)

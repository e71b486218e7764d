"""Real-space and self terms of the Ewald sum on the GPU (se_real_space,
se_self_term) against the reference's SE3P_direct_real_rc / SE3P_direct_real /
SE3P_direct_self outputs (FP64, 1e-12), the cell-list form against the oracle,
the real-space force against the oracle, and the three parts together: the
total Ewald potential does not depend on the splitting parameter xi."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from se_fast_gridding_b200 import solver
    return torch, solver


def cuda(torch, a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("tag", ["atoms_l1_rc1.5", "atoms_l0_rc1.2", "atoms_l1_nocut",
                                 "atoms_l2_rc2", "syn_l1_rc0.35", "syn_l1_rc0.5"])
def test_real_space_and_self_match_reference(env, tag):
    import oracle as O
    torch, S = env
    g = load_golden("realspace.npz")
    src = "atoms" if tag.startswith("atoms") else "syn"
    x, q = cuda(torch, g[f"{src}/x"]), cuda(torch, g[f"{src}/q"])
    L, xi, layers, rc = g[f"{tag}/params"]
    phi, _ = S.real_space(x, q, L, xi, int(layers), rc)
    assert O.rel_rms(phi.cpu().numpy(), g[f"{tag}/phi"]) < TOL
    selfp = S.self_term(q, xi).cpu().numpy()
    np.testing.assert_allclose(selfp, g[f"{tag}/self"], rtol=1e-15, atol=0)


@pytest.mark.parametrize("layers", [0, 1])
def test_cell_list_matches_oracle(env, layers):
    """0 < rc <= L/2 with >= 3 cells per axis: the cell-list form, positions
    partly outside the box (whole boxes away), potential and force."""
    import oracle as O
    torch, S = env
    N, L, xi, rc = 2500, 1.0, 12.0, 0.2
    x, q = O.synthetic_system(N, L, seed=40 + layers, charges="uniform")
    rng = np.random.Generator(np.random.Philox(3))
    shift = rng.integers(-1, 2, size=3 * N) * (rng.random(3 * N) < 0.1)
    x = x + shift * L
    phi, f = S.real_space(cuda(torch, x), cuda(torch, q), L, xi, layers, rc, want_force=True)
    ref = O.direct_real(x, q, L, xi, layers, rc)
    assert O.rel_rms(phi.cpu().numpy(), ref) < TOL
    fref = O.direct_real_force(x, q, L, xi, layers, rc)
    assert O.rel_rms(f.cpu().numpy(), fref) < TOL
    # accumulation into given buffers
    phi2, f2 = S.real_space(cuda(torch, x), cuda(torch, q), L, xi, layers, rc, phi=phi.clone(),
                            force=f.clone())
    np.testing.assert_allclose(phi2.cpu().numpy(), 2 * phi.cpu().numpy(), rtol=1e-14, atol=0)


def test_all_pairs_force_matches_oracle(env):
    import oracle as O
    torch, S = env
    x, q = O.synthetic_system(300, 1.0, seed=9, charges="uniform")
    _, f = S.real_space(cuda(torch, x), cuda(torch, q), 1.0, 5.0, 2, 0.0, want_force=True)
    assert O.rel_rms(f.cpu().numpy(), O.direct_real_force(x, q, 1.0, 5.0, 2, 0.0)) < TOL


def test_total_ewald_potential_independent_of_xi(env):
    """real (rc = L/2) + k-space (SE, FP64) + self = the Ewald potential of the
    periodic system, whatever the splitting xi."""
    import oracle as O
    torch, S = env
    N = 200
    x, q = O.synthetic_system(N, 1.0, seed=5, charges="pm1")
    xd, qd = cuda(torch, x), cuda(torch, q)
    totals = []
    for xi in (12.0, 14.0):
        se = S.SpectralEwald(64, 21, 1.0, xi, None, "potential", "fp64", N)
        phi = se.solve(xd, qd)
        S.real_space(xd, qd, 1.0, xi, 1, 0.5, phi=phi)
        S.self_term(qd, xi, phi=phi)
        totals.append(phi.cpu().numpy())
        se.close()
    assert O.rel_rms(totals[0], totals[1]) < 1e-8, O.rel_rms(totals[0], totals[1])


def test_invalid_arguments(env):
    torch, S = env
    from se_fast_gridding_b200 import _lib
    q = torch.ones(4, dtype=torch.float64, device="cuda")
    x = torch.zeros(12, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.SEError):
        S.real_space(x, q, -1.0, 5.0)
    with pytest.raises(_lib.SEError):
        S.real_space(x, q, 1.0, 5.0, layers=-1)

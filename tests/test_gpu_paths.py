"""Kernel paths (se_plan_create_ex): every spread / interpolation kernel
combination a configuration allows meets the accuracy bounds, forced paths
the configuration does not allow are refused, and the timed choice
(SE_PATH_TUNE) picks a valid path and remembers it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from se_fast_gridding_b200 import _lib, solver
    return torch, solver, _lib


ALL = [3, 7, 1, 2, 0, 4]


@pytest.mark.parametrize("mode", ["potential", "force"])
@pytest.mark.parametrize("P", [8, 12])
def test_every_path_meets_the_bounds(env, mode, P):
    import oracle as O
    torch, S, L = env
    M, N = 32, 3000
    x, q = O.synthetic_system(N, 1.0, seed=P, charges="uniform")
    m = S.default_m(P)
    ref = O.spectral_ewald(x, q, M, P, m, 1.0, 6.0, mode)
    xd, qd = torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda")
    for path in ALL:
        for prec, tol in (("fp64", 1e-12), ("fp32", 1e-6)):
            se = S.SpectralEwald(M, P, 1.0, 6.0, m, mode, prec, N, path=path)
            assert se.path == path
            out = se.solve(xd, qd).cpu().numpy()
            assert O.rel_rms(out, ref) < tol, (path, prec, O.rel_rms(out, ref))
            se.close()


def test_paths_the_configuration_does_not_allow(env):
    torch, S, L = env
    with pytest.raises(L.SEError):
        S.SpectralEwald(24, 8, 1.0, 6.0, None, "force", "fp32", 100, path=1)   # M % 16 != 0
    with pytest.raises(L.SEError):
        S.SpectralEwald(32, 21, 1.0, 6.0, None, "force", "fp64", 100, path=2)  # P > 16
    with pytest.raises(L.SEError):
        S.SpectralEwald(32, 8, 1.0, 6.0, None, "force", "fp32", 100, path=64)
    se = S.SpectralEwald(24, 8, 1.0, 6.0, None, "force", "fp32", 100, path=4)
    assert se.path == 4
    assert S.SpectralEwald(32, 8, 1.0, 6.0, None, "force", "fp32", 100).path == 3
    assert S.SpectralEwald(32, 6, 1.0, 6.0, None, "force", "fp32", 100).path == 1
    assert S.SpectralEwald(24, 8, 1.0, 6.0, None, "force", "fp32", 100).path == 0


def test_tuned_path(env):
    import oracle as O
    torch, S, L = env
    M, P, N = 64, 8, 20000
    se = S.SpectralEwald(M, P, 1.0, 10.0, None, "potential", "fp32", N, path="tune")
    assert se.path in ALL
    again = S.SpectralEwald(M, P, 1.0, 10.0, None, "potential", "fp32", N, path="tune")
    assert again.path == se.path                      # remembered, not re-timed
    x, q = O.synthetic_system(N, 1.0, seed=3)
    ref = O.spectral_ewald(x, q, M, P, S.default_m(P), 1.0, 10.0, "potential")
    out = se.solve(torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda"))
    assert O.rel_rms(out.cpu().numpy(), ref) < 1e-6
    small = S.SpectralEwald(24, 6, 1.0, 6.0, None, "force", "fp64", 500, path="tune")
    assert small.path in (0, 4)


@pytest.mark.parametrize("M,P,mode", [(64, 16, "force"), (64, 12, "potential"),
                                      (32, 8, "force"), (48, 12, "force")])
def test_bin_windows_equal_pair_windows(env, M, P, mode):
    """The pair interpolation's windows of two z-adjacent bins (the FP32
    default) and of one bin (SE_PATH_BIN_WINDOWS) sum the same cells in the
    same order: the results are bit-identical, in a single plan and in a
    batch of mixed stencils (the runtime-P kernel)."""
    import oracle as O
    torch, S, L = env
    N = 20000
    x, q = O.synthetic_system(N, 1.0, seed=M + P, charges="uniform")
    xd, qd = torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda")
    base = S.default_path(M, P)
    outs = []
    for path in (base, base | L.SE_PATH_BIN_WINDOWS):
        se = S.SpectralEwald(M, P, 1.0, 8.0 * M / 64, None, mode, "fp32", N, path=path)
        outs.append(se.solve(xd, qd).cpu().numpy())
        se.close()
    assert np.array_equal(outs[0], outs[1])
    ref = O.spectral_ewald(x, q, M, P, S.default_m(P), 1.0, 8.0 * M / 64, mode)
    assert O.rel_rms(outs[0], ref) < 1e-6


def test_bin_windows_equal_pair_windows_batch(env):
    import oracle as O
    torch, S, L = env
    systems = [S.System(N, M, P, 1.3, 8.0 / 1.3, None, mode)
               for M, P, N, mode in [(64, 8, 9000, "potential"), (32, 12, 4000, "force"),
                                     (64, 16, 15000, "force"), (48, 12, 7000, "potential")]]
    xs, qs = zip(*[O.synthetic_system(s.N, s.L, seed=40 + k, charges="pm1")
                   for k, s in enumerate(systems)])
    outs = []
    for extra in (0, L.SE_PATH_BIN_WINDOWS):
        b = S.BatchSolver(systems, "fp32",
                          paths=[S.default_path(s.M, s.P) | extra for s in systems])
        x, q = b.pack(xs, qs)
        outs.append(b.solve(x, q).cpu().numpy())
        b.close()
    assert np.array_equal(outs[0], outs[1])

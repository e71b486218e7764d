"""The three-kernel bin sort (the default where a batch has at most 8192 fine
bins and 2^19 particles) against the radix sort (SE_PATH_RADIX_SORT): both
are the stable counting sort by bin, so the solves agree bit for bit -- one
chunk and many, chunks longer than the minimum, clustered particles (long
runs of equal keys), positions outside the box, and batches of systems."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from se_fast_gridding_b200 import _lib, solver, workloads
    return torch, solver, workloads, _lib


def positions(W, N, L, seed, kind):
    x, q = W.synthetic_system(N, L, seed=seed, charges="uniform")
    rng = np.random.Generator(np.random.Philox(seed))
    if kind == "clustered":   # everything in a corner of 1/64 of the box
        x = x * 0.25 + 0.05 * L
    elif kind == "outside":   # whole boxes away, both signs
        x = x + rng.integers(-2, 3, size=x.size) * L
    return x, q


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("N,M,P,kind", [
    (100, 32, 8, "uniform"),          # one chunk
    (5000, 64, 16, "clustered"),      # long runs of equal keys
    (7000, 48, 12, "outside"),
    (400000, 64, 16, "uniform"),      # the most chunks, each above the minimum
])
def test_bin_sort_equals_radix_sort(env, prec, N, M, P, kind):
    torch, S, W, L = env
    mode = "force" if P % 2 == 0 else "potential"
    x, q = positions(W, N, 1.0, 11 + N, kind)
    xd, qd = torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda")
    path = S.default_path(M, P)
    a = S.SpectralEwald(M, P, 1.0, 8.0, None, mode, prec, N)
    b = S.SpectralEwald(M, P, 1.0, 8.0, None, mode, prec, N, path=path | L.SE_PATH_RADIX_SORT)
    assert a.path == path and b.path == path | L.SE_PATH_RADIX_SORT
    oa, ob = a.solve(xd, qd), b.solve(xd, qd)
    np.testing.assert_array_equal(oa.cpu().numpy(), ob.cpu().numpy())
    assert a.launches < b.launches      # the bin sort takes fewer kernels
    # fewer particles than the plan holds, and the host entry point
    n2 = N // 3
    x2, q2 = positions(W, n2, 1.0, 5 + N, kind)
    np.testing.assert_array_equal(a.solve_host(x2, q2), b.solve_host(x2, q2))
    a.close()
    b.close()


def test_batch_bin_sort_equals_radix_sort(env):
    torch, S, W, L = env
    systems = [S.System(N=800 + 2100 * i, M=(32, 64, 48, 128, 24)[i], P=(8, 16, 12, 16, 6)[i],
                        L=1.0 + 0.25 * i, xi=8.0 / (1.0 + 0.25 * i),
                        mode=("potential", "force")[i % 2]) for i in range(5)]
    paths = [S.default_path(s.M, s.P) for s in systems]
    a = S.BatchSolver(systems, "fp32")
    b = S.BatchSolver(systems, "fp32", paths=[p | L.SE_PATH_RADIX_SORT for p in paths])
    xs, qs = zip(*[positions(W, s.N, s.L, 20 + i, ("uniform", "clustered", "outside")[i % 3])
                   for i, s in enumerate(systems)])
    x, q = a.pack(xs, qs)
    np.testing.assert_array_equal(a.solve(x, q).cpu().numpy(), b.solve(x, q).cpu().numpy())
    a.close()
    b.close()

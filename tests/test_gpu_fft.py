"""The three-pass FP64 k-space step (SE_PATH_FFT3; M = 32, 64, 128) against
cuFFT's D2Z, scaling and Z2D: whole solves agree to rounding in both modes
and precisions, alone and in batches that mix both kinds of group, and the
step entry point (se_kspace) agrees as well."""
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


def rel(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


@pytest.mark.parametrize("M,P", [(32, 8), (64, 12), (128, 16)])
@pytest.mark.parametrize("mode", ["potential", "force"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_three_pass_fft_equals_cufft(env, M, P, mode, prec):
    torch, S, W, L = env
    N = 3000
    x, q = W.synthetic_system(N, 1.7, seed=M + P, charges="uniform")
    xd, qd = torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda")
    path = S.default_path(M, P)
    a = S.SpectralEwald(M, P, 1.7, 9.0 / 1.7, None, mode, prec, N)
    b = S.SpectralEwald(M, P, 1.7, 9.0 / 1.7, None, mode, prec, N, path=path | L.SE_PATH_FFT3)
    oa, ob = a.solve(xd, qd).cpu().numpy(), b.solve(xd, qd).cpu().numpy()
    assert rel(oa, ob) < (1e-13 if prec == "fp64" else 1e-7), rel(oa, ob)
    # the k-space step alone, on the same grid
    g = a.spread(xd, qd)
    ga, gb = g.clone(), g.clone()
    a.kspace(ga)
    b.kspace(gb)
    assert rel(ga.cpu().numpy(), gb.cpu().numpy()) < 1e-13
    a.close()
    b.close()


def test_batch_mixing_three_pass_and_cufft_groups(env):
    """With SE_PATH_FFT3, M = 48 and 96 still go through cuFFT and 32/64/128
    through the three passes, in one batch; every system agrees with the
    cuFFT-only batch, which equals each single-system solve bit for bit."""
    torch, S, W, L = env
    Ms = [32, 48, 64, 96, 128, 64]
    systems = [S.System(N=900 + 500 * i, M=M, P=(8, 12, 16)[i % 3], L=1.0 + 0.3 * i,
                        xi=9.0 / (1.0 + 0.3 * i), mode=("potential", "force")[i % 2])
               for i, M in enumerate(Ms)]
    xs, qs = zip(*[W.synthetic_system(s.N, s.L, seed=50 + i) for i, s in enumerate(systems)])
    a = S.BatchSolver(systems, "fp64")
    b = S.BatchSolver(systems, "fp64",
                      paths=[S.default_path(s.M, s.P) | L.SE_PATH_FFT3 for s in systems])
    x, q = a.pack(xs, qs)
    oa, ob = a.solve(x, q), b.solve(x, q)
    for i, (pa, pb) in enumerate(zip(a.split(oa), b.split(ob))):
        assert rel(pa.cpu().numpy(), pb.cpu().numpy()) < 1e-13, i
        s = systems[i]
        one = S.SpectralEwald(s.M, s.P, s.L, s.xi, None, s.mode, "fp64", s.N)
        np.testing.assert_array_equal(
            one.solve(torch.tensor(xs[i], device="cuda"), torch.tensor(qs[i], device="cuda"))
            .cpu().numpy(), pa.cpu().numpy())
        one.close()
    a.close()
    b.close()

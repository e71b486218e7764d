"""Parity of the device-resident solve (se_gpu.h) with the reference.

FP64: within 1e-12 relative RMS of the reference's spectral_ewald() (golden
vectors) and of the CPU oracle at identical P, m, eta, M.
FP32 (compensated): within 1e-6 relative RMS of the FP64 path and of the FP64
direct k-space Ewald sum.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-6


@pytest.fixture(scope="module")
def S():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from se_fast_gridding_b200 import solver
    return solver


def cuda(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def host(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    import oracle as O
    return O.rel_rms(a, b)


@pytest.mark.parametrize("N", [10, 100])
@pytest.mark.parametrize("P", [8, 12, 16, 21])
@pytest.mark.parametrize("mode", ["potential", "force"])
def test_fp64_matches_reference_spectral_ewald(S, N, P, mode):
    """test_accuracy.c's system (atoms.txt, L = 3.1814, xi = 8, M = 108)."""
    g = load_golden("test_accuracy.npz")
    x, q = g[f"N{N}/x"], g[f"N{N}/q"]
    M, m = int(g[f"N{N}/P{P}/M"]), float(g[f"N{N}/P{P}/m"])
    se = S.SpectralEwald(M, P, 3.1814, 8.0, m, mode=mode, precision="fp64", max_particles=N)
    out = host(se.solve(cuda(x), cuda(q)))
    ref = g[f"N{N}/P{P}/" + ("phi" if mode == "potential" else "force")]
    assert rel(out, ref) < FP64_TOL, rel(out, ref)
    # host-buffer entry point: identical numbers
    out_h = se.solve_host(x, q)
    np.testing.assert_array_equal(out_h, out)
    se.close()


@pytest.mark.parametrize("N,mode", [(60_000, "force"), (150_000, "potential")])
def test_solve_host_staged_pageable_and_pinned(S, N, mode):
    """se_solve_host with host arrays of 1 MiB and more: pageable arrays go
    through the pinned chunks of the host staging (threaded host copies),
    pinned ones through the stream; both give the device solve's numbers bit
    for bit, also with pinned inputs and a pageable output and the reverse."""
    import oracle as O
    import torch
    x, q = O.synthetic_system(N, 1.0, seed=N, charges="uniform")
    se = S.SpectralEwald(64, 12, 1.0, 10.0, None, mode, "fp32", N)
    ref = host(se.solve(cuda(x), cuda(q)))
    np.testing.assert_array_equal(se.solve_host(x, q), ref)        # pageable in and out
    xp = torch.tensor(x).pin_memory()
    qp = torch.tensor(q).pin_memory()
    op = torch.empty(ref.size, dtype=torch.float64).pin_memory()
    se.solve_host_ptr(N, xp.data_ptr(), qp.data_ptr(), op.data_ptr())   # pinned in and out
    np.testing.assert_array_equal(op.numpy(), ref)
    out = np.full(ref.size, np.nan)
    se.solve_host_ptr(N, xp.data_ptr(), qp.data_ptr(), out.ctypes.data)  # pinned in, pageable out
    np.testing.assert_array_equal(out, ref)
    op.fill_(float("nan"))
    xc, qc = np.ascontiguousarray(x), np.ascontiguousarray(q)
    se.solve_host_ptr(N, xc.ctypes.data, qc.ctypes.data, op.data_ptr())  # pageable in, pinned out
    np.testing.assert_array_equal(op.numpy(), ref)
    se.close()


def test_fp64_reference_error_figures(S):
    """abs-RMS vs the direct sum, as test_accuracy prints it."""
    import oracle as O
    g = load_golden("test_accuracy.npz")
    x, q = g["N10/x"], g["N10/q"]
    M, m = int(g["N10/P16/M"]), float(g["N10/P16/m"])
    se = S.SpectralEwald(M, 16, 3.1814, 8.0, m, "potential", "fp64", 10)
    phi = host(se.solve(cuda(x), cuda(q)))
    sf = S.SpectralEwald(M, 16, 3.1814, 8.0, m, "force", "fp64", 10)
    f = host(sf.solve(cuda(x), cuda(q)))
    assert 2.6e-10 < O.abs_rms(g["N10/direct_phi"], phi) < 2.7e-10
    assert 4.9e-9 < O.abs_rms(f, g["N10/direct_force"]) < 5.0e-9


def test_c1_plain_fp64(S):
    """N=100, M=32, P=21, xi=8, L=1, FP64."""
    import oracle as O
    g = load_golden("c1.npz")
    x, q = g["x"], g["q"]
    se = S.SpectralEwald(32, 21, 1.0, 8.0, O.c1_params(21), "potential", "fp64", 100)
    phi = host(se.solve(cuda(x), cuda(q)))
    assert rel(phi, g["phi_ref"]) < FP64_TOL
    assert rel(phi, g["phi_direct"]) < 1e-11
    sf = S.SpectralEwald(32, 21, 1.0, 8.0, O.c1_params(21), "force", "fp64", 100)
    f = host(sf.solve(cuda(x), cuda(q)))
    assert rel(f, g["force_ref"]) < FP64_TOL


@pytest.fixture(scope="module")
def c2(S):
    import oracle as O
    g = load_golden("c2.npz")
    N = 100_000
    x, q = O.synthetic_system(N, 1.0, seed=1, charges="uniform")
    np.testing.assert_array_equal(x[g["targets"]], g["x_check"])
    return g, x, q


def test_c2_fp64_force_and_potential(S, c2):
    from conftest import check_digest
    import oracle as O
    g, x, q = c2
    N, m = len(q), O.c1_params(16)
    t = g["targets"]
    sf = S.SpectralEwald(128, 16, 1.0, 20.0, m, "force", "fp64", N)
    f = host(sf.solve(cuda(x), cuda(q)))
    fsub = np.concatenate([f[t + d * N] for d in range(3)])
    assert rel(fsub, g["force_ref"]) < FP64_TOL
    check_digest(g, "force_ref_all", f, 1e-11)
    sp = S.SpectralEwald(128, 16, 1.0, 20.0, m, "potential", "fp64", N)
    phi = host(sp.solve(cuda(x), cuda(q)))
    assert rel(phi[t], g["phi_ref"]) < FP64_TOL
    check_digest(g, "phi_ref_all", phi, 1e-11)


def test_c2_fp32_accuracy(S, c2):
    """FP32 gridding with compensated sums vs FP64 and vs the direct sum."""
    import oracle as O
    g, x, q = c2
    N, m = len(q), O.c1_params(16)
    t = g["targets"]
    for mode, key in (("force", "force"), ("potential", "phi")):
        s64 = S.SpectralEwald(128, 16, 1.0, 20.0, m, mode, "fp64", N)
        s32 = S.SpectralEwald(128, 16, 1.0, 20.0, m, mode, "fp32", N)
        o64 = host(s64.solve(cuda(x), cuda(q)))
        o32 = host(s32.solve(cuda(x), cuda(q)))
        assert rel(o32, o64) < FP32_TOL, (mode, rel(o32, o64))
        w = 3 if mode == "force" else 1
        sub = np.concatenate([o32[t + d * N] for d in range(w)])
        assert rel(sub, g[f"{key}_direct"]) < FP32_TOL, (mode, rel(sub, g[f"{key}_direct"]))


def test_spread_grid_equals_oracle_wrap(S):
    """se_spread = SE_FGG_grid_split + SE_FGG_wrap_fcn (transposed layout)."""
    import oracle as O
    for M, P, N in ((16, 8, 200), (12, 16, 50), (20, 21, 300), (33, 7, 500)):
        x, q = O.synthetic_system(N, 1.0, seed=M + P, charges="uniform")
        m = 0.9 * np.sqrt(O.PI * P)
        se = S.SpectralEwald(M, P, 1.0, 6.0, m, "potential", "fp64", N)
        grid = host(se.spread(cuda(x), cuda(q)))
        s = O.Setup(M=M, P=P, L=1.0, xi=6.0, m=m, N=N)
        p = s.params()
        zs = O.base_gaussian(p)
        ex = O.expand_all(p, x, 3, False)
        Hper = O.wrap(p, O.grid_split(p, q, zs, ex), 3)
        ref = Hper.reshape(M, M, M).transpose(2, 1, 0)
        assert rel(grid, ref) < FP64_TOL, (M, P, rel(grid, ref))
        # and the interpolation of a given grid = extend + int_split
        rng = np.random.Generator(np.random.Philox(M))
        field = rng.standard_normal((M, M, M))
        phi = host(se.interp(cuda(x), cuda(q), cuda(field)))
        Hp = np.ascontiguousarray(field.transpose(2, 1, 0)).reshape(-1)
        phi_o = O.int_split(p, O.extend(p, Hp, 3), zs, ex)
        assert rel(phi, phi_o) < FP64_TOL, (M, P)


@pytest.mark.parametrize("M,P,N,clusters", [(32, 16, 3000, 0), (32, 1, 500, 0), (48, 5, 2000, 0),
                                             (64, 12, 20000, 4), (32, 9, 4000, 2),
                                             (64, 16, 30000, 0)])
def test_spread_tile_aligned_rows_equal_oracle(S, M, P, N, clusters):
    """Grids cut into whole 16^3 tiles with P <= 16 take the tile-aligned
    spread: every P, tiles at the periodic seam (M = 32: two tiles per axis),
    crowded clusters; FP64 within 1e-12 of the oracle's grid + wrap, FP32
    within the FP32 bound of the FP64 grid."""
    import oracle as O
    x, q = O.synthetic_system(N, 1.0, seed=M * P + N, charges="uniform", clusters=clusters,
                              sigma=0.03)
    m = 0.9 * np.sqrt(O.PI * P)
    s = O.Setup(M=M, P=P, L=1.0, xi=6.0, m=m, N=N)
    p = s.params()
    Hper = O.wrap(p, O.grid_split(p, q, O.base_gaussian(p), O.expand_all(p, x, 3, False)), 3)
    ref = Hper.reshape(M, M, M).transpose(2, 1, 0)
    se = S.SpectralEwald(M, P, 1.0, 6.0, m, "potential", "fp64", N)
    g64 = host(se.spread(cuda(x), cuda(q)))
    assert rel(g64, ref) < FP64_TOL, rel(g64, ref)
    s32 = S.SpectralEwald(M, P, 1.0, 6.0, m, "potential", "fp32", N)
    g32 = host(s32.spread(cuda(x), cuda(q)))
    assert rel(g32, g64) < FP32_TOL, rel(g32, g64)
    # deterministic: a second spread is bit-identical
    np.testing.assert_array_equal(host(s32.spread(cuda(x), cuda(q))), g32)
    # interpolation of a given grid = extend + int_split (window pair sums)
    rng = np.random.Generator(np.random.Philox(M + P))
    field = rng.standard_normal((M, M, M))
    Hp = np.ascontiguousarray(field.transpose(2, 1, 0)).reshape(-1)
    phi_o = O.int_split(p, O.extend(p, Hp, 3), O.base_gaussian(p), O.expand_all(p, x, 3, False))
    phi64 = host(se.interp(cuda(x), cuda(q), cuda(field)))
    assert rel(phi64, phi_o) < FP64_TOL, rel(phi64, phi_o)
    phi32 = host(s32.interp(cuda(x), cuda(q), cuda(field)))
    assert rel(phi32, phi_o) < 1e-6, rel(phi32, phi_o)
    # caller grids that are not 16-byte aligned give the same numbers
    import torch
    buf = torch.zeros(M ** 3 + 1, dtype=torch.float64, device="cuda")
    np.testing.assert_array_equal(host(se.spread(cuda(x), cuda(q), grid=buf[1:])),
                                  g64.reshape(-1))
    buf[1:] = cuda(field).reshape(-1)
    np.testing.assert_array_equal(host(se.interp(cuda(x), cuda(q), buf[1:])), phi64)
    np.testing.assert_array_equal(host(s32.interp(cuda(x), cuda(q), buf[1:])), phi32)
    se.close()
    s32.close()
    # full FORCE solve against the oracle pipeline
    f = S.SpectralEwald(M, P, 1.0, 6.0, m, "force", "fp64", N)
    got = host(f.solve(cuda(x), cuda(q)))
    ref = O.spectral_ewald(x, q, M, P, m, 1.0, 6.0, "force")
    assert rel(got, ref) < FP64_TOL, rel(got, ref)
    f32 = S.SpectralEwald(M, P, 1.0, 6.0, m, "force", "fp32", N)
    assert rel(host(f32.solve(cuda(x), cuda(q))), ref) < 1e-6
    f.close()
    f32.close()


@pytest.mark.parametrize("N", [60_000, 8_000])
def test_spread_split_tiles_equal_oracle(S, N):
    """Crowded tiles are summed in parts of at most 8192 candidates per warp
    block whose sums are added in part order: at M = 32 a block's bins hold
    9/16 of the particles, so 60,000 clustered particles split the tiles near
    the cluster into several parts (8,000: one part).
    FP64 within 1e-12 of the oracle's grid + wrap and full FORCE solve, FP32
    within its bound, the same bits on a second solve and inside a batch."""
    import oracle as O
    M, P = 32, 16
    x, q = O.synthetic_system(N, 1.0, seed=N, charges="uniform", clusters=1, sigma=0.05)
    m = S.default_m(P)
    s = O.Setup(M=M, P=P, L=1.0, xi=6.0, m=m, N=N)
    p = s.params()
    Hper = O.wrap(p, O.grid_split(p, q, O.base_gaussian(p), O.expand_all(p, x, 3, False)), 3)
    ref = Hper.reshape(M, M, M).transpose(2, 1, 0)
    se = S.SpectralEwald(M, P, 1.0, 6.0, m, "force", "fp64", N)
    g64 = host(se.spread(cuda(x), cuda(q)))
    assert rel(g64, ref) < FP64_TOL, rel(g64, ref)
    s32 = S.SpectralEwald(M, P, 1.0, 6.0, m, "force", "fp32", N)
    g32 = host(s32.spread(cuda(x), cuda(q)))
    assert rel(g32, g64) < FP32_TOL, rel(g32, g64)
    np.testing.assert_array_equal(host(s32.spread(cuda(x), cuda(q))), g32)
    f64 = host(se.solve(cuda(x), cuda(q)))
    fref = O.spectral_ewald(x, q, M, P, m, 1.0, 6.0, "force")
    assert rel(f64, fref) < FP64_TOL, rel(f64, fref)
    f32 = host(s32.solve(cuda(x), cuda(q)))
    assert rel(f32, fref) < FP32_TOL, rel(f32, fref)
    np.testing.assert_array_equal(host(s32.solve(cuda(x), cuda(q))), f32)
    # in a batch beside a second (uncrowded) system: the same bits
    x2, q2 = O.synthetic_system(3000, 2.0, seed=5, charges="uniform")
    systems = [S.System(N, M, P, 1.0, 6.0, m, "force"), S.System(3000, 48, 12, 2.0, 4.0, None, "force")]
    for prec, one in (("fp64", f64), ("fp32", f32)):
        b = S.BatchSolver(systems, precision=prec)
        xb, qb = b.pack([x, x2], [q, q2])
        outs = b.split(b.solve(xb, qb))
        np.testing.assert_array_equal(host(outs[0]), one)
        b.close()
    se.close()
    s32.close()


def test_fp32_spread_grid(S):
    import oracle as O
    M, P, N = 64, 12, 20000
    x, q = O.synthetic_system(N, 1.0, seed=9, charges="pm1")
    s64 = S.SpectralEwald(M, P, 1.0, 10.0, None, "potential", "fp64", N)
    s32 = S.SpectralEwald(M, P, 1.0, 10.0, None, "potential", "fp32", N)
    g64 = host(s64.spread(cuda(x), cuda(q)))
    g32 = host(s32.spread(cuda(x), cuda(q)))
    # FP32 factors carry ~3 roundings per product, and each FP32 partial sum
    # covers up to 512 particles: the FP32 bound
    assert rel(g32, g64) < FP32_TOL, rel(g32, g64)


@pytest.mark.parametrize("N,nkeys", [(1, 1), (1000, 1), (5000, 37), (100_000, 4096),
                                     (300_000, 70_000), (2_000_000, 262_144)])
def test_counting_sort_bit_exact(S, N, nkeys):
    import torch
    import oracle as O
    rng = np.random.Generator(np.random.Philox(N + nkeys))
    keys = rng.integers(0, nkeys, size=N).astype(np.int32)
    perm, offs = S.counting_sort(torch.tensor(keys, device="cuda"), nkeys)
    p_o, off_o = O.counting_sort(keys, nkeys)
    np.testing.assert_array_equal(perm.cpu().numpy(), p_o)
    np.testing.assert_array_equal(offs.cpu().numpy(), off_o)


def test_batch_equals_single_systems(S):
    """One batched launch set gives each system's own single-plan result."""
    import oracle as O
    systems, xs, qs = [], [], []
    rng = np.random.Generator(np.random.Philox(21))
    for i in range(7):
        N = int(rng.integers(50, 3000))
        P = int(rng.choice([8, 12, 16]))
        L = float(rng.uniform(1, 4))
        M = 32 if i % 2 else 24
        mode = "force" if i % 3 == 0 else "potential"
        systems.append(S.System(N=N, M=M, P=P, L=L, xi=8.0 / L, mode=mode))
        x, q = O.synthetic_system(N, L, seed=100 + i)
        xs.append(x)
        qs.append(q)
    for prec in ("fp64", "fp32"):
        b = S.BatchSolver(systems, precision=prec)
        xb, qb = b.pack(xs, qs)
        outs = b.split(b.solve(xb, qb))
        for s, x, q, o in zip(systems, xs, qs, outs):
            se = S.SpectralEwald(s.M, s.P, s.L, s.xi, None, s.mode, prec, s.N)
            one = host(se.solve(cuda(x), cuda(q)))
            np.testing.assert_array_equal(host(o), one)
            if prec == "fp64":
                ref = O.spectral_ewald(x, q, s.M, s.P, S.default_m(s.P), s.L, s.xi, s.mode)
                assert rel(host(o), ref) < FP64_TOL


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_plans_of_different_P_coexist(S, prec):
    """A plan created later with a smaller interpolation window must not
    break an earlier plan's launches (per-function launch limits are
    process-wide)."""
    import oracle as O
    x, q = O.synthetic_system(3000, 1.0, seed=31)
    xd, qd = cuda(x), cuda(q)
    big = S.SpectralEwald(32, 16, 1.0, 8.0, None, "force", prec, 3000)
    first = host(big.solve(xd, qd))
    small = [S.SpectralEwald(32, P, 1.0, 8.0, None, "force", prec, 3000) for P in (8, 12, 4)]
    for s in small:
        s.solve(xd, qd)
    np.testing.assert_array_equal(host(big.solve(xd, qd)), first)
    for s in small + [big]:
        s.close()


def test_energy(S):
    import torch
    rng = np.random.Generator(np.random.Philox(8))
    phi, q = rng.standard_normal(123457), rng.standard_normal(123457)
    e = S.energy(cuda(phi), cuda(q)).item()
    assert abs(e - 0.5 * np.dot(phi, q)) < 1e-10 * np.abs(phi * q).sum()
    assert torch.cuda.is_available()


def test_edge_positions_and_empty(S):
    import oracle as O
    # particles exactly on 0 and on L, and an empty solve
    x = np.array([0.0, 1.0, 0.5, 0.999999999999, 0.0, 0.25,
                  0.0, 1.0, 0.5, 0.0, 1.0, 0.75,
                  1.0, 0.0, 0.5, 0.5, 0.0, 1.0])
    q = np.array([1.0, -1.0, 0.5, -0.5, 0.25, -0.25])
    # x = L is the periodic image of x = 0 (and exactly so: L = M h); the
    # reference's padded grid only holds [0, L) for even P, so the oracle
    # gets the image inside the box
    x_in = np.where(x == 1.0, 0.0, x)
    for P in (7, 8):
        m = 0.94 * np.sqrt(O.PI * P)
        se = S.SpectralEwald(16, P, 1.0, 5.0, m, "potential", "fp64", 6)
        phi = host(se.solve(cuda(x), cuda(q)))
        ref = O.spectral_ewald(x_in, q, 16, P, m, 1.0, 5.0, "potential")
        assert rel(phi, ref) < FP64_TOL
        empty = se.solve(cuda(np.zeros(0)), cuda(np.zeros(0)))
        assert empty.numel() == 0


def test_nonfinite_position_reported(S):
    import se_fast_gridding_b200 as pkg
    se = S.SpectralEwald(16, 8, 1.0, 5.0, None, "potential", "fp64", 4)
    x = np.array([0.1, np.nan, 0.3, 0.4, 0.1, 0.2, 0.3, 0.4, 0.1, 0.2, 0.3, 0.4])
    with pytest.raises(pkg.SEError):
        se.solve_host(x, np.ones(4))
    # the plan stays usable
    x[1] = 0.2
    out = se.solve_host(x, np.ones(4))
    assert np.isfinite(out).all()


@pytest.mark.parametrize("eps", [1e-5, 1e-8, 1e-11])
def test_chosen_params_reach_the_target(S, eps):
    """se_choose_params' P and M give an absolute RMS error vs the direct
    k-space sum within a small factor of the target (the estimate is the
    reference's own, SE_init_params)."""
    import oracle as O
    g = load_golden("c1.npz")
    x, q = g["x"], g["q"]
    M, P, m = S.choose_params(eps, 1.0, 8.0, q, "potential")
    se = S.SpectralEwald(M, P, 1.0, 8.0, m, "potential", "fp64", len(q))
    phi = host(se.solve(cuda(x), cuda(q)))
    err = O.abs_rms(phi, g["phi_direct"])
    assert err < 10 * eps, (M, P, err)
    se.close()


def test_fp32_fft32_mode(S, c2):
    """SE_FP32_FFT32 (FP32 FFTs, Z in FP64): C2 within the FP32 bound of the
    FP64 path and of the direct sum."""
    import oracle as O
    g, x, q = c2
    N, m = len(q), O.c1_params(16)
    t = g["targets"]
    for mode, key in (("force", "force"), ("potential", "phi")):
        s64 = S.SpectralEwald(128, 16, 1.0, 20.0, m, mode, "fp64", N)
        s32 = S.SpectralEwald(128, 16, 1.0, 20.0, m, mode, "fp32-fft32", N)
        o64 = host(s64.solve(cuda(x), cuda(q)))
        o32 = host(s32.solve(cuda(x), cuda(q)))
        assert rel(o32, o64) < FP32_TOL, (mode, rel(o32, o64))
        w = 3 if mode == "force" else 1
        sub = np.concatenate([o32[t + d * N] for d in range(w)])
        assert rel(sub, g[f"{key}_direct"]) < FP32_TOL


def test_fp32_fft32_batch_and_steps(S):
    import oracle as O
    systems, xs, qs = [], [], []
    for i in range(4):
        N = 700 + 400 * i
        M = (32, 24)[i % 2]          # tile-aligned and general kernels together
        L = 1.0 + 0.3 * i
        systems.append(S.System(N=N, M=M, P=(8, 12)[i % 2], L=L, xi=8.0 / L,
                                mode=("force", "potential")[i % 2]))
        x, q = O.synthetic_system(N, L, seed=60 + i)
        xs.append(x)
        qs.append(q)
    b = S.BatchSolver(systems, precision="fp32-fft32")
    xb, qb = b.pack(xs, qs)
    outs = b.split(b.solve(xb, qb))
    for s, x, q, o in zip(systems, xs, qs, outs):
        one = host(S.SpectralEwald(s.M, s.P, s.L, s.xi, None, s.mode, "fp32-fft32",
                                   s.N).solve(cuda(x), cuda(q)))
        np.testing.assert_array_equal(host(o), one)
        ref = O.spectral_ewald(x, q, s.M, s.P, S.default_m(s.P), s.L, s.xi, s.mode)
        assert rel(one, ref) < FP32_TOL
    # the k-space step keeps the caller's FP64 grid contract
    s = systems[0]
    x, q = xs[0], qs[0]
    p64 = S.SpectralEwald(s.M, s.P, s.L, s.xi, None, s.mode, "fp64", s.N)
    p32 = S.SpectralEwald(s.M, s.P, s.L, s.xi, None, s.mode, "fp32-fft32", s.N)
    g64 = p64.kspace(p64.spread(cuda(x), cuda(q)))
    g32 = p32.kspace(p32.spread(cuda(x), cuda(q)))
    assert g32.dtype == g64.dtype
    assert rel(host(g32), host(g64)) < FP32_TOL

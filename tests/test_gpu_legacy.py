"""Parity of the legacy C ABI (SE_fgg.h / SE_general.h names) on the GPU.

Every entry point is called through libse_gpu.so and compared with the
reference's own outputs (tests/golden/fgg_steps.npz, made from SE_fast_gridding
compiled from source) and with the CPU oracle.  Bar: 1e-12 relative (FP64).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import check_digest, load_golden

pytestmark = pytest.mark.gpu

TOL = 1e-12
CASES = [(12, 7), (12, 8), (16, 12), (12, 16), (20, 21)]


@pytest.fixture(scope="module")
def F():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from se_fast_gridding_b200 import fgg
    fgg.lib()
    return fgg


def setup_case(F, g, M, P):
    import oracle as O
    m = 0.95 * np.sqrt(O.PI * P)
    opt, p = F.fcn_params(M, P, 1.0, 4.0, m, 10)
    return p


@pytest.mark.parametrize("where", ["host", "managed", "cuda"])
@pytest.mark.parametrize("case", CASES)
def test_fgg_steps_3p(F, case, where):
    import torch
    g = load_golden("fgg_steps.npz")
    M, P = case
    tag = f"M{M}P{P}"
    x, q = g["x"].copy(), g["q"].copy()
    if where == "cuda":
        xs, qs = torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda")
    else:
        xs, qs = x, q
    p = setup_case(F, g, M, P)
    st = F.state(xs, qs)
    w = F.Work(p, force=False, where=where)
    wf = F.Work(p, force=True, where=where)
    for ww in (w, wf):
        F.call("SE_FGG_base_gaussian", C.byref(ww.s), C.byref(p))
    np.testing.assert_allclose(w.get("zs"), g[f"{tag}/zs"], rtol=1e-13)
    F.call("SE_FGG_expand_all", C.byref(w.s), C.byref(st), C.byref(p))
    F.call("SE_FGG_expand_all_SSE_force", C.byref(wf.s), C.byref(st), C.byref(p))
    np.testing.assert_array_equal(w.get("idx"), g[f"{tag}/exp_idx"])
    for k in ("zx", "zy", "zz"):
        np.testing.assert_allclose(w.get(k), g[f"{tag}/exp_{k}"], rtol=1e-13)
    for k in ("zx", "zy", "zz", "zfx", "zfy", "zfz"):
        np.testing.assert_allclose(wf.get(k), g[f"{tag}/expf_{k}"], rtol=1e-13, atol=1e-300)
    # every spread entry point (dispatchers and leaves compute the same sum)
    for fn in ("SE_FGG_grid_split", "SE_FGG_grid_split_SSE_dispatch",
               "SE_FGG_grid_split_AVX_dispatch", "SE_FGG_grid_split_AVX_P16"):
        F.call("SE_fp_set_zero", w.s.H, p.npdims[0] * p.npdims[1] * p.npdims[2])
        F.call(fn, C.byref(w.s), C.byref(st), C.byref(p))
        check_digest(g, f"{tag}/grid_split", w.get("H"), TOL)
    F.call("SE_fp_set_zero", w.s.H, p.npdims[0] * p.npdims[1] * p.npdims[2])
    F.call("SE_FGG_grid", C.byref(w.s), C.byref(st), C.byref(p))
    check_digest(g, f"{tag}/grid_vanilla", w.get("H"), TOL)
    F.call("SE_fp_set_zero", wf.s.H, p.npdims[0] * p.npdims[1] * p.npdims[2])
    F.call("SE_FGG_grid_split_AVX_dispatch_force", C.byref(wf.s), C.byref(st), C.byref(p))
    check_digest(g, f"{tag}/grid_force", wf.get("H"), TOL)
    # wrap (+= into a column-major periodic grid)
    F.call("SE_fp_set_zero", w.s.H, p.npdims[0] * p.npdims[1] * p.npdims[2])
    F.call("SE_FGG_grid_split", C.byref(w.s), C.byref(st), C.byref(p))
    Hper = np.zeros(M ** 3)
    F.call("SE_FGG_wrap_fcn", F.dptr(Hper), C.byref(w.s), C.byref(p))
    ref = g[f"{tag}/wrap"]
    np.testing.assert_allclose(Hper, ref, rtol=0, atol=TOL * np.abs(ref).max())
    # extend a field, then every interpolation entry point
    field = g[f"{tag}/field"].copy()
    for ww in (w, wf):
        F.call("SE_FGG_extend_fcn", C.byref(ww.s), F.dptr(field), C.byref(p))
    check_digest(g, f"{tag}/extend", w.get("H"), 0.0)
    for fn in ("SE_FGG_int_split", "SE_FGG_int_split_SSE_dispatch", "SE_FGG_int_split_AVX_dispatch"):
        phi = np.zeros(10)
        F.call(fn, F.dptr(phi), C.byref(w.s), C.byref(p))
        np.testing.assert_allclose(phi, g[f"{tag}/int_split"], rtol=TOL)
    phi = np.zeros(10)
    F.call("SE_FGG_int", F.dptr(phi), C.byref(w.s), C.byref(st), C.byref(p))
    np.testing.assert_allclose(phi, g[f"{tag}/int_vanilla"], rtol=TOL)
    for fn in ("SE_FGG_int_split_force", "SE_FGG_int_split_AVX_dispatch_force",
               "SE_FGG_int_split_SSE_dispatch_force"):
        f = np.zeros(30)
        F.call(fn, F.dptr(f), C.byref(st), C.byref(wf.s), C.byref(p))
        ref = g[f"{tag}/int_force_split"]
        np.testing.assert_allclose(f, ref, rtol=0, atol=TOL * np.abs(ref).max())
    f = np.zeros(30)
    F.call("SE_FGG_int_force", F.dptr(f), C.byref(w.s), C.byref(st), C.byref(p))
    ref = g[f"{tag}/int_force_vanilla"]
    np.testing.assert_allclose(f, ref, rtol=0, atol=TOL * np.abs(ref).max())
    # calc_energy
    phi = g[f"{tag}/int_split"].copy()
    e = F.lib().calc_energy(F.state(x, q, phi), 10)
    assert abs(e - float(g[f"{tag}/energy"])) <= 1e-13 * abs(float(g[f"{tag}/energy"]))
    w.free()
    wf.free()


def test_int_avx_unroll4_accumulates(F):
    """SE_FGG_int_split_AVX (SE_fgg.c:1768-1858) adds into phi (:1856); the
    dispatcher routes P = 12 there, P = 16 / 8 elsewhere."""
    g = load_golden("fgg_steps.npz")
    M, P = 16, 12
    tag = f"M{M}P{P}"
    p = setup_case(F, g, M, P)
    w = F.Work(p, where="host")
    st = F.state(g["x"].copy(), g["q"].copy())
    F.call("SE_FGG_base_gaussian", C.byref(w.s), C.byref(p))
    F.call("SE_FGG_expand_all", C.byref(w.s), C.byref(st), C.byref(p))
    field = g[f"{tag}/field"].copy()
    F.call("SE_FGG_extend_fcn", C.byref(w.s), F.dptr(field), C.byref(p))
    phi = np.ones(10)
    F.call("SE_FGG_int_split_AVX_dispatch", F.dptr(phi), C.byref(w.s), C.byref(p))
    np.testing.assert_allclose(phi, 1.0 + g[f"{tag}/int_split"], rtol=TOL)
    phi = np.ones(10)
    F.call("SE_FGG_int_split", F.dptr(phi), C.byref(w.s), C.byref(p))
    np.testing.assert_allclose(phi, g[f"{tag}/int_split"], rtol=TOL)


def test_grid_split_contention(F):
    """The legacy spread scatters with FP64 atomics, one CTA per particle:
    40,000 particles in one Gaussian cluster of width 0.01 L at M = 32,
    P = 16 put thousands of concurrent contributions on the same cells.  The
    padded grid, its wrap and the interpolation of an extended field back to
    the particles are within 1e-12 of the oracle, which sums in the
    reference's order (SE_fgg.c:3866-4028, 327-352, 417-443, 1024-1100)."""
    import oracle as O
    import torch
    N, M, P, xi = 40_000, 32, 16, 4.0
    x, q = O.synthetic_system(N, 1.0, seed=11, charges="pm1", clusters=1, sigma=0.01)
    m = 0.95 * np.sqrt(O.PI * P)
    _, p = F.fcn_params(M, P, 1.0, xi, m, N)
    po = O.Setup(M=M, P=P, L=1.0, xi=xi, m=m, N=N).params()
    zs = O.base_gaussian(po)
    ex = O.expand_all(po, x, 3, False)
    H_ref = O.grid_split(po, q, zs, ex)
    w = F.Work(p, force=False, where="cuda")
    st = F.state(torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda"))
    F.call("SE_FGG_base_gaussian", C.byref(w.s), C.byref(p))
    F.call("SE_FGG_expand_all", C.byref(w.s), C.byref(st), C.byref(p))
    F.call("SE_fp_set_zero", w.s.H, p.npdims[0] * p.npdims[1] * p.npdims[2])
    F.call("SE_FGG_grid_split", C.byref(w.s), C.byref(st), C.byref(p))
    H = w.get("H")
    assert O.rel_rms(H, H_ref) < TOL, O.rel_rms(H, H_ref)
    Hper = np.zeros(M ** 3)
    F.call("SE_FGG_wrap_fcn", F.dptr(Hper), C.byref(w.s), C.byref(p))
    Hper_ref = O.wrap(po, H_ref, 3)
    assert O.rel_rms(Hper, Hper_ref) < TOL, O.rel_rms(Hper, Hper_ref)
    # the wrapped grid as the field: extend it and interpolate at the particles
    F.call("SE_FGG_extend_fcn", C.byref(w.s), F.dptr(Hper), C.byref(p))
    phi = np.zeros(N)
    F.call("SE_FGG_int_split", F.dptr(phi), C.byref(w.s), C.byref(p))
    phi_ref = O.int_split(po, O.extend(po, Hper_ref, 3), zs, ex)
    assert O.rel_rms(phi, phi_ref) < TOL, O.rel_rms(phi, phi_ref)
    w.free()


@pytest.mark.parametrize("case", CASES)
def test_fgg_steps_2p(F, case):
    g = load_golden("fgg_steps.npz")
    M, P = case
    tag = f"M{M}P{P}"
    x, q = g["x"].copy(), g["q"].copy()
    p3 = setup_case(F, g, M, P)
    p = F.pack_params(10, M, M, M, P, p3.c, 1.0 / M, float(g[f"{tag}/p2_a"]))
    st = F.state(x, q)
    w = F.Work(p, where="host")
    F.call("SE_FGG_base_gaussian", C.byref(w.s), C.byref(p))
    F.call("SE2P_FGG_expand_all", C.byref(w.s), C.byref(st), C.byref(p))
    np.testing.assert_array_equal(w.get("idx"), g[f"{tag}/exp2p_idx"])
    for k in ("zx", "zy", "zz"):
        np.testing.assert_allclose(w.get(k), g[f"{tag}/exp2p_{k}"], rtol=1e-13)
    F.call("SE_FGG_grid_split", C.byref(w.s), C.byref(st), C.byref(p))
    Hper = np.zeros(M * M * p.npdims[2])
    F.call("SE2P_FGG_wrap_fcn", F.dptr(Hper), C.byref(w.s), C.byref(p))
    check_digest(g, f"{tag}/wrap2p", Hper, TOL)
    field = g[f"{tag}/field2p"].copy()
    F.call("SE2P_FGG_extend_fcn", C.byref(w.s), F.dptr(field), C.byref(p))
    check_digest(g, f"{tag}/extend2p", w.get("H"), 0.0)


ONE_P = [((12, 12, 12), 7), ((12, 12, 12), 8), ((16, 16, 16), 12), ((12, 12, 12), 16),
         ((20, 20, 20), 21), ((10, 12, 14), 8)]


@pytest.mark.parametrize("case", ONE_P)
def test_fgg_steps_1p(F, case):
    """SE1P (x and y free, z periodic) against a -DONE_PERIODIC build of the
    reference: SE1P_FGG_pack_params, the 1P expansion, the split spread,
    SE1P_FGG_wrap_fcn (whose overlapping column-major map sums in the
    reference's order: exact), SE1P_FGG_extend_fcn and the interpolation."""
    g = load_golden("fgg_1p.npz")
    dims, P = case
    tag = "D{}x{}x{}P{}".format(*dims, P)
    x, q = g["x"].copy(), g["q"].copy()
    M0, M1, M2 = dims
    p = F.pack_params(10, M0, M1, M2, P, float(g[f"{tag}/c"]), 1.0 / M2, float(g[f"{tag}/a"]),
                      float(g[f"{tag}/b"]))
    assert p.d == float(g[f"{tag}/d"])
    st = F.state(x, q)
    w = F.Work(p, where="host")
    F.call("SE_FGG_base_gaussian", C.byref(w.s), C.byref(p))
    F.call("SE1P_FGG_expand_all", C.byref(w.s), C.byref(st), C.byref(p))
    np.testing.assert_array_equal(w.get("idx"), g[f"{tag}/exp_idx"])
    for k in ("zx", "zy", "zz"):
        np.testing.assert_allclose(w.get(k), g[f"{tag}/exp_{k}"], rtol=1e-13)
    F.call("SE_FGG_grid_split", C.byref(w.s), C.byref(st), C.byref(p))
    check_digest(g, f"{tag}/grid_split", w.get("H"), TOL)
    Hper = np.zeros(F.per_size(p, 1))
    assert Hper.size == g[f"{tag}/wrap"].size
    F.call("SE1P_FGG_wrap_fcn", F.dptr(Hper), C.byref(w.s), C.byref(p))
    np.testing.assert_allclose(Hper, g[f"{tag}/wrap"], rtol=0,
                               atol=TOL * np.abs(g[f"{tag}/wrap"]).max())
    field = g[f"{tag}/field"].copy()
    F.call("SE1P_FGG_extend_fcn", C.byref(w.s), F.dptr(field), C.byref(p))
    check_digest(g, f"{tag}/extend", w.get("H"), 0.0)
    phi = np.zeros(10)
    F.call("SE_FGG_int_split", F.dptr(phi), C.byref(w.s), C.byref(p))
    np.testing.assert_allclose(phi, g[f"{tag}/int_split"], rtol=TOL)


def test_reorder_system(F):
    from test_oracle_golden import reorder_agrees
    g = load_golden("fgg_steps.npz")
    import oracle as O
    N = 100
    opt, p = F.fcn_params(32, 8, 1.0, 4.0, 0.95 * np.sqrt(O.PI * 8), N)
    x, q = g["reorder/x_in"].copy(), g["reorder/q_in"].copy()
    w = F.Work(p, where="host")
    st = F.state(x, q)
    F.call("SE_FGG_expand_all", C.byref(w.s), C.byref(st), C.byref(p))
    idx = w.get("idx")
    np.testing.assert_array_equal(idx, g["reorder/idx"])
    F.call("SE_FGG_reorder_system", C.byref(st), C.byref(w.s), C.byref(p))
    assert reorder_agrees(x, q, g["reorder/x_out"], g["reorder/q_out"], idx)
    xo, qo = O.reorder(g["reorder/x_in"], g["reorder/q_in"], idx)   # stable: exact
    np.testing.assert_array_equal(x, xo)
    np.testing.assert_array_equal(q, qo)


@pytest.mark.parametrize("M", [8, 9, 32])
def test_kspace_legacy(F, M):
    import oracle as O
    L, xi, eta = 1.3, 5.0, 0.3
    scalar = -(1 - eta) / (4 * xi * xi)
    Z = np.zeros(M ** 3)
    box = (C.c_double * 3)(L, L, L)
    F.call("scaling", C.c_double(scalar), F.dptr(Z), M, M, M, box)
    Zo = O.scaling(scalar, M, L)
    np.testing.assert_allclose(Z[1:], Zo[1:], rtol=1e-14)
    Z[0] = 0.0
    rng = np.random.Generator(np.random.Philox(2))
    a = rng.standard_normal(2 * M ** 3)
    c = np.zeros_like(a)
    F.call("product_rc", F.dptr(a), F.dptr(Z), F.dptr(c), M, M, M, 1)
    np.testing.assert_array_equal(c.reshape(-1, 2), a.reshape(-1, 2) * Z[:, None])
    F.call("product_rc", F.dptr(a), F.dptr(Z), F.dptr(a), M, M, M, 1)   # in place
    np.testing.assert_array_equal(a, c)
    r = rng.standard_normal(M ** 3)
    cc = np.zeros(2 * M ** 3)
    F.call("copy_r2c", F.dptr(r), F.dptr(cc), M ** 3)
    np.testing.assert_array_equal(cc[0::2], r)
    np.testing.assert_array_equal(cc[1::2], 0.0)
    back = np.zeros(M ** 3)
    F.call("copy_c2r", F.dptr(cc), F.dptr(back), M ** 3)
    np.testing.assert_array_equal(back, r)


@pytest.mark.parametrize("shape", [(8, 8, 8), (6, 10, 9), (32, 32, 32), (64, 64, 65),
                                   (100, 100, 101)])
def test_fftw_shim(F, shape):
    """fftw_plan_dft_3d / r2c / c2r on cuFFT against numpy's FFT.  Arrays of
    1 MiB and more are staged through the pinned chunks of se_hoststage.cu
    (the last two shapes: one partial chunk, and two chunks and a partial
    one), and plans of a shape come back from the plan cache."""
    L = F.lib()
    n0, n1, n2 = shape
    rng = np.random.Generator(np.random.Philox(4))
    a = rng.standard_normal((n0, n1, n2)) + 1j * rng.standard_normal((n0, n1, n2))
    buf = np.ascontiguousarray(a).view(np.float64).reshape(-1).copy()
    L.fftw_plan_dft_3d.restype = C.c_void_p
    L.fftw_plan_dft_r2c_3d.restype = C.c_void_p
    L.fftw_plan_dft_c2r_3d.restype = C.c_void_p
    for sign, ref in ((-1, np.fft.fftn(a)), (1, np.fft.ifftn(a) * a.size)):
        b = buf.copy()
        pl = L.fftw_plan_dft_3d(n0, n1, n2, F.dptr(b), F.dptr(b), sign, 1 << 6)
        L.fftw_execute(C.c_void_p(pl))
        L.fftw_destroy_plan(C.c_void_p(pl))
        got = b.view(np.complex128).reshape(shape)
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    r = rng.standard_normal((n0, n1, n2))
    half = np.zeros(n0 * n1 * (n2 // 2 + 1) * 2)
    rr = r.reshape(-1).copy()
    pl = L.fftw_plan_dft_r2c_3d(n0, n1, n2, F.dptr(rr), F.dptr(half), 1 << 6)
    L.fftw_execute(C.c_void_p(pl))
    L.fftw_destroy_plan(C.c_void_p(pl))
    ref = np.fft.rfftn(r)
    got = half.view(np.complex128).reshape(ref.shape)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    out = np.zeros(n0 * n1 * n2)
    pl = L.fftw_plan_dft_c2r_3d(n0, n1, n2, F.dptr(half), F.dptr(out), 1 << 6)
    L.fftw_execute(C.c_void_p(pl))
    L.fftw_destroy_plan(C.c_void_p(pl))
    np.testing.assert_allclose(out.reshape(shape), r * r.size, rtol=0, atol=1e-11 * r.size)
    # in place on a host array: FFTW's padded layout, n0 x n1 x 2(n2/2 + 1)
    # reals in, the half spectrum out (and back)
    pad = 2 * (n2 // 2 + 1)
    ip = np.zeros((n0, n1, pad))
    ip[:, :, :n2] = r
    ip = ip.reshape(-1)
    pl = L.fftw_plan_dft_r2c_3d(n0, n1, n2, F.dptr(ip), F.dptr(ip), 1 << 6)
    L.fftw_execute(C.c_void_p(pl))
    L.fftw_destroy_plan(C.c_void_p(pl))
    got = ip.view(np.complex128).reshape(ref.shape)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    pl = L.fftw_plan_dft_c2r_3d(n0, n1, n2, F.dptr(ip), F.dptr(ip), 1 << 6)
    L.fftw_execute(C.c_void_p(pl))
    L.fftw_destroy_plan(C.c_void_p(pl))
    np.testing.assert_allclose(ip.reshape(n0, n1, pad)[:, :, :n2], r * r.size, rtol=0,
                               atol=1e-11 * r.size)


def test_out_of_box_position_reported(F):
    """A position outside [0, L] gives a stencil outside the padded grid (the
    reference writes out of bounds there); the kernels skip it and the call
    reports the error."""
    import oracle as O
    import se_fast_gridding_b200 as S
    opt, p = F.fcn_params(16, 8, 1.0, 4.0, 0.95 * np.sqrt(O.PI * 8), 2)
    x = np.array([0.5, 3.0, 0.5, 0.5, 0.5, 0.5])
    q = np.array([1.0, -1.0])
    w = F.Work(p, where="host")
    st = F.state(x, q)
    F.call("SE_FGG_base_gaussian", C.byref(w.s), C.byref(p))
    F.call("SE_FGG_expand_all", C.byref(w.s), C.byref(st), C.byref(p))
    with pytest.raises(S.SEError):
        F.call("SE_FGG_grid_split", C.byref(w.s), C.byref(st), C.byref(p))
    # the in-box particle was still spread, and the library keeps working
    assert np.abs(w.get("H")).sum() > 0
    F.call("SE_FGG_base_gaussian", C.byref(w.s), C.byref(p))


def test_invalid_params_reported(F):
    """P beyond SE_P_MAX is refused with an error, not computed."""
    p = F.pack_params(4, 8, 8, 8, 40, 10.0, 0.125)
    w = F.Work(F.pack_params(4, 8, 8, 8, 8, 10.0, 0.125), where="host")
    import se_fast_gridding_b200 as S
    with pytest.raises(S.SEError):
        F.call("SE_FGG_base_gaussian", C.byref(w.s), C.byref(p))

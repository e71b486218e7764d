"""Pin the CPU oracle against the reference's own outputs (tests/golden/).

The fixtures were produced by tests/golden/make_golden.py from SE_fast_gridding
compiled from source.  These tests need no GPU.
"""
import numpy as np
import pytest

from conftest import check_digest, load_golden

EXACT = 1e-13      # same operation order; gcc may contract a*b+c to FMA differently
SIMD = 1e-12       # the reference's SSE/AVX kernels sum in another order


def _case_params(O, M, P):
    m = 0.95 * np.sqrt(O.PI * P)
    return O.Setup(M=int(M), P=int(P), L=1.0, xi=4.0, m=m, N=10)


@pytest.mark.parametrize("case", [(12, 7), (12, 8), (16, 12), (12, 16), (20, 21)])
def test_fgg_steps_3p(oracle_mod, case):
    O = oracle_mod
    g = load_golden("fgg_steps.npz")
    M, P = case
    tag = f"M{M}P{P}"
    x, q = g["x"], g["q"]
    p = _case_params(O, M, P).params()
    zs = O.base_gaussian(p)
    np.testing.assert_allclose(zs, g[f"{tag}/zs"], rtol=EXACT, atol=0)
    ex = O.expand_all(p, x, 3, False)
    exf = O.expand_all(p, x, 3, True)
    np.testing.assert_array_equal(ex["idx"], g[f"{tag}/exp_idx"])
    np.testing.assert_array_equal(exf["idx"], g[f"{tag}/expf_idx"])
    for k in ("zx", "zy", "zz"):
        np.testing.assert_allclose(ex[k], g[f"{tag}/exp_{k}"], rtol=EXACT, atol=0)
    for k in ("zx", "zy", "zz", "zfx", "zfy", "zfz"):
        np.testing.assert_allclose(exf[k], g[f"{tag}/expf_{k}"], rtol=EXACT, atol=0)
    H = O.grid_split(p, q, zs, ex)
    check_digest(g, f"{tag}/grid_split", H, EXACT)
    check_digest(g, f"{tag}/grid_avx", H, SIMD)
    check_digest(g, f"{tag}/grid_vanilla", O.grid(p, x, q, zs, 3), EXACT)
    check_digest(g, f"{tag}/grid_force", O.grid_split(p, q, zs, exf, force_order=1), EXACT)
    Hper = O.wrap(p, H, 3)
    np.testing.assert_allclose(Hper, g[f"{tag}/wrap"], rtol=0,
                               atol=EXACT * np.abs(g[f"{tag}/wrap"]).max())
    He = O.extend(p, g[f"{tag}/field"], 3)
    check_digest(g, f"{tag}/extend", He, 0.0)
    phi = O.int_split(p, He, zs, ex)
    np.testing.assert_allclose(phi, g[f"{tag}/int_split"], rtol=EXACT)
    np.testing.assert_allclose(phi, g[f"{tag}/int_avx"], rtol=SIMD)
    np.testing.assert_allclose(O.int_vanilla(p, He, x, zs, 3), g[f"{tag}/int_vanilla"], rtol=EXACT)
    f = O.int_split_force(p, q, He, zs, exf)
    np.testing.assert_allclose(f, g[f"{tag}/int_force_split"], rtol=EXACT)
    np.testing.assert_allclose(f, g[f"{tag}/int_force_avx"], rtol=SIMD,
                               atol=SIMD * np.abs(f).max())
    np.testing.assert_allclose(O.int_force_vanilla(p, He, x, q, zs),
                               g[f"{tag}/int_force_vanilla"], rtol=EXACT)
    assert abs(O.calc_energy(g[f"{tag}/int_split"], q) - float(g[f"{tag}/energy"])) <= \
        EXACT * abs(float(g[f"{tag}/energy"]))


@pytest.mark.parametrize("case", [(12, 7), (12, 8), (16, 12), (12, 16), (20, 21)])
def test_fgg_steps_2p(oracle_mod, case):
    O = oracle_mod
    g = load_golden("fgg_steps.npz")
    M, P = case
    tag = f"M{M}P{P}"
    x, q = g["x"], g["q"]
    p3 = _case_params(O, M, P).params()
    p = O.pack_params(10, M, M, M, P, p3.c, 1.0 / M, float(g[f"{tag}/p2_a"]))
    zs = O.base_gaussian(p)
    ex = O.expand_all(p, x, 2, False)
    np.testing.assert_array_equal(ex["idx"], g[f"{tag}/exp2p_idx"])
    for k in ("zx", "zy", "zz"):
        np.testing.assert_allclose(ex[k], g[f"{tag}/exp2p_{k}"], rtol=EXACT, atol=0)
    check_digest(g, f"{tag}/grid2p_vanilla", O.grid(p, x, q, zs, 2), EXACT)
    H = O.grid_split(p, q, zs, ex)
    check_digest(g, f"{tag}/wrap2p", O.wrap(p, H, 2), EXACT)
    He = O.extend(p, g[f"{tag}/field2p"], 2)
    check_digest(g, f"{tag}/extend2p", He, 0.0)
    np.testing.assert_allclose(O.int_vanilla(p, He, x, zs, 2), g[f"{tag}/int2p_vanilla"],
                               rtol=EXACT)


ONE_P = [((12, 12, 12), 7), ((12, 12, 12), 8), ((16, 16, 16), 12), ((12, 12, 12), 16),
         ((20, 20, 20), 21), ((10, 12, 14), 8)]


def one_p_params(O, g, tag):
    d = g[f"{tag}/dims"]
    P = int(tag.split("P")[-1])
    p = O.pack_params(len(g["q"]), int(d[0]), int(d[1]), int(d[2]), P, float(g[f"{tag}/c"]),
                      1.0 / int(d[2]), float(g[f"{tag}/a"]), float(g[f"{tag}/b"]))
    return p


@pytest.mark.parametrize("case", ONE_P)
def test_fgg_steps_1p(oracle_mod, case):
    """SE1P (x and y free, z periodic) against a -DONE_PERIODIC build of the
    reference: the expansion (fgg_expansion_1p, SE_fgg.c:823-916), spread,
    SE1P_FGG_wrap_fcn (:387-411, whose column-major map of the padded x, y
    overlaps itself), SE1P_FGG_extend_fcn (:478-502), interpolation."""
    O = oracle_mod
    g = load_golden("fgg_1p.npz")
    dims, P = case
    tag = "D{}x{}x{}P{}".format(*dims, P)
    x, q = g["x"], g["q"]
    p = one_p_params(O, g, tag)
    assert p.d == float(g[f"{tag}/d"])
    zs = O.base_gaussian(p)
    ex = O.expand_all(p, x, 1, False)
    np.testing.assert_array_equal(ex["idx"], g[f"{tag}/exp_idx"])
    for k in ("zx", "zy", "zz"):
        np.testing.assert_allclose(ex[k], g[f"{tag}/exp_{k}"], rtol=EXACT, atol=0)
    check_digest(g, f"{tag}/grid_vanilla", O.grid(p, x, q, zs, 1), EXACT)
    H = O.grid_split(p, q, zs, ex)
    check_digest(g, f"{tag}/grid_split", H, EXACT)
    Hper = O.wrap(p, H, 1)
    assert Hper.size == g[f"{tag}/wrap"].size
    np.testing.assert_allclose(Hper, g[f"{tag}/wrap"], rtol=0,
                               atol=EXACT * np.abs(g[f"{tag}/wrap"]).max())
    He = O.extend(p, g[f"{tag}/field"], 1)
    check_digest(g, f"{tag}/extend", He, 0.0)
    np.testing.assert_allclose(O.int_vanilla(p, He, x, zs, 1), g[f"{tag}/int_vanilla"],
                               rtol=EXACT)
    np.testing.assert_allclose(O.int_split(p, He, zs, ex), g[f"{tag}/int_split"], rtol=EXACT)


@pytest.mark.parametrize("N", [10, 100])
@pytest.mark.parametrize("P", [8, 12, 16, 21])
def test_pipeline_matches_reference_spectral_ewald(oracle_mod, N, P):
    """The oracle's full solve equals the reference's spectral_ewald()
    (test_accuracy.c settings: atoms.txt, L = 3.1814, xi = 8)."""
    O = oracle_mod
    g = load_golden("test_accuracy.npz")
    x, q = g[f"N{N}/x"], g[f"N{N}/q"]
    M, m = O.init_params(P, 3.1814, 8.0, q)
    assert M == int(g[f"N{N}/P{P}/M"]) and m == float(g[f"N{N}/P{P}/m"])
    phi = O.spectral_ewald(x, q, M, P, m, 3.1814, 8.0, "potential")
    assert O.rel_rms(phi, g[f"N{N}/P{P}/phi"]) < 1e-12
    f = O.spectral_ewald(x, q, M, P, m, 3.1814, 8.0, "force")
    assert O.rel_rms(f, g[f"N{N}/P{P}/force"]) < 1e-12


def test_direct_sums_match_reference(oracle_mod):
    O = oracle_mod
    g = load_golden("test_accuracy.npz")
    x, q = g["N10/x"], g["N10/q"]
    layers = int(g["N10/layers"])
    np.testing.assert_allclose(O.direct_fd(x, q, 3.1814, 8.0, layers), g["N10/direct_phi"],
                               rtol=1e-13)
    np.testing.assert_allclose(O.direct_force_fd(x, q, 3.1814, 8.0, layers),
                               g["N10/direct_force"], rtol=1e-12, atol=1e-14)
    # the structure-factor form of the same sums (the cube |j| <= layers)
    phi, f = O.sf_kspace(x, q, 3.1814, 8.0, np.arange(10), jmax=layers, kcut2=-1.0)
    np.testing.assert_allclose(phi, g["N10/direct_phi"], rtol=1e-11)
    np.testing.assert_allclose(f, g["N10/direct_force"], rtol=1e-10, atol=1e-13)
    # and its torch restatement (the checker of the GPU tests at millions of
    # particles), here on the CPU
    phi_t, f_t = O.sf_kspace_torch(x, q, 3.1814, 8.0, np.arange(10), jmax=layers, kcut2=-1.0)
    np.testing.assert_allclose(phi_t, g["N10/direct_phi"], rtol=1e-11)
    np.testing.assert_allclose(f_t, g["N10/direct_force"], rtol=1e-10, atol=1e-13)


@pytest.mark.parametrize("clusters", [0, 4])
def test_torch_structure_factor_sum_equals_oracle(oracle_mod, clusters):
    """sf_kspace_torch = sf_kspace (the C oracle's structure-factor sum) with
    and without the sphere cut, over several particle chunks."""
    O = oracle_mod
    x, q = O.synthetic_system(300, 1.3, seed=3 + clusters, charges="uniform",
                              clusters=clusters, sigma=0.05)
    t = np.arange(0, 300, 7)
    jmax, kc2 = O.kspace_converged_jmax(1.3, 6.0)
    for cut in (kc2, -1.0):
        p0, f0 = O.sf_kspace(x, q, 1.3, 6.0, t, jmax, cut)
        p1, f1 = O.sf_kspace_torch(x, q, 1.3, 6.0, t, jmax, cut, chunk=128)
        assert O.rel_rms(p1, p0) < 1e-13
        assert O.rel_rms(f1, f0) < 1e-13


def test_reference_accuracy_figures(oracle_mod):
    """The abs-RMS errors test_accuracy prints (SE vs direct), reproduced."""
    O = oracle_mod
    g = load_golden("test_accuracy.npz")
    e_pot = O.abs_rms(g["N10/direct_phi"], g["N10/P16/phi"])
    e_force = O.abs_rms(g["N10/P16/force"], g["N10/direct_force"])
    assert 2.6e-10 < e_pot < 2.7e-10
    assert 4.9e-9 < e_force < 5.0e-9


def test_c1_oracle(oracle_mod):
    O = oracle_mod
    g = load_golden("c1.npz")
    x, q = g["x"], g["q"]
    phi = O.spectral_ewald(x, q, 32, 21, O.c1_params(21), 1.0, 8.0, "potential")
    assert O.rel_rms(phi, g["phi_ref"]) < 1e-12
    # FP64 SE at P = 21 agrees with the converged direct sum
    assert O.rel_rms(g["phi_ref"], g["phi_direct"]) < 1e-11
    assert O.rel_rms(g["force_ref"], g["force_direct"]) < 1e-10


def test_counting_sort_is_stable(oracle_mod):
    O = oracle_mod
    rng = np.random.Generator(np.random.Philox(3))
    keys = rng.integers(0, 50, size=5000).astype(np.int32)
    perm, offs = O.counting_sort(keys, 50)
    np.testing.assert_array_equal(perm, np.argsort(keys, kind="stable"))
    np.testing.assert_array_equal(offs, np.concatenate([[0], np.cumsum(np.bincount(keys, minlength=50))]))


def reorder_agrees(x, q, xr, qr, idx):
    """x, q equal the reference's reordered xr, qr up to the order of
    particles that share a grid index (qsort leaves that order unspecified)."""
    N = len(q)
    keys = np.sort(idx)
    for k in np.unique(keys):
        sl = np.nonzero(keys == k)[0]
        a = sorted(zip(q[sl], *(x[d * N + sl] for d in range(3))))
        b = sorted(zip(qr[sl], *(xr[d * N + sl] for d in range(3))))
        if a != b:
            return False
    return True


def test_reorder_matches_reference(oracle_mod):
    """SE_FGG_reorder_system (SE_fgg.c:5894-5932) sorts by grid index."""
    O = oracle_mod
    g = load_golden("fgg_steps.npz")
    idx = g["reorder/idx"]
    x, q = O.reorder(g["reorder/x_in"], g["reorder/q_in"], idx)
    assert reorder_agrees(x, q, g["reorder/x_out"], g["reorder/q_out"], idx)
    # the oracle keeps ties in input order (stable)
    order = np.argsort(idx, kind="stable")
    np.testing.assert_array_equal(q, g["reorder/q_in"][order])


REAL_CASES = ["atoms_l1_rc1.5", "atoms_l0_rc1.2", "atoms_l1_nocut", "atoms_l2_rc2",
              "syn_l1_rc0.35", "syn_l1_rc0.5"]


@pytest.mark.parametrize("tag", REAL_CASES)
def test_oracle_real_space_and_self_match_reference(oracle_mod, tag):
    """SE3P_direct_real_rc / SE3P_direct_real / SE3P_direct_self
    (SE_direct.c:464-562) against the reference's own outputs."""
    O = oracle_mod
    g = load_golden("realspace.npz")
    src = "atoms" if tag.startswith("atoms") else "syn"
    x, q = g[f"{src}/x"], g[f"{src}/q"]
    L, xi, layers, rc = g[f"{tag}/params"]
    phi = O.direct_real(x, q, L, xi, int(layers), rc)
    assert O.rel_rms(phi, g[f"{tag}/phi"]) < EXACT
    np.testing.assert_allclose(O.direct_self(q, xi), g[f"{tag}/self"], rtol=1e-15, atol=0)


def test_oracle_real_space_force_is_the_gradient(oracle_mod):
    """The real-space force (no reference counterpart) is -q_m times the
    gradient of the real-space potential at x_m: central differences."""
    O = oracle_mod
    x, q = O.synthetic_system(40, 1.0, seed=4, charges="uniform")
    L, xi, layers, rc = 1.0, 6.0, 1, 0.0
    f = O.direct_real_force(x, q, L, xi, layers, rc)
    N, h = len(q), 1e-6
    for m in (0, 7, 31):
        for a in range(3):
            xp, xm = x.copy(), x.copy()
            xp[m + a * N] += h
            xm[m + a * N] -= h
            # energy of particle m only: phi_m(x) q_m (the pair terms' other
            # half acts on the partner)
            dphi = (O.direct_real(xp, q, L, xi, layers, rc)[m] -
                    O.direct_real(xm, q, L, xi, layers, rc)[m]) / (2 * h)
            assert abs(f[m + a * N] - (-q[m] * dphi)) < 1e-6 * max(1.0, abs(f[m + a * N]))

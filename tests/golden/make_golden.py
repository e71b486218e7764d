"""Generate the golden vectors in tests/golden/ from the reference itself.

Run here, where the SE_fast_gridding sources are available: ``make -C oracle
ref`` compiles them (unchanged, FFTW replaced by oracle/fftw_cpu.c) into
oracle/_ref/, and this script calls those libraries through ctypes:

    python tests/golden/make_golden.py [--ref /path/to/SE_fast_gridding]

Every fixture holds reference outputs only (inputs are regenerated from seeds or
stored beside them).  Large grids are stored as checksums plus a seeded sample
of entries, so the fixtures stay small.  The files are committed; the GPU box
never runs this script.
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def grid_digest(a: np.ndarray, nsample=256, seed=7):
    """Checksums and a seeded sample of a large array."""
    a = np.asarray(a, dtype=np.float64).ravel()
    rng = np.random.Generator(np.random.Philox(seed))
    idx = np.sort(rng.choice(a.size, size=min(nsample, a.size), replace=False)).astype(np.int64)
    w = rng.uniform(-1, 1, size=a.size)
    return {"size": np.int64(a.size), "sum": a.sum(), "l1": np.abs(a).sum(),
            "l2": float(np.sqrt((a * a).sum())), "wsum": float((w * a).sum()),
            "sidx": idx, "sval": a[idx].copy()}


def put(d, prefix, a, full=False):
    if full:
        d[prefix] = np.asarray(a).copy()
    else:
        for k, v in grid_digest(a).items():
            d[f"{prefix}__{k}"] = v


class Ref:
    """ctypes view of one reference build."""

    def __init__(self, kind):
        self.lib = O.ref_lib(kind)
        if self.lib is None:
            raise SystemExit(f"oracle/_ref/libse_ref_{kind}.so missing: run make -C oracle ref")

    def work(self, p, H, zs, ex, force=False):
        w = O.FGGWork()
        w.H = O.dptr(H)
        w.zs = O.dptr(zs)
        if ex is not None:
            w.zx, w.zy, w.zz = O.dptr(ex["zx"]), O.dptr(ex["zy"]), O.dptr(ex["zz"])
            w.idx = O.iptr(ex["idx"])
            if force:
                w.zfx, w.zfy, w.zfz = O.dptr(ex["zfx"]), O.dptr(ex["zfy"]), O.dptr(ex["zfz"])
        return w


def new_exp(N, P, force):
    ex = {k: O.aligned_zeros(N * P) for k in ("zx", "zy", "zz")}
    if force:
        ex.update({k: O.aligned_zeros(N * P) for k in ("zfx", "zfy", "zfz")})
    ex["idx"] = O.aligned_zeros(N, dtype=np.int32)
    return ex


def atoms(ref_dir):
    a = np.loadtxt(os.path.join(ref_dir, "atoms.txt"))
    return a


def fgg_steps(ref: Ref, ref2p: Ref, x, q, M, P, L, xi, m, tag, out):
    """Every step of the FGG path, 3P (and the 2P library calls), small grid."""
    N = len(q)
    lib = ref.lib
    s = O.Setup(M=M, P=P, L=L, xi=xi, m=m, N=N)
    opt = s.opt()
    p = O.FGGParams()
    lib.parse_params(C.byref(opt), C.c_double(xi))
    lib.SE_FGG_FCN_params(C.byref(p), C.byref(opt), N)
    n_pad = int(np.prod(p.npdims))
    zs = O.aligned_zeros(P ** 3)
    H = O.aligned_zeros(n_pad)
    w = ref.work(p, H, zs, None)
    lib.SE_FGG_base_gaussian(C.byref(w), C.byref(p))
    out[f"{tag}/zs"] = zs.copy()
    st = O.State()
    st.x, st.q = O.dptr(x), O.dptr(q)
    # expansion vectors (POTENTIAL and FORCE)
    ex = new_exp(N, P, False)
    w = ref.work(p, H, zs, ex)
    lib.SE_FGG_expand_all(C.byref(w), C.byref(st), C.byref(p))
    for k in ("zx", "zy", "zz", "idx"):
        out[f"{tag}/exp_{k}"] = ex[k].copy()
    exf = new_exp(N, P, True)
    w = ref.work(p, H, zs, exf, force=True)
    lib.SE_FGG_expand_all_SSE_force(C.byref(w), C.byref(st), C.byref(p))
    for k in ("zx", "zy", "zz", "zfx", "zfy", "zfz", "idx"):
        out[f"{tag}/expf_{k}"] = exf[k].copy()
    # spread: split (scalar), AVX dispatch, vanilla, force split
    for name, fn, e in (("grid_split", "SE_FGG_grid_split", ex),
                        ("grid_avx", "SE_FGG_grid_split_AVX_dispatch", ex),
                        ("grid_vanilla", "SE_FGG_grid", ex),
                        ("grid_force", "SE_FGG_grid_split_force", exf)):
        Hn = O.aligned_zeros(n_pad)
        w = ref.work(p, Hn, zs, e, force=(e is exf))
        getattr(lib, fn)(C.byref(w), C.byref(st), C.byref(p))
        put(out, f"{tag}/{name}", Hn, full=n_pad <= 8000)
        if name == "grid_split":
            H = Hn.copy()
    # wrap (H_per is column-major M^3)
    Hper = O.aligned_zeros(M ** 3)
    w = ref.work(p, H, zs, ex)
    lib.SE_FGG_wrap_fcn(O.dptr(Hper), C.byref(w), C.byref(p))
    out[f"{tag}/wrap"] = Hper.copy()
    # extend a seeded periodic field
    rng = np.random.Generator(np.random.Philox(11))
    F = O.aligned_copy(rng.standard_normal(M ** 3))
    out[f"{tag}/field"] = F.copy()
    He = O.aligned_zeros(n_pad)
    w = ref.work(p, He, zs, ex)
    lib.SE_FGG_extend_fcn(C.byref(w), O.dptr(F), C.byref(p))
    put(out, f"{tag}/extend", He, full=n_pad <= 8000)
    # interpolate that field: split, AVX dispatch, vanilla, force
    for name, fn in (("int_split", "SE_FGG_int_split"), ("int_avx", "SE_FGG_int_split_AVX_dispatch")):
        phi = O.aligned_zeros(N)
        w = ref.work(p, He, zs, ex)
        getattr(lib, fn)(O.dptr(phi), C.byref(w), C.byref(p))
        out[f"{tag}/{name}"] = phi
    phi = O.aligned_zeros(N)
    w = ref.work(p, He, zs, ex)
    lib.SE_FGG_int(O.dptr(phi), C.byref(w), C.byref(st), C.byref(p))
    out[f"{tag}/int_vanilla"] = phi
    for name, fn in (("int_force_split", "SE_FGG_int_split_force"),
                     ("int_force_avx", "SE_FGG_int_split_AVX_dispatch_force")):
        f = O.aligned_zeros(3 * N)
        w = ref.work(p, He, zs, exf, force=True)
        getattr(lib, fn)(O.dptr(f), C.byref(st), C.byref(w), C.byref(p))
        out[f"{tag}/{name}"] = f
    f = O.aligned_zeros(3 * N)
    w = ref.work(p, He, zs, None)
    lib.SE_FGG_int_force(O.dptr(f), C.byref(w), C.byref(st), C.byref(p))
    out[f"{tag}/int_force_vanilla"] = f
    # energy
    lib.calc_energy.restype = C.c_double
    lib.calc_energy.argtypes = [O.State, C.c_int]
    st2 = O.State()
    phi = out[f"{tag}/int_split"].copy()
    st2.x, st2.q, st2.phi = O.dptr(x), O.dptr(q), O.dptr(phi)
    out[f"{tag}/energy"] = np.float64(lib.calc_energy(st2, N))

    # ---- 2P library calls (x,y periodic, z free with offset a) ----
    l2 = ref2p.lib
    h = L / M
    ph = P // 2 if P % 2 == 0 else (P - 1) // 2
    a = -(ph + 1) * h
    p2 = O.FGGParams()
    l2.SE2P_FGG_pack_params(C.byref(p2), N, M, M, M, P, C.c_double(p.c), C.c_double(h),
                            C.c_double(a))
    out[f"{tag}/p2_a"] = np.float64(a)
    n_pad2 = int(np.prod(p2.npdims))
    zs2 = O.aligned_zeros(P ** 3)
    w = ref2p.work(p2, O.aligned_zeros(n_pad2), zs2, None)
    l2.SE_FGG_base_gaussian(C.byref(w), C.byref(p2))
    ex2 = new_exp(N, P, False)
    w = ref2p.work(p2, O.aligned_zeros(n_pad2), zs2, ex2)
    l2.SE_FGG_expand_all(C.byref(w), C.byref(st), C.byref(p2))
    for k in ("zx", "zy", "zz", "idx"):
        out[f"{tag}/exp2p_{k}"] = ex2[k].copy()
    H2 = O.aligned_zeros(n_pad2)
    w = ref2p.work(p2, H2, zs2, ex2)
    l2.SE_FGG_grid(C.byref(w), C.byref(st), C.byref(p2))
    put(out, f"{tag}/grid2p_vanilla", H2, full=n_pad2 <= 8000)
    Hs = O.aligned_zeros(n_pad2)
    w = ref2p.work(p2, Hs, zs2, ex2)
    l2.SE_FGG_grid_split(C.byref(w), C.byref(st), C.byref(p2))
    Hper2 = O.aligned_zeros(M * M * p2.npdims[2])
    l2.SE2P_FGG_wrap_fcn(O.dptr(Hper2), C.byref(w), C.byref(p2))
    put(out, f"{tag}/wrap2p", Hper2, full=Hper2.size <= 8000)
    F2 = O.aligned_copy(rng.standard_normal(M * M * p2.npdims[2]))
    out[f"{tag}/field2p"] = F2.copy()
    He2 = O.aligned_zeros(n_pad2)
    w = ref2p.work(p2, He2, zs2, ex2)
    l2.SE2P_FGG_extend_fcn(C.byref(w), O.dptr(F2), C.byref(p2))
    put(out, f"{tag}/extend2p", He2, full=n_pad2 <= 8000)
    phi2 = O.aligned_zeros(N)
    w = ref2p.work(p2, He2, zs2, ex2)
    l2.SE_FGG_int(O.dptr(phi2), C.byref(w), C.byref(st), C.byref(p2))
    out[f"{tag}/int2p_vanilla"] = phi2


def one_periodic_steps(ref1p: Ref, x, q, dims, P, c, tag, out):
    """The 1P library calls (x and y free with offsets a and b, z periodic):
    SE1P_FGG_pack_params (SE_fgg.c:113-132), the expansion of a -DONE_PERIODIC
    build (fgg_expansion_1p, :823-916) through SE_FGG_expand_all, the spread
    (SE_FGG_grid and SE_FGG_grid_split), SE1P_FGG_wrap_fcn (:387-411),
    SE1P_FGG_extend_fcn (:478-502) of a seeded field, and the interpolation
    (SE_FGG_int, SE_FGG_int_split).  The offsets keep every stencil inside
    the padded grid for positions in [0, 1)."""
    N = len(q)
    lib = ref1p.lib
    M0, M1, M2 = dims
    h = 1.0 / M2
    ph = P // 2 if P % 2 == 0 else (P - 1) // 2
    a, b = -ph * h, -(ph + 0.25) * h
    p = O.FGGParams()
    lib.SE1P_FGG_pack_params(C.byref(p), N, M0, M1, M2, P, C.c_double(c), C.c_double(h),
                             C.c_double(a), C.c_double(b))
    out[f"{tag}/a"], out[f"{tag}/b"], out[f"{tag}/c"] = np.float64(a), np.float64(b), np.float64(c)
    out[f"{tag}/dims"] = np.array(dims, dtype=np.int32)
    out[f"{tag}/d"] = np.float64(p.d)
    n_pad = int(np.prod(p.npdims))
    zs = O.aligned_zeros(P ** 3)
    w = ref1p.work(p, O.aligned_zeros(n_pad), zs, None)
    lib.SE_FGG_base_gaussian(C.byref(w), C.byref(p))
    st = O.State()
    st.x, st.q = O.dptr(x), O.dptr(q)
    ex = new_exp(N, P, False)
    w = ref1p.work(p, O.aligned_zeros(n_pad), zs, ex)
    lib.SE_FGG_expand_all(C.byref(w), C.byref(st), C.byref(p))
    for k in ("zx", "zy", "zz", "idx"):
        out[f"{tag}/exp_{k}"] = ex[k].copy()
    Hv = O.aligned_zeros(n_pad)
    w = ref1p.work(p, Hv, zs, ex)
    lib.SE_FGG_grid(C.byref(w), C.byref(st), C.byref(p))
    put(out, f"{tag}/grid_vanilla", Hv, full=n_pad <= 8000)
    H = O.aligned_zeros(n_pad)
    w = ref1p.work(p, H, zs, ex)
    lib.SE_FGG_grid_split(C.byref(w), C.byref(st), C.byref(p))
    put(out, f"{tag}/grid_split", H, full=n_pad <= 8000)
    nper = O.per_size(p, 1)
    Hper = O.aligned_zeros(nper)
    lib.SE1P_FGG_wrap_fcn(O.dptr(Hper), C.byref(w), C.byref(p))
    out[f"{tag}/wrap"] = Hper.copy()
    rng = np.random.Generator(np.random.Philox(13))
    F = O.aligned_copy(rng.standard_normal(nper))
    out[f"{tag}/field"] = F.copy()
    He = O.aligned_zeros(n_pad)
    w = ref1p.work(p, He, zs, ex)
    lib.SE1P_FGG_extend_fcn(C.byref(w), O.dptr(F), C.byref(p))
    put(out, f"{tag}/extend", He, full=n_pad <= 8000)
    phi = O.aligned_zeros(N)
    w = ref1p.work(p, He, zs, ex)
    lib.SE_FGG_int(O.dptr(phi), C.byref(w), C.byref(st), C.byref(p))
    out[f"{tag}/int_vanilla"] = phi
    phi = O.aligned_zeros(N)
    lib.SE_FGG_int_split(O.dptr(phi), C.byref(w), C.byref(p))
    out[f"{tag}/int_split"] = phi


ONE_P_CASES = [((12, 12, 12), 7), ((12, 12, 12), 8), ((16, 16, 16), 12), ((12, 12, 12), 16),
               ((20, 20, 20), 21), ((10, 12, 14), 8)]


def make_one_periodic(ref_dir):
    """tests/golden/fgg_1p.npz: the 1P library calls on atoms.txt's first 10
    atoms rescaled into the unit box."""
    ref1p = Ref("1p")
    A = atoms(ref_dir)
    N, Lb = 10, 3.1814
    xa = O.aligned_copy(A[:N, :3].T.reshape(-1) / Lb)
    qa = O.aligned_copy(A[:N, 3])
    out = {"x": xa, "q": qa, "cases": np.array([list(d) + [P] for d, P in ONE_P_CASES],
                                                 dtype=np.int32)}
    for dims, P in ONE_P_CASES:
        m = 0.95 * np.sqrt(O.PI * P)
        s = O.Setup(M=dims[2], P=P, L=1.0, xi=4.0, m=m, N=N)
        c = s.params().c
        one_periodic_steps(ref1p, xa, qa, dims, P, c, "D{}x{}x{}P{}".format(*dims, P), out)
    np.savez_compressed(os.path.join(OUT, "fgg_1p.npz"), **out)
    print("fgg_1p.npz", len(out), "arrays")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SE_REF_DIR"),
                    help="SE_fast_gridding checkout (default: $SE_REF_DIR)")
    ap.add_argument("--skip-c2", action="store_true")
    ap.add_argument("--realspace-only", action="store_true")
    ap.add_argument("--one-periodic-only", action="store_true",
                    help="write tests/golden/fgg_1p.npz only")
    args = ap.parse_args()
    if not args.ref or not os.path.isfile(os.path.join(args.ref, "SE_fgg.c")):
        ap.error("the reference sources are needed: pass --ref <SE_fast_gridding checkout> "
                 "or set SE_REF_DIR")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={args.ref}", "all", "ref"],
                   check=True)
    if args.realspace_only:
        return realspace(Ref("pot"), atoms(args.ref))
    if args.one_periodic_only:
        return make_one_periodic(args.ref)
    ref = Ref("pot")
    reff = Ref("force")
    ref2p = Ref("2p")
    A = atoms(args.ref)

    # ---------------- 1. every FGG step on small grids (atoms.txt, rescaled)
    out = {}
    Lb = 3.1814
    N = 10
    xa = O.aligned_copy(A[:N, :3].T.reshape(-1) / Lb)   # unit box
    qa = O.aligned_copy(A[:N, 3])
    cases = [(12, 7), (12, 8), (16, 12), (12, 16), (20, 21)]
    out["cases"] = np.array(cases, dtype=np.int32)
    out["x"] = xa
    out["q"] = qa
    for M, P in cases:
        m = 0.95 * np.sqrt(O.PI * P)
        fgg_steps(ref, ref2p, xa, qa, M, P, 1.0, 4.0, m, f"M{M}P{P}", out)
    # reorder (SE_fgg.c:5894-5932) on 100 atoms of atoms.txt, M=32, P=8
    N = 100
    xr = O.aligned_copy(A[:N, :3].T.reshape(-1) / Lb)
    qr = O.aligned_copy(A[:N, 3])
    s = O.Setup(M=32, P=8, L=1.0, xi=4.0, m=0.95 * np.sqrt(O.PI * 8), N=N)
    opt = s.opt()
    p = O.FGGParams()
    ref.lib.SE_FGG_FCN_params(C.byref(p), C.byref(opt), N)
    ex = new_exp(N, 8, False)
    st = O.State()
    st.x, st.q = O.dptr(xr), O.dptr(qr)
    w = ref.work(p, O.aligned_zeros(int(np.prod(p.npdims))), O.aligned_zeros(512), ex)
    ref.lib.SE_FGG_expand_all(C.byref(w), C.byref(st), C.byref(p))
    out["reorder/x_in"] = np.array(xr)
    out["reorder/q_in"] = np.array(qr)
    out["reorder/idx"] = ex["idx"].copy()
    ref.lib.SE_FGG_reorder_system(C.byref(st), C.byref(w), C.byref(p))
    out["reorder/x_out"] = np.array(xr)
    out["reorder/q_out"] = np.array(qr)
    np.savez_compressed(os.path.join(OUT, "fgg_steps.npz"), **out)
    print("fgg_steps.npz", len(out), "arrays")

    # ---------------- 2. the reference's own test: atoms.txt, L=3.1814, xi=8
    out = {}
    L, xi = 3.1814, 8.0
    for N in (10, 100):
        xN = O.aligned_copy(A[:N, :3].T.reshape(-1))
        qN = O.aligned_copy(A[:N, 3])
        out[f"N{N}/x"] = xN
        out[f"N{N}/q"] = qN
        for P in (8, 12, 16, 21):
            M, m = O.init_params(P, L, xi, qN)
            out[f"N{N}/P{P}/M"] = np.int32(M)
            out[f"N{N}/P{P}/m"] = np.float64(m)
            out[f"N{N}/P{P}/phi"] = O.ref_spectral_ewald(ref.lib, xN, qN, M, P, m, L, xi, N)
            out[f"N{N}/P{P}/force"] = O.ref_spectral_ewald(reff.lib, xN, qN, M, P, m, L, xi, 3 * N)
        if N == 10:
            M = out["N10/P16/M"]
            layers = int((M - 1) // 2)
            box = np.array([L, L, L])
            phi_d = O.aligned_zeros(N)
            ref.lib.SE3P_direct_fd(O.dptr(phi_d), O.dptr(xN), O.dptr(qN), N,
                                   _ewald_opts(L, xi, layers))
            f_d = O.aligned_zeros(3 * N)
            reff.lib.SE3P_direct_force_fd(O.dptr(f_d), O.dptr(xN), O.dptr(qN), N,
                                          _ewald_opts(L, xi, layers))
            out["N10/direct_phi"] = phi_d
            out["N10/direct_force"] = f_d
            out["N10/layers"] = np.int32(layers)
            del box
    np.savez_compressed(os.path.join(OUT, "test_accuracy.npz"), **out)
    print("test_accuracy.npz", len(out), "arrays")

    # ---------------- 3. C1: plain SE3P POTENTIAL FP64, N=100, M=32, P=21, xi=8
    out = {}
    x, q = O.synthetic_system(100, 1.0, seed=0, charges="pm1")
    P, M, xi = 21, 32, 8.0
    m = O.c1_params(P)
    out["x"], out["q"] = x, q
    out["phi_ref"] = O.ref_spectral_ewald(ref.lib, x, q, M, P, m, 1.0, xi, 100)
    out["force_ref"] = O.ref_spectral_ewald(reff.lib, x, q, M, P, m, 1.0, xi, 300)
    targets = np.arange(100, dtype=np.int32)
    phi_d, f_d = O.sf_kspace(x, q, 1.0, xi, targets, jmax=20, kcut2=(2 * O.PI * 20) ** 2)
    out["phi_direct"], out["force_direct"] = phi_d, f_d
    np.savez_compressed(os.path.join(OUT, "c1.npz"), **out)
    print("c1.npz: rel-RMS SE vs direct", O.rel_rms(out["phi_ref"], phi_d))

    realspace(ref, A)
    make_one_periodic(args.ref)
    if args.skip_c2:
        return
    # ---------------- 4. C2: FORCE N=1e5, M=128, P=16, xi=20 (1000-particle subset)
    out = {}
    N, P, M, xi = 100_000, 16, 128, 20.0
    x, q = O.synthetic_system(N, 1.0, seed=1, charges="uniform")
    m = O.c1_params(P)
    rng = np.random.Generator(np.random.Philox(5))
    targets = np.sort(rng.choice(N, size=1000, replace=False)).astype(np.int32)
    out["targets"] = targets
    out["x_check"] = x[targets].copy()    # guards the seeded inputs
    f = O.ref_spectral_ewald(reff.lib, x, q, M, P, m, 1.0, xi, 3 * N)
    phi = O.ref_spectral_ewald(ref.lib, x, q, M, P, m, 1.0, xi, N)
    out["force_ref"] = np.concatenate([f[targets + d * N] for d in range(3)])
    out["phi_ref"] = phi[targets]
    put(out, "force_ref_all", f)
    put(out, "phi_ref_all", phi)
    phi_d, f_d = O.sf_kspace(x, q, 1.0, xi, targets)
    out["phi_direct"], out["force_direct"] = phi_d, f_d
    np.savez_compressed(os.path.join(OUT, "c2.npz"), **out)
    print("c2.npz: rel-RMS SE force vs direct", O.rel_rms(out["force_ref"], f_d),
          "phi", O.rel_rms(out["phi_ref"], phi_d))


def realspace(ref, A):
    """5. The real-space and self terms: SE3P_direct_real_rc
    (SE_direct.c:464-506), SE3P_direct_real (:508-549), SE3P_direct_self
    (:551-562) on atoms.txt (N=100, L=3.1814) and a seeded N=400 unit-box
    system."""
    out = {}
    Lb = 3.1814
    xa = O.aligned_copy(A[:100, :3].T.reshape(-1))
    qa = O.aligned_copy(A[:100, 3])
    xs, qs = O.synthetic_system(400, 1.0, seed=21, charges="uniform")
    xs, qs = O.aligned_copy(xs), O.aligned_copy(qs)
    cases = [("atoms_l1_rc1.5", xa, qa, Lb, 2.0, 1, 1.5), ("atoms_l0_rc1.2", xa, qa, Lb, 2.0, 0, 1.2),
             ("atoms_l1_nocut", xa, qa, Lb, 3.0, 1, 0.0), ("atoms_l2_rc2", xa, qa, Lb, 1.5, 2, 2.0),
             ("syn_l1_rc0.35", xs, qs, 1.0, 9.0, 1, 0.35), ("syn_l1_rc0.5", xs, qs, 1.0, 7.0, 1, 0.5)]
    out["atoms/x"], out["atoms/q"], out["syn/x"], out["syn/q"] = xa, qa, xs, qs
    for tag, x, q, L, xi, layers, rc in cases:
        N = len(q)
        e = _ewald_opts(L, xi, layers)
        e.rc = rc
        phi = O.aligned_zeros(N)
        if rc > 0:
            ref.lib.SE3P_direct_real_rc(O.dptr(phi), O.dptr(x), O.dptr(q), N, e)
        else:
            ref.lib.SE3P_direct_real(O.dptr(phi), O.dptr(x), O.dptr(q), N, e)
        out[f"{tag}/params"] = np.array([L, xi, layers, rc])
        out[f"{tag}/phi"] = np.array(phi)
        self_ = O.aligned_zeros(N)
        ref.lib.SE3P_direct_self(O.dptr(self_), O.dptr(q), N, e)
        out[f"{tag}/self"] = np.array(self_)
    np.savez_compressed(os.path.join(OUT, "realspace.npz"), **out)
    print("realspace.npz", len(out), "arrays")


class _EwaldOpts(C.Structure):
    """SE_direct.h:11-17 ewald_opts."""
    _fields_ = [("box", C.c_double * 3), ("xi", C.c_double), ("layers", C.c_int),
                ("rc", C.c_double)]


def _ewald_opts(L, xi, layers):
    e = _EwaldOpts()
    e.box[:] = (L, L, L)
    e.xi = xi
    e.layers = layers
    e.rc = 0.0
    return e


if __name__ == "__main__":
    main()

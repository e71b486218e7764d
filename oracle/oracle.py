"""CPU oracle of the SE fast-Gaussian-gridding path (test infrastructure only).

This module is the checker for libse_gpu.so.  It is imported by tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` and by
nothing in the product.  It wraps ``oracle/libse_oracle.so`` (our C restatement
of the reference algorithm, ``se_oracle.c``) and, where it was built, the
reference compiled from its own sources (``oracle/_ref/libse_ref_*.so``).

The full solve (:func:`spectral_ewald`) follows ``spectral_ewald.c:20-182`` of
SE_fast_gridding: pack -> base Gaussian -> expand -> grid -> wrap -> forward
FFT -> Green's function scaling -> backward FFT -> extend -> interpolate, with
numpy's FFT standing in for FFTW (the reference calls a C2C FFTW plan on the
column-major wrapped grid read as row-major, ``spectral_ewald.c:119-134``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
PI = 3.14159265358979323846

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class FGGParams(C.Structure):
    """Layout of SE_FGG_params (SE_fgg.h:121-134)."""
    _fields_ = [("N", C.c_int), ("P", C.c_int), ("P_half", C.c_int),
                ("dims", C.c_int * 3), ("npdims", C.c_int * 3),
                ("c", C.c_double), ("d", C.c_double), ("h", C.c_double),
                ("a", C.c_double), ("b", C.c_double)]


class FGGWork(C.Structure):
    """Layout of SE_FGG_work (SE_fgg.h:100-118)."""
    _fields_ = [("H", _dp), ("zs", _dp), ("zx", _dp), ("zy", _dp), ("zz", _dp),
                ("idx", _ip), ("zfx", _dp), ("zfy", _dp), ("zfz", _dp),
                ("free_zs", C.c_int), ("free_fgg_expa", C.c_int)]


class State(C.Structure):
    """Layout of SE_state (SE_fgg.h:142-148)."""
    _fields_ = [("x", _dp), ("q", _dp), ("phi", _dp)]


class Opt(C.Structure):
    """Layout of SE_opt (SE_general.h:20-24)."""
    _fields_ = [("m", C.c_double), ("c", C.c_double), ("box", C.c_double * 3),
                ("h", C.c_double), ("xi", C.c_double), ("w", C.c_double),
                ("eta", C.c_double), ("P", C.c_int), ("M", C.c_int), ("N", C.c_int)]


def aligned_zeros(n, dtype=np.float64, align=64):
    """Zeroed array whose data starts on an `align`-byte boundary (the
    reference's SIMD kernels use aligned AVX loads, SE_fgg.h:46-54)."""
    dt = np.dtype(dtype)
    buf = np.zeros(n * dt.itemsize + align, dtype=np.uint8)
    off = (-buf.ctypes.data) % align
    return buf[off:off + n * dt.itemsize].view(dt)


def aligned_copy(a, dtype=np.float64):
    a = np.asarray(a, dtype=dtype).ravel()
    b = aligned_zeros(a.size, dtype)
    b[:] = a
    return b


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


_lib = None


def build() -> None:
    """Compile libse_oracle.so (and oracle/_ref when the reference is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "libse_oracle.so")
        if not os.path.exists(path):
            build()
        _lib = C.CDLL(path)
        _lib.orc_expand.restype = C.c_int
        _lib.orc_calc_energy.restype = C.c_double
        _lib.orc_per_size.restype = C.c_long
    return _lib


# ------------------------------------------------------------------ params --

@dataclass
class Setup:
    """Solver parameters derived as in parse_params (SE_general.c:16-29) and
    SE_FGG_FCN_params (SE_general.c:180-200)."""
    M: int
    P: int
    L: float
    xi: float
    m: float
    N: int

    def opt(self) -> Opt:
        o = Opt()
        o.m = self.m
        o.box[:] = (self.L, self.L, self.L)
        o.P, o.M, o.N = self.P, self.M, self.N
        lib().orc_parse_params(C.byref(o), C.c_double(self.xi))
        return o

    def params(self) -> FGGParams:
        p = FGGParams()
        o = self.opt()
        lib().orc_fcn_params(C.byref(p), C.byref(o), self.N)
        return p

    @property
    def eta(self) -> float:
        return self.opt().eta


def pack_params(N, M0, M1, M2, P, c, h, a=-1.0, b=-1.0) -> FGGParams:
    """SE_FGG_pack_params / SE2P_FGG_pack_params (offset a of the free z) /
    SE1P_FGG_pack_params (offsets a, b of the free x, y), SE_fgg.c:69-132."""
    p = FGGParams()
    lib().orc_pack_params(C.byref(p), N, M0, M1, M2, P, C.c_double(c), C.c_double(h),
                          C.c_double(a))
    p.b = b
    return p


def init_params(P: int, L: float, xi: float, q: np.ndarray):
    """SE_init_params (SE_general.c:517-572): returns (M, m)."""
    M = C.c_int(0)
    Pc = C.c_int(P)
    m = C.c_double(0)
    Q = C.c_double(0)
    q = np.ascontiguousarray(q, dtype=np.float64)
    lib().orc_init_params(C.byref(M), C.byref(Pc), C.byref(m), C.c_double(L),
                          C.c_double(xi), dptr(q), len(q), C.byref(Q))
    return M.value, m.value


def padded_shape(p: FGGParams):
    return tuple(p.npdims)


# --------------------------------------------------------------- FGG steps --

def base_gaussian(p: FGGParams) -> np.ndarray:
    zs = np.zeros(p.P ** 3)
    lib().orc_base_gaussian(dptr(zs), C.byref(p))
    return zs


def expand_all(p: FGGParams, x: np.ndarray, periodicity=3, force=False) -> dict:
    N, P = p.N, p.P
    out = {k: np.zeros(N * P) for k in ("zx", "zy", "zz")}
    if force:
        out.update({k: np.zeros(N * P) for k in ("zfx", "zfy", "zfz")})
    out["idx"] = np.zeros(N, dtype=np.int32)
    nul = _dp()
    lib().orc_expand_all(C.byref(p), dptr(np.ascontiguousarray(x)), periodicity, int(force),
                         dptr(out["zx"]), dptr(out["zy"]), dptr(out["zz"]),
                         dptr(out["zfx"]) if force else nul, dptr(out["zfy"]) if force else nul,
                         dptr(out["zfz"]) if force else nul, iptr(out["idx"]))
    return out


def grid_split(p, q, zs, ex, force_order=0, H=None):
    H = np.zeros(int(np.prod(p.npdims))) if H is None else H
    lib().orc_grid_split(dptr(H), dptr(q), dptr(zs), dptr(ex["zx"]), dptr(ex["zy"]),
                         dptr(ex["zz"]), iptr(ex["idx"]), C.byref(p), int(force_order))
    return H


def grid(p, x, q, zs, periodicity=3, H=None):
    H = np.zeros(int(np.prod(p.npdims))) if H is None else H
    lib().orc_grid(dptr(H), dptr(x), dptr(q), dptr(zs), C.byref(p), periodicity)
    return H


def per_size(p, periodicity=3) -> int:
    """Elements of the periodic grid of the wrap / extend calls (orc_per_size)."""
    return int(lib().orc_per_size(C.byref(p), periodicity))


def wrap(p, H, periodicity=3, H_per=None):
    H_per = np.zeros(per_size(p, periodicity)) if H_per is None else H_per
    lib().orc_wrap(dptr(H_per), dptr(H), C.byref(p), periodicity)
    return H_per


def extend(p, H_per, periodicity=3):
    H = np.zeros(int(np.prod(p.npdims)))
    lib().orc_extend(dptr(H), dptr(H_per), C.byref(p), periodicity)
    return H


def int_split(p, H, zs, ex, accumulate=False, phi=None):
    phi = np.zeros(p.N) if phi is None else phi
    lib().orc_int_split(dptr(phi), dptr(H), dptr(zs), dptr(ex["zx"]), dptr(ex["zy"]),
                        dptr(ex["zz"]), iptr(ex["idx"]), C.byref(p), int(accumulate))
    return phi


def int_vanilla(p, H, x, zs, periodicity=3):
    phi = np.zeros(p.N)
    lib().orc_int(dptr(phi), dptr(H), dptr(x), dptr(zs), C.byref(p), periodicity)
    return phi


def int_split_force(p, q, H, zs, ex):
    f = np.zeros(3 * p.N)
    lib().orc_int_split_force(dptr(f), dptr(q), dptr(H), dptr(zs), dptr(ex["zx"]),
                              dptr(ex["zy"]), dptr(ex["zz"]), dptr(ex["zfx"]),
                              dptr(ex["zfy"]), dptr(ex["zfz"]), iptr(ex["idx"]), C.byref(p))
    return f


def int_force_vanilla(p, H, x, q, zs):
    f = np.zeros(3 * p.N)
    lib().orc_int_force(dptr(f), dptr(H), dptr(x), dptr(q), dptr(zs), C.byref(p))
    return f


# ----------------------------------------------------------------- k-space --

def scaling(scalar: float, M: int, L: float) -> np.ndarray:
    Z = np.zeros(M ** 3)
    box = np.array([L, L, L])
    lib().orc_scaling(C.c_double(scalar), dptr(Z), M, M, M, dptr(box))
    return Z


def kspace_solve(H_per: np.ndarray, M: int, L: float, xi: float, eta: float) -> np.ndarray:
    """spectral_ewald.c:119-134: C2C forward FFT of the wrapped grid, multiply
    by Z (with Z[0] = 0), backward FFT, real part."""
    Z = scaling(-(1. - eta) / (4. * xi * xi), M, L)
    Z[0] = 0.
    G = np.fft.fftn(H_per.reshape(M, M, M))
    G *= Z.reshape(M, M, M)
    return np.ascontiguousarray(np.real(np.fft.ifftn(G)) * float(M) ** 3).reshape(-1)


# ------------------------------------------------------------- full solve --

def spectral_ewald(x, q, M, P, m, L, xi, mode="potential", split=True,
                   int_accumulate=False, phi_init=None):
    """The SE k-space solve of spectral_ewald.c:20-182 (3P)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    N = len(q)
    s = Setup(M=M, P=P, L=L, xi=xi, m=m, N=N)
    p = s.params()
    eta = s.eta
    zs = base_gaussian(p)
    force = mode == "force"
    if split:
        ex = expand_all(p, x, 3, force)
        H = grid_split(p, q, zs, ex, force_order=int(force))
    else:
        H = grid(p, x, q, zs, 3)
    H_per = wrap(p, H, 3)
    H_in = kspace_solve(H_per, M, L, xi, eta)
    H = extend(p, H_in, 3)
    if force:
        return int_split_force(p, q, H, zs, ex) if split else int_force_vanilla(p, H, x, q, zs)
    if split:
        phi = np.zeros(N) if phi_init is None else np.array(phi_init, dtype=np.float64)
        return int_split(p, H, zs, ex, accumulate=int_accumulate, phi=phi)
    return int_vanilla(p, H, x, zs, 3)


# ------------------------------------------------------------ direct sums --

def direct_fd(x, q, L, xi, layers):
    N = len(q)
    phi = np.zeros(N)
    box = np.array([L, L, L], dtype=np.float64)
    lib().orc_direct_fd(dptr(phi), dptr(np.ascontiguousarray(x)), dptr(np.ascontiguousarray(q)),
                        N, dptr(box), C.c_double(xi), layers)
    return phi


def direct_real(x, q, L, xi, layers, rc=0.0, phi=None):
    """Real-space Ewald potential (SE_direct.c:464-549): rc <= 0 no cutoff."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros(len(q)) if phi is None else np.array(phi, dtype=np.float64)
    box = np.array([L, L, L], dtype=np.float64)
    lib().orc_direct_real(dptr(out), dptr(x), dptr(q), len(q), dptr(box), C.c_double(xi),
                          int(layers), C.c_double(rc))
    return out


def direct_self(q, xi, phi=None):
    """Self term phi -= 2 xi / sqrt(pi) q (SE_direct.c:551-562)."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros(len(q)) if phi is None else np.array(phi, dtype=np.float64)
    lib().orc_direct_self(dptr(out), dptr(q), len(q), C.c_double(xi))
    return out


def direct_real_force(x, q, L, xi, layers, rc=0.0):
    """Force of the real-space potential (its gradient times -q; no
    counterpart in the reference)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros(3 * len(q))
    box = np.array([L, L, L], dtype=np.float64)
    lib().orc_direct_real_force(dptr(out), dptr(x), dptr(q), len(q), dptr(box),
                                C.c_double(xi), int(layers), C.c_double(rc))
    return out


def direct_force_fd(x, q, L, xi, layers):
    N = len(q)
    f = np.zeros(3 * N)
    box = np.array([L, L, L], dtype=np.float64)
    lib().orc_direct_force_fd(dptr(f), dptr(np.ascontiguousarray(x)),
                              dptr(np.ascontiguousarray(q)), N, dptr(box), C.c_double(xi),
                              layers)
    return f


def kspace_converged_jmax(L, xi, tol=1e-18):
    """Half-width (in units of 2 pi/L) beyond which e^{-k^2/4xi^2} < tol."""
    kmax = 2. * xi * np.sqrt(-np.log(tol))
    return int(np.ceil(kmax * L / (2 * PI))), kmax * kmax


def sf_kspace(x, q, L, xi, targets, jmax=None, kcut2=None, want_phi=True, want_force=True):
    """Direct k-space Ewald sums (SE_direct.c:377-461) through structure
    factors, for the listed target particles."""
    N = len(q)
    if jmax is None:
        jmax, kc2 = kspace_converged_jmax(L, xi)
        kcut2 = kc2 if kcut2 is None else kcut2
    kcut2 = -1.0 if kcut2 is None else kcut2
    targets = np.ascontiguousarray(targets, dtype=np.int32)
    T = len(targets)
    phi = np.zeros(T) if want_phi else None
    f = np.zeros(3 * T) if want_force else None
    box = np.array([L, L, L], dtype=np.float64)
    lib().orc_sf_kspace(dptr(np.ascontiguousarray(x)), dptr(np.ascontiguousarray(q)), N,
                        dptr(box), C.c_double(xi), int(jmax), C.c_double(kcut2), iptr(targets),
                        T, dptr(phi) if want_phi else _dp(), dptr(f) if want_force else _dp())
    return phi, f


def sf_kspace_torch(x, q, L, xi, targets, jmax, kcut2, device="cpu", chunk=4096):
    """The structure-factor k-space Ewald sum of :func:`sf_kspace`
    (SE_direct.c:377-461: potential, and the force with its 1/2 factor) in
    torch complex128 arithmetic on any device, for systems whose O(K N) cost
    is out of reach on the host (millions of particles, tens of thousands of
    wave vectors).  It is a checker like the rest of this module: the full
    cube |j_d| <= jmax of wave vectors k = 2 pi j / L, k != 0, |k|^2 <= kcut2
    (kcut2 <= 0: no sphere), S(k) = sum_n q_n e^{i k.x_n} built in particle
    chunks as one complex GEMM per chunk, then
      phi_t = 4pi/V sum_k e^{-k^2/4xi^2}/k^2 Re(S(k) e^{-i k.x_t}),
      F_t   = 1/2 q_t 4pi/V sum_k e^{-k^2/4xi^2}/k^2 k Im(S(k) e^{-i k.x_t}).
    Returns (phi[T], force[3T] SoA) as numpy arrays."""
    import torch
    dev = torch.device(device)
    x = torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=dev)
    q = torch.as_tensor(np.ascontiguousarray(q, dtype=np.float64), device=dev)
    N = q.numel()
    J = int(jmax)
    nj = 2 * J + 1
    kf = 2.0 * PI / L
    js = torch.arange(-J, J + 1, device=dev, dtype=torch.float64)

    def phases(v, sign):   # e^{sign i kf j v}, (len(v), nj)
        return torch.polar(torch.ones(v.numel(), nj, dtype=torch.float64, device=dev),
                           sign * kf * v[:, None] * js[None, :])

    S = torch.zeros(nj, nj * nj, dtype=torch.complex128, device=dev)
    for c0 in range(0, N, chunk):
        c1 = min(N, c0 + chunk)
        ex = phases(x[c0:c1], 1.0) * q[c0:c1, None]
        ey = phases(x[N + c0:N + c1], 1.0)
        ez = phases(x[2 * N + c0:2 * N + c1], 1.0)
        W = (ey[:, :, None] * ez[:, None, :]).reshape(c1 - c0, nj * nj)
        S += ex.transpose(0, 1) @ W
    S = S.reshape(nj, nj, nj)
    k = kf * js
    K2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    keep = K2 > 0
    if kcut2 is not None and kcut2 > 0:
        keep &= K2 <= kcut2
    g = torch.where(keep, torch.exp(-K2 / (4.0 * xi * xi)) / torch.where(keep, K2, 1.0),
                    torch.zeros_like(K2))
    G = g * S
    t = torch.as_tensor(np.ascontiguousarray(targets, dtype=np.int64), device=dev)
    et_x = phases(x[t], -1.0)
    et_y = phases(x[N + t], -1.0)
    et_z = phases(x[2 * N + t], -1.0)

    def at_targets(F):   # sum_k F(k) e^{-i k.x_t}
        A = (et_x @ F.reshape(nj, nj * nj)).reshape(-1, nj, nj)
        B = torch.einsum("tb,tbc->tc", et_y, A)
        return torch.einsum("tc,tc->t", et_z, B)

    pref = 4.0 * PI / (L * L * L)
    phi = pref * at_targets(G).real
    qt = q[t]
    force = torch.cat([0.5 * pref * qt * at_targets(G * kd).imag for kd in
                       (k[:, None, None], k[None, :, None], k[None, None, :])])
    return phi.cpu().numpy(), force.cpu().numpy()


# -------------------------------------------------------------- reductions --

def calc_energy(phi, q):
    return lib().orc_calc_energy(dptr(np.ascontiguousarray(phi)),
                                 dptr(np.ascontiguousarray(q)), len(q))


def counting_sort(keys: np.ndarray, nkeys: int):
    keys = np.ascontiguousarray(keys, dtype=np.int32)
    perm = np.zeros(len(keys), dtype=np.int32)
    offs = np.zeros(nkeys + 1, dtype=np.int32)
    lib().orc_counting_sort(iptr(keys), len(keys), nkeys, iptr(perm), iptr(offs))
    return perm, offs


def reorder(x, q, idx):
    x = np.array(x, dtype=np.float64)
    q = np.array(q, dtype=np.float64)
    lib().orc_reorder(dptr(x), dptr(q), iptr(np.ascontiguousarray(idx, dtype=np.int32)), len(q))
    return x, q


def rel_rms(a, b):
    """||a - b||_2 / ||b||_2 over all entries."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


def abs_rms(a, b):
    """sqrt(mean((a-b)^2)), the error measure of test_accuracy.c:107-118."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.sqrt(np.mean((a - b) ** 2)))


# -------------------------------------------------------------- the reference --

def ref_lib(kind="pot"):
    """The reference compiled from its sources (oracle/_ref/libse_ref_<kind>.so),
    or None when it was not built (e.g. on a machine without the sources)."""
    path = os.path.join(REF_DIR, f"libse_ref_{kind}.so")
    if not os.path.exists(path):
        return None
    return C.CDLL(path)


def ref_spectral_ewald(reflib, x, q, M, P, m, L, xi, out_len):
    """Run the reference's own spectral_ewald() (spectral_ewald.c:20-182)."""
    N = len(q)
    o = Opt()
    o.m = m
    o.box[:] = (L, L, L)
    o.P, o.M, o.N = P, M, N
    out = aligned_zeros(out_len)
    energy = aligned_zeros(N)
    reflib.spectral_ewald.restype = C.c_int
    reflib.spectral_ewald.argtypes = [_dp, _dp, Opt, C.c_double, _dp, _dp]
    reflib.spectral_ewald(dptr(aligned_copy(x)), dptr(aligned_copy(q)), o,
                          C.c_double(xi), dptr(out), dptr(energy))
    return np.array(out)


# ------------------------------------------------------- synthetic inputs --

def synthetic_system(N: int, L: float = 1.0, seed: int = 0, charges="pm1",
                     clusters: int = 0, sigma: float = 0.02):
    """Seeded particle system: positions in [0, L)^3 (SoA, x[n], x[n+N],
    x[n+2N]), charges +-1 with zero sum ('pm1') or uniform in [-1, 1] shifted
    to zero sum ('uniform').  With clusters > 0 positions are drawn from that
    many isotropic Gaussians of width sigma*L with uniform centres, wrapped."""
    rng = np.random.Generator(np.random.Philox(seed))
    if clusters > 0:
        centres = rng.random((clusters, 3)) * L
        which = rng.integers(0, clusters, size=N)
        pos = centres[which] + rng.normal(0.0, sigma * L, size=(N, 3))
        pos = np.mod(pos, L)
    else:
        pos = rng.random((N, 3)) * L
    pos[pos >= L] = 0.0
    if charges == "pm1":
        q = np.ones(N)
        q[N // 2:] = -1.0
        if N % 2:
            q[-1] = 0.0
        rng.shuffle(q)
    else:
        q = rng.uniform(-1.0, 1.0, size=N)
        q -= q.mean()
    x = np.ascontiguousarray(pos.T.reshape(-1))
    return x, np.ascontiguousarray(q)


def c1_params(P=21):
    """m = 0.94 sqrt(pi P) as in the configuration of the plain FP64 case."""
    return 0.94 * np.sqrt(PI * P)

"""Python view of the reference C interface (SE_fgg.h / SE_general.h) as
exported by libse_gpu.so.

The functions keep the reference names and argument meaning; buffers are
numpy arrays (host memory, staged by the library), torch CUDA tensors (used in
place) or library-allocated managed memory (SE_FGG_allocate_*).  Each call
raises SEError when the library reports a failure.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import SE_FGG_params, SE_FGG_work, SE_opt, SE_state, legacy_check, lib

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def dptr(a):
    """double* of a numpy array or torch CUDA tensor (None -> NULL)."""
    if a is None:
        return _dp()
    if isinstance(a, np.ndarray):
        assert a.dtype == np.float64 and a.flags.c_contiguous
        return a.ctypes.data_as(_dp)
    assert a.dtype.__str__() == "torch.float64" and a.is_contiguous()
    return C.cast(C.c_void_p(a.data_ptr()), _dp)


def iptr(a):
    if a is None:
        return _ip()
    if isinstance(a, np.ndarray):
        assert a.dtype == np.int32 and a.flags.c_contiguous
        return a.ctypes.data_as(_ip)
    assert a.dtype.__str__() == "torch.int32" and a.is_contiguous()
    return C.cast(C.c_void_p(a.data_ptr()), _ip)


def call(name: str, *args):
    """Call a legacy (void) entry point and raise on a reported failure."""
    r = getattr(lib(), name)(*args)
    legacy_check(name)
    return r


def fcn_params(M: int, P: int, L: float, xi: float, m: float, N: int) -> tuple[SE_opt, SE_FGG_params]:
    """parse_params + SE_FGG_FCN_params (SE_general.c:16-29, 180-200)."""
    o = SE_opt()
    o.m = m
    o.box[:] = (L, L, L)
    o.P, o.M, o.N = P, M, N
    lib().parse_params(C.byref(o), C.c_double(xi))
    p = SE_FGG_params()
    lib().SE_FGG_FCN_params(C.byref(p), C.byref(o), N)
    return o, p


def pack_params(N, M0, M1, M2, P, c, h, a=None, b=None) -> SE_FGG_params:
    """SE_FGG_pack_params; with a, SE2P_FGG_pack_params (z free); with a and
    b, SE1P_FGG_pack_params (x and y free) -- SE_fgg.c:69-132."""
    p = SE_FGG_params()
    if a is None:
        lib().SE_FGG_pack_params(C.byref(p), N, M0, M1, M2, P, C.c_double(c), C.c_double(h))
    elif b is None:
        lib().SE2P_FGG_pack_params(C.byref(p), N, M0, M1, M2, P, C.c_double(c), C.c_double(h),
                                   C.c_double(a))
    else:
        lib().SE1P_FGG_pack_params(C.byref(p), N, M0, M1, M2, P, C.c_double(c), C.c_double(h),
                                   C.c_double(a), C.c_double(b))
    return p


def per_size(p: SE_FGG_params, periodicity: int = 3) -> int:
    """Elements of the periodic grid SE*_FGG_wrap_fcn writes and
    SE*_FGG_extend_fcn reads: 3P M0 M1 M2, 2P M0 M1 (M2 + P), 1P the reach of
    the reference's overlapping column-major map of the padded x, y."""
    m0, m1, m2 = p.dims
    if periodicity == 2:
        return m0 * m1 * p.npdims[2]
    if periodicity == 1:
        return (p.npdims[0] - 1) + (p.npdims[1] - 1) * m0 + (m2 - 1) * m0 * m1 + 1
    return m0 * m1 * m2


class Work:
    """An SE_FGG_work whose arrays are owned here (numpy or torch) or, with
    where='managed', allocated by SE_FGG_allocate_workspace(_SSE_force)."""

    def __init__(self, p: SE_FGG_params, force=False, where="host", periodic_z=True):
        self.p, self.force, self.where = p, force, where
        self.s = SE_FGG_work()
        n_pad = p.npdims[0] * p.npdims[1] * p.npdims[2]
        NP = p.N * p.P
        if where == "managed":
            fn = "SE_FGG_allocate_workspace_SSE_force" if force else "SE_FGG_allocate_workspace"
            call(fn, C.byref(self.s), C.byref(p), 1, 1)
            self.arrays = None
            return
        if where == "host":
            z = lambda n, dt=np.float64: np.zeros(max(n, 1), dtype=dt)
        else:
            import torch
            z = lambda n, dt=np.float64: torch.zeros(
                max(n, 1), dtype=torch.float64 if dt == np.float64 else torch.int32, device="cuda")
        self.arrays = {"H": z(n_pad), "zs": z(p.P ** 3), "zx": z(NP), "zy": z(NP), "zz": z(NP),
                       "idx": z(p.N, np.int32)}
        if force:
            self.arrays.update({"zfx": z(NP), "zfy": z(NP), "zfz": z(NP)})
        for k, v in self.arrays.items():
            setattr(self.s, k, iptr(v) if k == "idx" else dptr(v))
        self.s.free_zs = 0
        self.s.free_fgg_expa = 0

    def get(self, name: str) -> np.ndarray:
        """A host copy of one work array."""
        p = self.p
        n = {"H": p.npdims[0] * p.npdims[1] * p.npdims[2], "zs": p.P ** 3, "idx": p.N}.get(name, p.N * p.P)
        if self.arrays is not None:
            a = self.arrays[name]
            a = a.cpu().numpy() if hasattr(a, "cpu") else a
            return np.array(a[:n])
        ptr = getattr(self.s, name)
        ct = C.c_int if name == "idx" else C.c_double
        buf = C.cast(ptr, C.POINTER(ct * n)).contents
        return np.array(np.frombuffer(buf, dtype=np.int32 if name == "idx" else np.float64))

    def free(self):
        if self.where == "managed":
            fn = "SE_FGG_free_workspace_SSE_force" if self.force else "SE_FGG_free_workspace"
            getattr(lib(), fn)(C.byref(self.s))
            self.where = "freed"


def state(x, q, phi=None) -> SE_state:
    st = SE_state()
    st.x, st.q, st.phi = dptr(x), dptr(q), dptr(phi)
    return st

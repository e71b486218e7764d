"""Device-resident Spectral Ewald solves (se_gpu.h) for torch CUDA tensors.

Positions follow the reference layout: one float64 vector of length 3N,
x[n], x[n+N], x[n+2N] (SE_state, SE_fgg.h:142-148).  FORCE results are the
same SoA layout.  Nothing here computes on the CPU: every call goes to
libse_gpu.so on the current CUDA device and stream.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import SE_FORCE, SE_FP32, SE_FP64, SE_POTENTIAL, check, lib

PI = 3.14159265358979323846


def _mode(mode) -> int:
    if mode in (SE_POTENTIAL, "potential", "POTENTIAL"):
        return SE_POTENTIAL
    if mode in (SE_FORCE, "force", "FORCE"):
        return SE_FORCE
    raise ValueError(f"mode {mode!r}: expected 'potential' or 'force'")


def _prec(p) -> int:
    if p in (SE_FP64, "fp64", "float64", torch.float64):
        return SE_FP64
    if p in (SE_FP32, "fp32", "float32", torch.float32):
        return SE_FP32
    if p in (_lib.SE_FP32_FFT32, "fp32-fft32"):
        return _lib.SE_FP32_FFT32
    raise ValueError(f"precision {p!r}: expected 'fp64', 'fp32' or 'fp32-fft32'")


def _stream(stream) -> C.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _ptr(t: torch.Tensor | None) -> C.c_void_p:
    if t is None:
        return C.c_void_p(0)
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return C.c_void_p(t.data_ptr())


def default_path(M: int, P: int) -> int:
    """The SE_PATH_* bits the default kernel choice gives grid M, stencil P."""
    return int(lib().se_default_path(int(M), int(P)))


def default_m(P: int) -> float:
    """Gaussian shape factor m = 0.94 sqrt(pi P)."""
    return 0.94 * math.sqrt(PI * P)


@dataclass(frozen=True)
class Params:
    """Derived FGG parameters (parse_params, SE_general.c:16-29)."""
    h: float
    w: float
    eta: float
    c: float
    d: float


def choose_params(eps: float, L: float, xi: float, q, mode="potential") -> tuple[int, int, float]:
    """(M, P, m) for an absolute RMS error target eps (se_choose_params): the
    smallest P whose Lindbo-Tornberg estimate (SE_init_params,
    SE_general.c:517-572) is <= eps, the Kolafa-Perram grid rounded for the
    tile-aligned kernels.  q: the charges (or their sum of squares)."""
    Q = float(q) if np.isscalar(q) else float(np.sum(np.asarray(q, dtype=np.float64) ** 2))
    M, P, m = C.c_int(), C.c_int(), C.c_double()
    check(lib().se_choose_params(float(eps), float(L), float(xi), Q, _mode(mode), C.byref(M),
                                 C.byref(P), C.byref(m)), "se_choose_params")
    return M.value, P.value, m.value


def error_estimate(P: int, L: float, xi: float, q, mode="potential") -> float:
    """The Lindbo-Tornberg error estimate SE_init_params prints."""
    Q = float(q) if np.isscalar(q) else float(np.sum(np.asarray(q, dtype=np.float64) ** 2))
    return float(lib().se_error_estimate(int(P), float(L), float(xi), Q, _mode(mode)))


def derive(M: int, P: int, L: float, xi: float, m: float) -> Params:
    cfg = _lib.se_config(M=M, P=P, L=L, xi=xi, m=m, mode=0, precision=0, max_particles=0)
    out = [C.c_double() for _ in range(5)]
    check(lib().se_config_derive(C.byref(cfg), *[C.byref(o) for o in out]), "se_config_derive")
    return Params(*(o.value for o in out))


class SpectralEwald:
    """A plan for k-space SE solves of one cubic 3P system of up to
    ``max_particles`` particles (se_plan_create)."""

    def __init__(self, M: int, P: int, L: float = 1.0, xi: float = 8.0, m: float | None = None,
                 mode="potential", precision="fp64", max_particles: int = 0, path=None):
        """path: None (the default kernels), "tune" (timed choice,
        se_plan_create_ex with SE_PATH_TUNE) or SE_PATH_* bits."""
        self.M, self.P, self.L, self.xi = int(M), int(P), float(L), float(xi)
        self.m = float(default_m(P) if m is None else m)
        self.mode = _mode(mode)
        self.precision = _prec(precision)
        self.max_particles = int(max_particles)
        self.cfg = _lib.se_config(M=self.M, P=self.P, L=self.L, xi=self.xi, m=self.m,
                                  mode=self.mode, precision=self.precision,
                                  max_particles=self.max_particles)
        self._plan = C.c_void_p()
        if path is None:
            check(lib().se_plan_create(C.byref(self._plan), C.byref(self.cfg)), "se_plan_create")
        else:
            code = _lib.SE_PATH_TUNE if path == "tune" else int(path)
            check(lib().se_plan_create_ex(C.byref(self._plan), C.byref(self.cfg), code),
                  "se_plan_create_ex")
        self.params = derive(self.M, self.P, self.L, self.xi, self.m)

    @property
    def out_width(self) -> int:
        return 3 if self.mode == SE_FORCE else 1

    @property
    def path(self) -> int:
        """The kernel path this plan runs (SE_PATH_* bits)."""
        return int(lib().se_plan_path(self._plan))

    def device_bytes(self) -> int:
        return int(lib().se_plan_device_bytes(C.byref(self.cfg)))

    def solve(self, x: torch.Tensor, q: torch.Tensor, out: torch.Tensor | None = None,
              phi_out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        N = q.numel()
        if x.numel() != 3 * N:
            raise ValueError("x must hold 3N coordinates (SoA)")
        if out is None:
            out = torch.empty(self.out_width * N, dtype=torch.float64, device=q.device)
        check(lib().se_solve(self._plan, N, _ptr(x), _ptr(q), _ptr(out), _ptr(phi_out),
                             _stream(stream)), "se_solve")
        return out

    def solve_system(self, system: "System", x: torch.Tensor, q: torch.Tensor,
                     out: torch.Tensor | None = None, phi_out: torch.Tensor | None = None,
                     stream=None) -> torch.Tensor:
        """Solve `system` (same M, P and mode as the plan; its own N, L, xi,
        m) on this plan (se_solve_system)."""
        if x.numel() != 3 * system.N or q.numel() != system.N:
            raise ValueError("x, q sizes do not match system.N")
        if out is None:
            out = torch.empty(self.out_width * system.N, dtype=torch.float64, device=q.device)
        s = system.c_struct()
        check(lib().se_solve_system(self._plan, C.byref(s), _ptr(x), _ptr(q), _ptr(out),
                                    _ptr(phi_out), _stream(stream)), "se_solve_system")
        return out

    def solve_host(self, x: np.ndarray, q: np.ndarray, out: np.ndarray | None = None,
                   stream=None) -> np.ndarray:
        """Host buffers in and out (copies inside, waits for the result)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        N = q.size
        if out is None:
            out = np.empty(self.out_width * N, dtype=np.float64)
        check(lib().se_solve_host(self._plan, N, C.c_void_p(x.ctypes.data),
                                  C.c_void_p(q.ctypes.data), C.c_void_p(out.ctypes.data),
                                  _stream(stream)), "se_solve_host")
        return out

    def solve_host_ptr(self, N: int, x_ptr: int, q_ptr: int, out_ptr: int, stream=None) -> None:
        check(lib().se_solve_host(self._plan, N, C.c_void_p(x_ptr), C.c_void_p(q_ptr),
                                  C.c_void_p(out_ptr), _stream(stream)), "se_solve_host")

    def spread(self, x, q, grid=None, stream=None) -> torch.Tensor:
        if grid is None:
            grid = torch.empty((self.M,) * 3, dtype=torch.float64, device=q.device)
        check(lib().se_spread(self._plan, q.numel(), _ptr(x), _ptr(q), _ptr(grid),
                              _stream(stream)), "se_spread")
        return grid

    def kspace(self, grid, stream=None) -> torch.Tensor:
        check(lib().se_kspace(self._plan, _ptr(grid), _stream(stream)), "se_kspace")
        return grid

    def interp(self, x, q, grid, out=None, phi_out=None, stream=None) -> torch.Tensor:
        N = q.numel()
        if out is None:
            out = torch.empty(self.out_width * N, dtype=torch.float64, device=q.device)
        check(lib().se_interp(self._plan, N, _ptr(x), _ptr(q), _ptr(grid), _ptr(out),
                              _ptr(phi_out), _stream(stream)), "se_interp")
        return out

    @property
    def launches(self) -> int:
        """Kernels of this library the last solve launched (cuFFT's not counted)."""
        return int(lib().se_plan_launch_count(self._plan))

    def set_timing(self, on: bool = True) -> None:
        check(lib().se_plan_set_timing(self._plan, int(on)), "se_plan_set_timing")

    def set_graph(self, on: bool = True) -> None:
        """Replay repeated solves on the same buffers from a CUDA graph
        (se_plan_set_graph)."""
        check(lib().se_plan_set_graph(self._plan, int(on)), "se_plan_set_graph")

    def stage_ms(self) -> dict:
        """CUDA-event milliseconds of the last solve's stages (timing on)."""
        ms = (C.c_float * 4)()
        check(lib().se_plan_stage_ms(self._plan, C.byref(ms)), "se_plan_stage_ms")
        return dict(zip(("sort", "spread", "kspace", "interp"), (float(v) for v in ms)))

    def close(self) -> None:
        if self._plan:
            lib().se_plan_destroy(self._plan)
            self._plan = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class System:
    """One independent system of a batch (se_system)."""
    N: int
    M: int
    P: int
    L: float
    xi: float
    m: float | None = None
    mode: str = "potential"

    def c_struct(self) -> _lib.se_system:
        return _lib.se_system(N=self.N, M=self.M, P=self.P, L=self.L, xi=self.xi,
                              m=default_m(self.P) if self.m is None else self.m,
                              mode=_mode(self.mode))

    @property
    def out_width(self) -> int:
        return 3 if _mode(self.mode) == SE_FORCE else 1


class BatchSolver:
    """Many independent systems in one set of launches (se_batch_*)."""

    def __init__(self, systems: list[System], precision="fp32", paths=None):
        """paths: None (the default kernels) or one SE_PATH_* bit set per
        system (se_batch_create_ex)."""
        self.systems = list(systems)
        self.precision = _prec(precision)
        arr = (_lib.se_system * len(self.systems))(*[s.c_struct() for s in self.systems])
        self._arr = arr
        self._b = C.c_void_p()
        if paths is None:
            check(lib().se_batch_create(C.byref(self._b), arr, len(self.systems),
                                        self.precision), "se_batch_create")
        else:
            if len(paths) != len(self.systems):
                raise ValueError("one path per system")
            pa = (C.c_int * len(paths))(*[int(v) for v in paths])
            check(lib().se_batch_create_ex(C.byref(self._b), arr, len(self.systems),
                                           self.precision, pa), "se_batch_create_ex")
        self.part_off = np.concatenate([[0], np.cumsum([s.N for s in self.systems])])
        self.out_off = np.concatenate([[0], np.cumsum([s.N * s.out_width for s in self.systems])])

    @staticmethod
    def device_bytes(systems, precision="fp32") -> int:
        arr = (_lib.se_system * len(systems))(*[s.c_struct() for s in systems])
        return int(lib().se_batch_device_bytes(arr, len(systems), _prec(precision)))

    def pack(self, xs, qs, device="cuda"):
        """Concatenate per-system (x SoA, q) into the batch layout."""
        x = torch.cat([torch.as_tensor(v, dtype=torch.float64).reshape(-1) for v in xs])
        q = torch.cat([torch.as_tensor(v, dtype=torch.float64).reshape(-1) for v in qs])
        return x.to(device).contiguous(), q.to(device).contiguous()

    def solve(self, x: torch.Tensor, q: torch.Tensor, out: torch.Tensor | None = None,
              stream=None) -> torch.Tensor:
        if out is None:
            out = torch.empty(int(self.out_off[-1]), dtype=torch.float64, device=q.device)
        check(lib().se_batch_solve(self._b, _ptr(x), _ptr(q), _ptr(out), _stream(stream)),
              "se_batch_solve")
        return out

    def split(self, out: torch.Tensor):
        return [out[int(self.out_off[i]):int(self.out_off[i + 1])] for i in range(len(self.systems))]

    @property
    def launches(self) -> int:
        return int(lib().se_batch_launch_count(self._b))

    def set_timing(self, on: bool = True) -> None:
        check(lib().se_batch_set_timing(self._b, int(on)), "se_batch_set_timing")

    def set_graph(self, on: bool = True) -> None:
        check(lib().se_batch_set_graph(self._b, int(on)), "se_batch_set_graph")

    def stage_ms(self) -> dict:
        ms = (C.c_float * 4)()
        check(lib().se_batch_stage_ms(self._b, C.byref(ms)), "se_batch_stage_ms")
        return dict(zip(("sort", "spread", "kspace", "interp"), (float(v) for v in ms)))

    def close(self) -> None:
        if self._b:
            lib().se_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fma_peak_tflops(stream=None) -> float:
    """Measured FP32 FMA throughput of the current GPU (TFLOP/s)."""
    v = C.c_double()
    check(lib().se_probe_fma_tflops(C.byref(v), _stream(stream)), "se_probe_fma_tflops")
    return v.value


def energy(phi: torch.Tensor, q: torch.Tensor, stream=None) -> torch.Tensor:
    """E = 1/2 sum phi q (calc_energy, SE_fgg.c:5934-5946), FP64 on the GPU."""
    e = torch.empty(1, dtype=torch.float64, device=q.device)
    check(lib().se_energy(_ptr(phi), _ptr(q), q.numel(), _ptr(e), _stream(stream)), "se_energy")
    return e


def counting_sort(keys: torch.Tensor, nkeys: int, stream=None):
    """Stable counting sort on the GPU: (perm, offsets), bit-exact with a CPU
    stable sort."""
    keys = keys.to(torch.int32).contiguous()
    N = keys.numel()
    perm = torch.empty(max(N, 1), dtype=torch.int32, device=keys.device)
    offs = torch.empty(nkeys + 1, dtype=torch.int32, device=keys.device)
    nb = int(lib().se_sort_scratch_bytes(N, nkeys))
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device=keys.device)
    check(lib().se_counting_sort(_ptr(keys), N, nkeys, _ptr(perm), _ptr(offs), _ptr(scratch),
                                 nb, _stream(stream)), "se_counting_sort")
    return perm[:N], offs


def real_space(x: torch.Tensor, q: torch.Tensor, L: float, xi: float, layers: int = 1,
               rc: float = 0.0, phi: torch.Tensor | None = None, force: torch.Tensor | None = None,
               want_force: bool = False, stream=None):
    """Real-space Ewald potential (and force) of a cubic box, accumulated into
    phi / force (se_real_space; SE3P_direct_real_rc, SE_direct.c:464-506).
    Returns (phi, force)."""
    N = q.numel()
    if phi is None:
        phi = torch.zeros(N, dtype=torch.float64, device=q.device)
    if want_force and force is None:
        force = torch.zeros(3 * N, dtype=torch.float64, device=q.device)
    check(lib().se_real_space(_ptr(x), _ptr(q), N, float(L), float(xi), int(layers), float(rc),
                              _ptr(phi), _ptr(force), _stream(stream)), "se_real_space")
    return phi, force


def self_term(q: torch.Tensor, xi: float, phi: torch.Tensor | None = None,
              stream=None) -> torch.Tensor:
    """phi -= 2 xi / sqrt(pi) q (se_self_term; SE3P_direct_self)."""
    if phi is None:
        phi = torch.zeros(q.numel(), dtype=torch.float64, device=q.device)
    check(lib().se_self_term(_ptr(q), q.numel(), float(xi), _ptr(phi), _stream(stream)),
          "se_self_term")
    return phi

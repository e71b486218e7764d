"""ctypes binding of libse_gpu.so (built in-tree by ``make -C csrc``).

There is no fallback: importing a compute entry point without the shared
library raises, so a missing build can never silently run something else.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libse_gpu.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


class SE_FGG_params(C.Structure):
    """SE_fgg.h:121-134."""
    _fields_ = [("N", C.c_int), ("P", C.c_int), ("P_half", C.c_int),
                ("dims", C.c_int * 3), ("npdims", C.c_int * 3),
                ("c", C.c_double), ("d", C.c_double), ("h", C.c_double),
                ("a", C.c_double), ("b", C.c_double)]


class SE_FGG_work(C.Structure):
    """SE_fgg.h:100-118."""
    _fields_ = [("H", _dp), ("zs", _dp), ("zx", _dp), ("zy", _dp), ("zz", _dp),
                ("idx", _ip), ("zfx", _dp), ("zfy", _dp), ("zfz", _dp),
                ("free_zs", C.c_int), ("free_fgg_expa", C.c_int)]


class SE_state(C.Structure):
    """SE_fgg.h:142-148."""
    _fields_ = [("x", _dp), ("q", _dp), ("phi", _dp)]


class SE_opt(C.Structure):
    """SE_general.h:20-24."""
    _fields_ = [("m", C.c_double), ("c", C.c_double), ("box", C.c_double * 3),
                ("h", C.c_double), ("xi", C.c_double), ("w", C.c_double),
                ("eta", C.c_double), ("P", C.c_int), ("M", C.c_int), ("N", C.c_int)]


class se_config(C.Structure):
    """se_gpu.h se_config."""
    _fields_ = [("M", C.c_int), ("P", C.c_int), ("L", C.c_double), ("xi", C.c_double),
                ("m", C.c_double), ("mode", C.c_int), ("precision", C.c_int),
                ("max_particles", C.c_int)]


class se_system(C.Structure):
    """se_gpu.h se_system."""
    _fields_ = [("N", C.c_int), ("M", C.c_int), ("P", C.c_int), ("L", C.c_double),
                ("xi", C.c_double), ("m", C.c_double), ("mode", C.c_int)]


class se_server_config(C.Structure):
    """se_gpu.h se_server_config."""
    _fields_ = [("slots", C.c_int), ("precision", C.c_int), ("hbm_budget", C.c_size_t),
                ("max_queue", C.c_int)]


class se_request(C.Structure):
    """se_gpu.h se_request."""
    _fields_ = [("sys", se_system), ("x", C.c_void_p), ("q", C.c_void_p), ("out", C.c_void_p),
                ("where", C.c_int)]


class se_completion(C.Structure):
    """se_gpu.h se_completion."""
    _fields_ = [("ticket", C.c_longlong), ("status", C.c_int), ("queue_s", C.c_double),
                ("latency_s", C.c_double)]


class se_server_stats(C.Structure):
    """se_gpu.h se_server_stats."""
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong),
                ("failed", C.c_longlong), ("queued", C.c_int), ("in_flight", C.c_int),
                ("plans", C.c_int), ("plans_created", C.c_longlong),
                ("plans_evicted", C.c_longlong), ("hbm_used", C.c_size_t),
                ("hbm_peak", C.c_size_t)]


SE_OK, SE_ERR_CUDA, SE_ERR_INVALID, SE_ERR_UNSUPPORTED, SE_ERR_NOMEM, SE_ERR_CUFFT, \
    SE_ERR_INPUT, SE_ERR_BUSY, SE_ERR_TIMEOUT = range(9)
SE_WHERE_HOST, SE_WHERE_DEVICE = 0, 1
SE_PATH_DEFAULT, SE_PATH_TUNE = -1, -2
SE_PATH_TILE_SPREAD, SE_PATH_PAIR_INTERP, SE_PATH_RUNTIME_P, SE_PATH_RADIX_SORT = 1, 2, 4, 8
SE_PATH_FFT3 = 16
SE_PATH_BIN_WINDOWS = 32
SE_POTENTIAL, SE_FORCE = 0, 1
SE_FP64, SE_FP32, SE_FP32_FFT32 = 0, 1, 2

_ERR_NAMES = {1: "CUDA error", 2: "invalid argument", 3: "unsupported", 4: "out of memory",
              5: "cuFFT error", 6: "non-finite position", 7: "queue full",
              8: "timed out"}


class SEError(RuntimeError):
    pass


_lib = None


def build(quiet: bool = True) -> None:
    """Compile libse_gpu.so for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-s" if quiet else "-w", "-j4", "-C", os.path.join(HERE, "csrc")],
                   check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {HERE}/csrc` "
                          "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    sig = {
        # device-resident API
        "se_config_derive": (C.c_int, [C.POINTER(se_config), _dp, _dp, _dp, _dp, _dp]),
        "se_plan_device_bytes": (C.c_size_t, [C.POINTER(se_config)]),
        "se_plan_create": (C.c_int, [C.POINTER(_vp), C.POINTER(se_config)]),
        "se_plan_destroy": (C.c_int, [_vp]),
        "se_solve": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp]),
        "se_solve_host": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp]),
        "se_spread": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp]),
        "se_kspace": (C.c_int, [_vp, _vp, _vp]),
        "se_interp": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp]),
        "se_energy": (C.c_int, [_vp, _vp, C.c_int, _vp, _vp]),
        "se_plan_launch_count": (C.c_int, [_vp]),
        "se_gpu_error_detail": (C.c_char_p, []),
        "se_sort_scratch_bytes": (C.c_size_t, [C.c_int, C.c_int]),
        "se_counting_sort": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, _vp, C.c_size_t, _vp]),
        "se_batch_create": (C.c_int, [C.POINTER(_vp), C.POINTER(se_system), C.c_int, C.c_int]),
        "se_default_path": (C.c_int, [C.c_int, C.c_int]),
        "se_batch_create_ex": (C.c_int, [C.POINTER(_vp), C.POINTER(se_system), C.c_int, C.c_int,
                                         C.POINTER(C.c_int)]),
        "se_batch_destroy": (C.c_int, [_vp]),
        "se_batch_device_bytes": (C.c_size_t, [C.POINTER(se_system), C.c_int, C.c_int]),
        "se_batch_solve": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
        "se_batch_launch_count": (C.c_int, [_vp]),
        "se_plan_set_timing": (C.c_int, [_vp, C.c_int]),
        "se_plan_stage_ms": (C.c_int, [_vp, C.POINTER(C.c_float * 4)]),
        "se_batch_set_timing": (C.c_int, [_vp, C.c_int]),
        "se_batch_stage_ms": (C.c_int, [_vp, C.POINTER(C.c_float * 4)]),
        "se_probe_fma_tflops": (C.c_int, [_dp, _vp]),
        "se_plan_set_graph": (C.c_int, [_vp, C.c_int]),
        "se_plan_create_ex": (C.c_int, [C.POINTER(_vp), C.POINTER(se_config), C.c_int]),
        "se_plan_path": (C.c_int, [_vp]),
        "se_choose_params": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                       _ip, _ip, _dp]),
        "se_error_estimate": (C.c_double, [C.c_int, C.c_double, C.c_double, C.c_double,
                                           C.c_int]),
        "se_real_space": (C.c_int, [_vp, _vp, C.c_int, C.c_double, C.c_double, C.c_int,
                                    C.c_double, _vp, _vp, _vp]),
        "se_self_term": (C.c_int, [_vp, C.c_int, C.c_double, _vp, _vp]),
        "se_batch_set_graph": (C.c_int, [_vp, C.c_int]),
        "se_solve_system": (C.c_int, [_vp, C.POINTER(se_system), _vp, _vp, _vp, _vp, _vp]),
        "se_server_request_bytes": (C.c_size_t, [C.POINTER(se_system), C.c_int]),
        "se_server_create": (C.c_int, [C.POINTER(_vp), C.POINTER(se_server_config)]),
        "se_server_reserve": (C.c_int, [_vp, C.POINTER(se_system), C.c_int]),
        "se_server_submit": (C.c_int, [_vp, C.POINTER(se_request), C.POINTER(C.c_longlong)]),
        "se_server_poll": (C.c_int, [_vp, C.POINTER(se_completion), C.c_int,
                                     C.POINTER(C.c_int)]),
        "se_server_drain": (C.c_int, [_vp, C.c_double]),
        "se_server_get_stats": (C.c_int, [_vp, C.POINTER(se_server_stats)]),
        "se_server_destroy": (C.c_int, [_vp]),
        # legacy helpers with return values
        "SE_gettime": (C.c_double, []),
        "SE_prod3": (C.c_int, [C.POINTER(C.c_int * 3)]),
        "calc_energy": (C.c_double, [SE_state, C.c_int]),
        "SE_init_params": (C.c_double, [_ip, _ip, _dp, C.c_double, C.c_double, C.c_double,
                                        _vp, C.c_int]),
        "SE_FGG_allocate_grid": (_dp, [C.POINTER(SE_FGG_params)]),
        "SE_FGG_allocate_vec": (_dp, [C.c_int]),
        "se_gpu_last_error": (C.c_int, []),
        "se_gpu_last_error_string": (C.c_char_p, []),
        "half": (C.c_int, [C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(code: int, what: str = "") -> None:
    if code != SE_OK:
        detail = lib().se_gpu_error_detail()
        raise SEError(f"{what}: {_ERR_NAMES.get(code, code)}"
                      + (f" ({detail.decode()})" if detail else ""))


def legacy_check(what: str) -> None:
    """Raise if the last legacy (void) call on this thread failed."""
    code = lib().se_gpu_last_error()
    if code:
        raise SEError(f"{what}: {lib().se_gpu_last_error_string().decode()}")

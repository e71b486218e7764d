"""The C ABI of libse_gpu.so without a GPU: the library loads, exports every
function its headers declare, and its host-only functions (parameter
packing, parse_params, SE_init_params, k_vec, ...) agree with the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = ["se_fgg_gpu.h", "se_gpu.h", "fftw3.h"]


def declared_functions(header):
    """Names of the functions a header declares (the first identifier
    followed by '(' in each declaration statement)."""
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    text = "\n".join(ln for ln in text.splitlines() if not ln.strip().startswith("#"))
    text = re.sub(r"typedef\s+struct\s*\w*\s*\{.*?\}\s*\w+\s*;", " ", text, flags=re.S)
    text = re.sub(r"typedef[^;]*;", " ", text)
    text = re.sub(r"enum\s*\{.*?\}\s*;", " ", text, flags=re.S)
    text = text.replace('extern "C" {', " ").replace("}", " ")
    names = set()
    for stmt in text.split(";"):
        m = re.search(r"([A-Za-z_]\w*)\s*\(", stmt)
        if m:
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def L():
    from se_fast_gridding_b200 import _lib
    return _lib.lib()


def test_headers_parse():
    names = declared_functions("se_fgg_gpu.h")
    for must in ("SE_FGG_grid_split_AVX_dispatch", "SE_FGG_int_split_force", "scaling",
                 "product_rc", "SE_FGG_wrap_fcn", "SE2P_FGG_extend_fcn", "calc_energy"):
        assert must in names
    assert "se_solve" in declared_functions("se_gpu.h")
    assert "fftw_plan_dft_3d" in declared_functions("fftw3.h")


@pytest.mark.parametrize("header", HEADERS)
def test_every_declared_symbol_is_exported(L, header):
    missing = [n for n in declared_functions(header) if not hasattr(L, n)]
    assert not missing, missing


def test_params_match_oracle(L, oracle_mod):
    from se_fast_gridding_b200 import fgg
    O = oracle_mod
    for M, P, Lb, xi in ((32, 21, 1.0, 8.0), (128, 16, 1.0, 20.0), (108, 12, 3.1814, 8.0)):
        m = 0.94 * np.sqrt(O.PI * P)
        opt, p = fgg.fcn_params(M, P, Lb, xi, m, 77)
        s = O.Setup(M=M, P=P, L=Lb, xi=xi, m=m, N=77)
        oo, po = s.opt(), s.params()
        for f in ("h", "c", "w", "eta", "xi"):
            assert getattr(opt, f) == getattr(oo, f), f
        for f in ("N", "P", "P_half", "c", "d", "h", "a"):
            assert getattr(p, f) == getattr(po, f), f
        assert list(p.dims) == list(po.dims) and list(p.npdims) == list(po.npdims)
        # se_config_derive gives the same numbers
        from se_fast_gridding_b200 import solver
        d = solver.derive(M, P, Lb, xi, m)
        assert (d.h, d.c, d.eta, d.d) == (p.h, p.c, opt.eta, p.d)


def test_pack_params(L):
    from se_fast_gridding_b200 import fgg
    p = fgg.pack_params(10, 8, 9, 10, 7, 123.0, 0.1)
    assert (p.N, p.P, p.P_half, list(p.dims), list(p.npdims)) == (10, 7, 3, [8, 9, 10], [15, 16, 17])
    assert p.a == -1 and p.b == -1 and p.d == (123.0 / 3.14159265358979323846) ** 1.5
    p2 = fgg.pack_params(10, 8, 8, 8, 8, 50.0, 0.125, a=-0.6)
    assert p2.a == -0.6 and p2.P_half == 4


def test_init_params_and_kvec(L, oracle_mod):
    O = oracle_mod
    q = np.linspace(-1, 1, 10)
    for P in (8, 12, 16, 21):
        M, P_, m = C.c_int(), C.c_int(P), C.c_double()
        Q = L.SE_init_params(C.byref(M), C.byref(P_), C.byref(m), 1.0, 3.1814, 8.0,
                             C.c_void_p(q.ctypes.data), 10)
        Mo, mo = O.init_params(P, 3.1814, 8.0, q)
        assert (M.value, m.value) == (Mo, mo)
        assert Q == pytest.approx(np.sum(q * q), rel=1e-15)
    for M in (8, 9, 108):
        box = (C.c_double * 3)(1.0, 2.0, 3.0)
        ks = [np.zeros(M) for _ in range(3)]
        L.k_vec(M, box, *[k.ctypes.data_as(C.POINTER(C.c_double)) for k in ks])
        ko = [np.zeros(M) for _ in range(3)]
        O.lib().orc_k_vec(M, np.array([1.0, 2.0, 3.0]).ctypes.data_as(C.POINTER(C.c_double)),
                          *[k.ctypes.data_as(C.POINTER(C.c_double)) for k in ko])
        for a, b in zip(ks, ko):
            np.testing.assert_array_equal(a, b)


def test_small_helpers(L):
    assert [L.half(p) for p in (7, 8, 21, 16)] == [3, 4, 10, 8]
    assert L.is_odd(7) == 1 and L.is_odd(8) == 0 and L.isnot_div_by_4(6) == 2
    v = (C.c_int * 3)(3, 4, 5)
    assert L.SE_prod3(C.byref(v)) == 60
    assert L.SE_gettime() > 1e9


def test_device_bytes_without_gpu(L):
    from se_fast_gridding_b200 import _lib
    cfg = _lib.se_config(M=128, P=16, L=1.0, xi=20.0, m=6.66, mode=1, precision=1,
                         max_particles=100_000)
    b = L.se_plan_device_bytes(C.byref(cfg))
    assert 128 ** 3 * 8 < b < 200 * 2 ** 20


def test_default_path_without_gpu(L):
    """Tile-aligned kernels for M a multiple of 16 (>= 32) and P <= 16, the
    pair interpolation from P = 8 on."""
    assert L.se_default_path(128, 16) == 3
    assert L.se_default_path(64, 6) == 1
    assert L.se_default_path(24, 8) == 0
    assert L.se_default_path(128, 21) == 0


def test_path_constants_match_the_header():
    """The SE_PATH_* bits the Python layer passes are the header's."""
    import re
    from se_fast_gridding_b200 import _lib
    hdr = open(os.path.join(ROOT, "include", "se_gpu.h")).read()
    defs = dict(re.findall(r"#define (SE_PATH_\w+) \(?(-?\d+)\)?", hdr))
    for name, value in defs.items():
        assert getattr(_lib, name) == int(value), name
    assert {"SE_PATH_TILE_SPREAD", "SE_PATH_PAIR_INTERP", "SE_PATH_RUNTIME_P",
            "SE_PATH_RADIX_SORT", "SE_PATH_FFT3", "SE_PATH_BIN_WINDOWS"} <= set(defs)

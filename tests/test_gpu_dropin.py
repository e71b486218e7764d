"""The reference's own driver, unchanged, running on libse_gpu.so.

oracle/Makefile links SE_fast_gridding's spectral_ewald.c + test_accuracy.c +
SE_direct.c (unchanged sources) against libse_gpu.so, which supplies SE_fgg.c,
SE_general.c and FFTW; the same sources are also linked against the CPU
reference (SE_fgg.c, SE_general.c and a CPU FFT).  Both binaries are build
products under oracle/_ref/ (they travel with the repository snapshot).  The
error each prints (SE vs the direct Ewald sum, test_accuracy.c:71,91) must
agree.  spectral_ewald() alone, unchanged and built on libse_gpu.so, must
also return the reference's own arrays: phi / force of atoms.txt (N = 100,
every P of test_accuracy) and of the 100,000-particle FORCE system, whose
wall time per call the last test prints.
"""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


def run(binary, N, P):
    path = os.path.join(REF, binary)
    if not os.path.exists(path):
        pytest.skip(f"{binary} not built (make -C oracle ref drop-in)")
    r = subprocess.run([path, str(N), str(P)], cwd=REF, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    m = re.search(r"error in (potential|force): ([0-9.eE+-]+)", r.stdout)
    assert m, r.stdout
    return float(m.group(2)), r.stdout


@pytest.mark.parametrize("mode", ["pot", "force"])
@pytest.mark.parametrize("P", [8, 12, 16, 21])
def test_test_accuracy_drop_in(mode, P):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    e_cpu, _ = run(f"test_accuracy_cpu_{mode}", 10, P)
    e_gpu, out = run(f"test_accuracy_gpu_{mode}", 10, P)
    assert "[se_gpu]" not in out
    assert abs(e_gpu - e_cpu) <= 1e-4 * e_cpu + 1e-15, (e_gpu, e_cpu)


def dropin(kind):
    """spectral_ewald() of the reference, unchanged, built as a shared library
    on libse_gpu.so (oracle/Makefile target drop-in)."""
    import ctypes as C
    path = os.path.join(REF, f"libse_dropin_{kind}.so")
    if not os.path.exists(path):
        pytest.skip(f"libse_dropin_{kind}.so not built (make -C oracle drop-in)")
    return C.CDLL(path)


@pytest.mark.parametrize("mode", ["pot", "force"])
@pytest.mark.parametrize("P", [8, 12, 16, 21])
def test_dropin_arrays_equal_reference(mode, P):
    """The arrays the unchanged spectral_ewald() returns on the GPU equal the
    ones the reference's own build returns (atoms.txt, N = 100, L = 3.1814,
    xi = 8; tests/golden/test_accuracy.npz) within 1e-12 relative RMS."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import oracle as O
    from conftest import load_golden
    g = load_golden("test_accuracy.npz")
    N = 100
    x, q = g[f"N{N}/x"], g[f"N{N}/q"]
    M, m = int(g[f"N{N}/P{P}/M"]), float(g[f"N{N}/P{P}/m"])
    w = 3 if mode == "force" else 1
    out = O.ref_spectral_ewald(dropin(mode), x, q, M, P, m, 3.1814, 8.0, w * N)
    ref = g[f"N{N}/P{P}/" + ("force" if mode == "force" else "phi")]
    assert O.rel_rms(out, ref) < 1e-12, O.rel_rms(out, ref)


def test_dropin_c2_force_and_time(capsys):
    """The unchanged spectral_ewald() on the headline FORCE system (N = 1e5,
    M = 128, P = 16, xi = 20), host buffers as the driver has them: within
    1e-12 of the reference's own result on the 1,000-particle subset and its
    checksums; the wall time per call is printed (the drop-in's speed)."""
    import time
    import numpy as np
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import oracle as O
    from conftest import check_digest, load_golden
    g = load_golden("c2.npz")
    N = 100_000
    x, q = O.synthetic_system(N, 1.0, seed=1, charges="uniform")
    lib = dropin("force")
    m = O.c1_params(16)
    f = O.ref_spectral_ewald(lib, x, q, 128, 16, m, 1.0, 20.0, 3 * N)   # first call: set-up
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        f = O.ref_spectral_ewald(lib, x, q, 128, 16, m, 1.0, 20.0, 3 * N)
        times.append(time.perf_counter() - t0)
    t = g["targets"]
    sub = np.concatenate([f[t + d * N] for d in range(3)])
    assert O.rel_rms(sub, g["force_ref"]) < 1e-12, O.rel_rms(sub, g["force_ref"])
    check_digest(g, "force_ref_all", f, 1e-11)
    with capsys.disabled():
        print(f"\n[drop-in] spectral_ewald() FORCE N=1e5 M=128 P=16 on libse_gpu.so: "
              f"{1e3 * min(times):.1f} ms per call (best of 3; "
              f"{1e3 * float(np.median(times)):.1f} ms median)")

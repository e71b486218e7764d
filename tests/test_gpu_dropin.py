"""The reference's own driver, unchanged, running on libse_gpu.so.

oracle/Makefile links SE_fast_gridding's spectral_ewald.c + test_accuracy.c +
SE_direct.c (unchanged sources) against libse_gpu.so, which supplies SE_fgg.c,
SE_general.c and FFTW; the same sources are also linked against the CPU
reference (SE_fgg.c, SE_general.c and a CPU FFT).  Both binaries are build
products under oracle/_ref/ (they travel with the repository snapshot).  The
error each prints (SE vs the direct Ewald sum, test_accuracy.c:71,91) must
agree.
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

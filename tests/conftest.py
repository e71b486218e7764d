import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name} not generated")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def check_digest(g, prefix, a, rtol):
    """Compare an array with a golden digest (checksums + seeded sample) or a
    full golden array."""
    a = np.asarray(a, dtype=np.float64).ravel()
    if prefix in g:
        ref = g[prefix].ravel()
        scale = np.abs(ref).max() or 1.0
        np.testing.assert_allclose(a, ref, rtol=0, atol=rtol * scale, err_msg=prefix)
        return
    assert a.size == int(g[prefix + "__size"]), prefix
    l1 = float(g[prefix + "__l1"])
    scale = l1 / a.size if a.size else 1.0
    sidx = g[prefix + "__sidx"]
    np.testing.assert_allclose(a[sidx], g[prefix + "__sval"], rtol=0,
                               atol=rtol * max(np.abs(g[prefix + "__sval"]).max(), scale),
                               err_msg=prefix + " sample")
    assert abs(a.sum() - float(g[prefix + "__sum"])) <= rtol * l1 + 1e-300, prefix + " sum"
    assert abs(np.abs(a).sum() - l1) <= rtol * l1 + 1e-300, prefix + " l1"
    rng = np.random.Generator(np.random.Philox(7))
    rng.choice(a.size, size=min(256, a.size), replace=False)
    w = rng.uniform(-1, 1, size=a.size)
    assert abs((w * a).sum() - float(g[prefix + "__wsum"])) <= rtol * l1 + 1e-300, prefix + " wsum"


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as O
    O.lib()
    return O

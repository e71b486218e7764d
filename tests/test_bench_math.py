"""The roofline arithmetic of bench.py on CPU: the algorithmic bytes and
flops per launch of the C2 spread and interpolation, the choice of the
dominant kernel, and achieved / peak."""
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


C2 = [(100_000, 128, 16, "force")]


def test_kernel_work_c2(bench):
    b, f = bench.kernel_work("spread", C2, "fp32")
    assert b == 100_000 * 32 + 128 ** 3 * 8            # x, q in; the FP64 grid out
    assert f == 2.0 * 16 ** 3 * 100_000                 # one FMA per stencil point
    b, f = bench.kernel_work("interp", C2, "fp32")
    assert b == 128 ** 3 * 4 + 100_000 * 32 + 100_000 * 8 * 3   # FP32 grid copy, records, forces
    assert f == 4.0 * 16 ** 3 * 100_000                 # value and z-derivative sums
    b64, _ = bench.kernel_work("interp", C2, "fp64")
    assert b64 == b + 128 ** 3 * 4                      # the FP64 grid itself
    _, fpot = bench.kernel_work("interp", [(100_000, 128, 16, "potential")], "fp32")
    assert fpot == 2.0 * 16 ** 3 * 100_000


def test_roofline_picks_the_longer_stage(bench, monkeypatch):
    monkeypatch.setattr(bench, "_FMA_PEAK", 69.0)
    stages = {"sort": 0.04, "spread": 0.136, "kspace": 0.068, "interp": 0.138}
    hbm, fma = bench.roofline_of(stages, C2, "fp32", lambda k: "k_" + k,
                                 traffic={"spread": 1, "interp": 2})
    assert hbm["kernel"] == fma["kernel"] == "k_interp"
    b, f = bench.kernel_work("interp", C2, "fp32")
    t = 0.138e-3
    assert hbm["achieved"] == pytest.approx(b / t / 1e9)
    assert hbm["frac"] == pytest.approx(hbm["achieved"] / hbm["peak"])
    assert hbm["traffic"] == 2
    assert fma["achieved"] == pytest.approx(f / t / 1e12)
    assert fma["frac"] == pytest.approx(fma["achieved"] / 69.0)
    peaks = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks):
        with open(peaks) as fh:
            assert hbm["peak"] == pytest.approx(float(json.load(fh)["hbm_gbs"]))
    stages["spread"] = 0.2
    hbm, _ = bench.roofline_of(stages, C2, "fp32", lambda k: k)
    assert hbm["kernel"] == "spread" and hbm["traffic"] is None

"""The bench line's roofline arithmetic (CPU): algorithmic bytes per
gate-eval are the 2-bit code and the 1-bit mark of every (net, pair) written
once plus the primary inputs' codes read, and the limiter is named from the
numbers the line carries."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _Net:
    def __init__(self, g, pi):
        self.n_gates, self.n_pi = g, pi


def test_algorithmic_bytes(bench):
    # 0.375 B per gate-eval plus 0.25 B per primary input and pair
    assert bench.alg_bytes(_Net(20_000, 1_500), 32_768) == pytest.approx(0.375 * 20_000 * 32_768 + 0.25 * 1_500 * 32_768)
    assert bench.alg_bytes(_Net(1_000_000, 8_192), 1) / 1_000_000 == pytest.approx(0.377048)


def test_roofline_fraction_and_limiter(bench, monkeypatch):
    monkeypatch.setattr(bench, "measured_peaks", lambda: {"hbm_gbs": 1000.0, "source": "measured"})
    # 1 GB in 2 ms = 500 GB/s = half of the peak; 1e9 warp instructions in
    # 2 ms on 10 SMs at 1,000 MHz fill 1e9 / (10 * 4 * 1e9 * 2e-3) = 12.5x
    # the slots: issue-bound
    prof = {"dram_bytes_per_launch": 1e8, "scale": 2.0, "warp_inst_per_launch": 1e9, "source": "test"}
    r = bench.roofline(1e9, 2.0, "k", prof, 1e9, 10, 1000.0)
    assert r["achieved"] == pytest.approx(500.0) and r["frac"] == pytest.approx(0.5)
    assert r["traffic"] == pytest.approx(2e8)
    assert r["limiter"] == "issue"
    r = bench.roofline(1e9, 2.0, "k", dict(prof, warp_inst_per_launch=1e7), 1e9, 10, 1000.0)
    assert r["limiter"] == "latency"
    r = bench.roofline(1.9e9, 2.0, "k", None, 1e9, 10, 1000.0)
    assert r["frac"] == pytest.approx(0.95) and r["limiter"] == "hbm"

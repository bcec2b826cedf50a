"""bench.py's host-side pieces on the CPU: the clock sampler's reading of nvidia-smi rows (only
the bench GPU's rows count, throttle reasons are collected), and the ncu traffic lookup from the
committed profile summary."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_clock_sampler_summary_filters_by_gpu_and_collects_reasons(tmp_path):
    s = bench.ClockSampler("GPU-aaa")
    s.path = str(tmp_path / "clocks.csv")
    rows = [
        "0, GPU-aaa, 1965, 1965, 500.1, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, GPU-aaa, 1900, 1965, 650.0, 0x4, Not Active, Not Active, Not Active, Active",
        "1, GPU-bbb, 800, 1965, 100.0, 0x8, Active, Not Active, Not Active, Not Active",
        "0, GPU-aaa, 1965, 1965, 640.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    open(s.path, "w").write("\n".join(rows) + "\n")
    s.proc = object()  # as if nvidia-smi had run
    out = s.summary()
    assert out["samples"] == 3
    assert out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]  # hw_slowdown belongs to the other GPU
    assert out["power_w_max"] == 650.0


def test_clock_sampler_without_nvidia_smi():
    s = bench.ClockSampler(None)
    s.proc = None
    assert s.summary()["reasons"] == ["nvidia-smi unavailable"]


def test_traffic_comes_from_the_committed_profile():
    for k in ("k_sweep_x", "k_sweep_y", "k_sweep_z"):
        v, src = bench.ncu_traffic(k)
        assert src == "profiles/k_sweep_400cube_2sub.md"
        # read + write of one launch: close to the 1.024 GB of algorithmic bytes
        assert 0.9e9 < v < 1.1e9
    assert bench.ncu_traffic("k_not_profiled") == (None, None)

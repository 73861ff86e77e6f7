"""Host helpers of bench.py (CPU): the nvidia-smi clock record and the whole-job rate."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
import bench  # noqa: E402

ROWS = """0, 1965, 1965, 812.5, 0x0000000000000004, Not Active, Not Active, Not Active, Active
0, 1702, 1965, 998.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active
0, 1507, 1965, 1001.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active
garbage line
0, [N/A], 1965, 1.0, 0x0, Not Active, Not Active, Not Active, Not Active
"""


def test_clock_record_median_and_reasons():
    c = bench.parse_clocks(ROWS)
    assert c["samples"] == 3 and c["sm_mhz"] == 1702.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"]
    hot = ROWS.replace("Not Active, Not Active, Not Active, Active", "Active, Not Active, Active, Not Active", 1)
    assert bench.parse_clocks(hot)["reasons"] == ["hw_slowdown", "sw_power_cap", "sw_thermal_slowdown"]
    assert bench.parse_clocks("")["reasons"] == ["unavailable"]


def test_clock_sampler_without_a_gpu_leaves_no_file(monkeypatch):
    monkeypatch.setenv("PATH", "/nonexistent")  # nvidia-smi cannot start
    with bench.ClockSampler(0) as clk:
        path = clk.f.name
        assert os.path.exists(path)
    assert not os.path.exists(path)
    assert clk.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}


def test_whole_job_rate():
    # updates of every rank over the slowest rank's time for the given steps
    assert np.isclose(bench.whole_job_rate(4.0e10, 3, 6000.0), 4.0e10 * 3 / 6.0)


def test_clock_sampler_reads_a_running_sampler(tmp_path, monkeypatch):
    """The sampling path as on a GPU box: a stand-in nvidia-smi that prints a
    CSV row every 20 ms until it is terminated."""
    import time
    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!/bin/sh\nwhile true; do echo '0, 1800, 1965, 900.0, 0x4, Not Active, Not Active, "
                    "Not Active, Active'; sleep 0.02; done\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}:{os.environ.get('PATH', '')}")
    with bench.ClockSampler(0) as clk:
        path = clk.f.name
        time.sleep(0.3)
    c = clk.summary()
    assert c["samples"] >= 3 and c["sm_mhz"] == 1800.0 and c["reasons"] == ["sw_power_cap"]
    assert not os.path.exists(path)


def test_sample_parity_compares_only_the_sampled_rays():
    """The bench's parity record: TL-line differences of the sampled rays, in
    their ragged layout, and nothing of the other rays."""
    from types import SimpleNamespace
    rays = np.zeros(3, dtype=[("line_off", "i8"), ("nvr", "i4")])
    rays["line_off"] = [0, 4, 9]
    rays["nvr"] = [4, 5, 2]
    batch = SimpleNamespace(rays=rays)
    tll = np.arange(11, dtype=np.float64)
    ref = {"tll": tll.copy()}
    ref["tll"][5] += 0.002  # ray 1
    ref["tll"][10] += 5.0   # ray 2: not sampled
    p = bench.sample_parity(batch, np.array([0, 1]), ref, tll)
    assert p["rays"] == 2 and p["outputs"] == 9
    assert abs(p["max_db"] - 0.002) < 1e-12
    assert abs(p["rms_db"] - np.sqrt(0.002 ** 2 / 9)) < 1e-12

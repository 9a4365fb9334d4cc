"""bench.py's one-line JSON contract, checked without a GPU.

The reference arm (`--impl reference`) runs the reference's own CPU path
(zgrid_cpu + malley_cpu, compiled into oracle/_ref) on the host cores: it
must print exactly one JSON line with the metric, unit, step counts and the
reference-arm fields (impl, cpu_baseline, e2e without copies).  The helpers
that turn profile figures into roofline fractions are checked on their own.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
from oracle_lib import Reference  # noqa: E402
import bench  # noqa: E402

KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "e2e", "cpu_baseline")


@pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built")
def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--cpu-sample-every", "64"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [line for line in r.stdout.splitlines() if line.strip()]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    for k in KEYS:
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "rays/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    assert d["e2e"] == {"value": d["value"], "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]


def test_issue_roofline_arithmetic():
    d = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    for shape in (0, 7, 5):
        got = bench.issue_roofline(10.0, 1_000_000, 2000.0, 100, shape=shape)
        ipr = d.get("warp_inst_per_ray_by_shape", {}).get(str(shape), d["k_form_factors_warp_inst_per_ray"])
        assert got["warp_inst_per_ray"] == ipr
    got = bench.issue_roofline(10.0, 1_000_000, 2000.0, 100)
    ipr = d.get("warp_inst_per_ray_by_shape", {}).get("0", d["k_form_factors_warp_inst_per_ray"])
    achieved = ipr * 1_000_000 / 10e-3
    peak = 4 * 100 * 2000e6
    assert got["frac"] == pytest.approx(achieved / peak)
    assert got["achieved"] == pytest.approx(achieved / 1e9) and got["peak"] == pytest.approx(peak / 1e9)
    assert bench.issue_roofline(10.0, 1_000_000, None, 100) is None  # no clock sample: no figure


def test_hbm_peak_names_its_source():
    gbs, source = bench.hbm_peak()
    assert gbs > 0 and source in ("measured", "fallback")
    assert source == ("measured" if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else "fallback")


def test_clock_sampler_with_a_fake_nvml():
    """The timed region's clock record from NVML (read-only queries): the
    sampler polls every 2 ms, takes the median of the loaded samples, and
    names the clock-event reasons from their bits."""
    import time

    class FakeNvml:
        NVML_CLOCK_SM = 1
        calls = 0

        def nvmlDeviceGetClockInfo(self, h, kind):
            FakeNvml.calls += 1
            return 1965 if FakeNvml.calls % 4 else 1800

        def nvmlDeviceGetMaxClockInfo(self, h, kind):
            return 1965

        def nvmlDeviceGetCurrentClocksEventReasons(self, h):
            return 0x4 if FakeNvml.calls > 6 else 0x0  # sw_power_cap from the seventh sample on

    clk = bench.Clocks(0)
    clk._nvml_handle = lambda: (FakeNvml(), object())
    clk.start()
    assert clk.thread is not None
    time.sleep(0.06)
    rec = clk.stop()
    assert rec["samples"] >= 10
    assert rec["sm_mhz"] == 1965.0 and rec["sm_max_mhz"] == 1965.0 and rec["sm_min_mhz"] == 1800.0
    assert rec["reasons"] == ["sw_power_cap"]
    assert rec["source"].startswith("nvml")

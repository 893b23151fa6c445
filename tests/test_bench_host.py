"""Host-side pieces of bench.py that need no GPU: the clock-record summary
that decides whether a timed run saw throttling, and the workload arithmetic."""

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


def _line(sm, smax=1965, power=700.0, active="0x0", hw="Not Active", hwt="Not Active",
          swt="Not Active", cap="Not Active"):
    return "0, %s, %s, %s, %s, %s, %s, %s, %s\n" % (sm, smax, power, active, hw, hwt, swt, cap)


def test_clock_summary_median_under_load_and_no_reason(bench):
    lines = [_line(345)] + [_line(1965)] * 5 + [_line(1950)] * 2
    s = bench.clock_summary(lines)
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == [] and s["samples"] == 8


def test_clock_summary_reports_throttle_reasons(bench):
    lines = [_line(1965)] * 3 + [_line(1300, cap="Active")] + [_line(1100, hwt="Active")]
    s = bench.clock_summary(lines)
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert s["sm_mhz"] == 1965.0


def test_clock_summary_skips_unavailable_fields(bench):
    lines = [_line("[N/A]", "[N/A]")] + [_line(1900)] * 3 + ["garbage\n"]
    s = bench.clock_summary(lines)
    assert s["sm_mhz"] == 1900.0 and s["samples"] == 4
    assert bench.clock_summary([_line("[N/A]", "[N/A]")])["reasons"] == ["no samples"]
    assert bench.clock_summary([])["sm_mhz"] is None


def test_entries_per_step(bench):
    # (N_train^2 + N_test * N_train) kernel entries per sigma
    assert bench.entries_per_step(32768, 8192, 3) == (32768 ** 2 + 8192 * 32768) * 3


def test_clock_sampler_end_to_end_with_a_stand_in_nvidia_smi(bench, tmp_path, monkeypatch):
    """start()/stop() around a stand-in `nvidia-smi` that prints one sample
    per 20 ms: the samples are read back and summarised."""
    import time
    exe = tmp_path / "nvidia-smi"
    exe.write_text("#!/bin/sh\nwhile true; do echo '%s'; sleep 0.02; done\n"
                   % _line(1965, cap="Active").strip())
    exe.chmod(0o755)
    monkeypatch.setenv("PATH", str(tmp_path) + os.pathsep + os.environ["PATH"])
    cs = bench.ClockSampler(0)
    cs.start()
    time.sleep(0.3)
    s = cs.stop()
    assert s["sm_mhz"] == 1965.0 and s["reasons"] == ["sw_power_cap"] and s["samples"] >= 2


def test_reference_arm_reports_our_arms_config(bench, monkeypatch):
    """`bench.py --impl reference` (CPU only) prints one JSON line on the same
    config, metric, unit and direction as our arm at its defaults, with its
    bounded sample stated in cpu_baseline and no host<->device bytes."""
    import json
    import subprocess
    import sys
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0", "--cpu-ntrain", "256",
                          "--cpu-ntest", "64"], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, OMP_NUM_THREADS="2", OPENBLAS_NUM_THREADS="2"))
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()  # our arm's defaults
    ours = bench.headline_config(a, [float(s) for s in a.sigmas.split(",")], 1)
    assert line["impl"] == "reference"
    assert line["config"] == ours and ours["n_train"] == 32768 and ours["n_test"] == 8192
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is True
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port"
    assert "N_train=256" in line["cpu_baseline"]["sample"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0

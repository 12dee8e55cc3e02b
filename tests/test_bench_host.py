"""Host-side parts of the bench on the CPU: the clock sampler against a fake NVML, the peak
lookup, and the reference arm under a multi-rank launch (only rank 0 works and prints)."""
import importlib
import json
import os
import subprocess
import sys
import time
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    return importlib.import_module("bench")


def fake_nvml(clock=1860, reasons=0x1 | 0x4):
    m = types.ModuleType("pynvml")
    m.NVML_CLOCK_SM = 1
    m.nvmlInit = lambda: None
    m.nvmlDeviceGetHandleByIndex = lambda i: ("gpu", i)
    m.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    m.nvmlDeviceGetClockInfo = lambda h, kind: clock
    m.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reasons
    return m


def test_clock_sampler_with_fake_nvml(monkeypatch):
    bench = load_bench()
    monkeypatch.setitem(sys.modules, "pynvml", fake_nvml(1860, 0x1 | 0x4 | 0x40))
    with bench.ClockSampler(0) as clk:
        time.sleep(0.05)
    s = clk.summary()
    assert s["sm_mhz"] == 1860 and s["sm_max_mhz"] == 1965 and s["samples"] > 0
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]      # gpu_idle is not reported


def test_clock_sampler_without_nvml(monkeypatch):
    bench = load_bench()
    broken = types.ModuleType("pynvml")

    def fail():
        raise RuntimeError("no driver")

    broken.nvmlInit = fail
    monkeypatch.setitem(sys.modules, "pynvml", broken)
    with bench.ClockSampler(0) as clk:
        pass
    assert clk.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def test_measured_peak_reads_the_file_or_falls_back(monkeypatch, tmp_path):
    bench = load_bench()
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.measured_peak() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6546.9, "bf16_tflops": 1590}))
    assert bench.measured_peak() == (6546.9, "measured")


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "1", "--workload", "plain_64m",
                        "--cpu-sample-bytes", str(1 << 20)], capture_output=True, text=True, cwd=ROOT, env=env,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_help_lists_every_option():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                       cwd=ROOT, timeout=120)
    assert r.returncode == 0, r.stderr
    for opt in ("--gpus", "--steps", "--warmup", "--impl", "--form", "--approach", "--workload"):
        assert opt in r.stdout, opt


def test_map_headroom_defaults(monkeypatch):
    """The MD5 series sizes its digest map for all 20 checkpoints at the baseline (about 0.3 N new
    entries per checkpoint), so no rehash falls in its timed steps; other workloads keep the
    library's default; an explicit value wins."""
    bench = load_bench()
    monkeypatch.setattr(sys, "argv", ["bench.py", "--workload", "md5_f32_8g"])
    a = bench.parse()
    assert (a.map_headroom, a.chunk_size, a.nbytes) == (400, 256, 8 << 30)
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    assert bench.parse().map_headroom == 0
    monkeypatch.setattr(sys, "argv", ["bench.py", "--workload", "md5_f32_8g", "--map-headroom", "250"])
    assert bench.parse().map_headroom == 250

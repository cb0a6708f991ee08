"""bench.py's output: one JSON line per run with the keys, types and relations the benchmark
reports, for the reference arm (on the CPU) and for this library's arm (on a B200), on short
runs."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COMMON = {"metric": str, "value": float, "unit": str, "n_gpus": int, "steps": int, "warmup": int,
          "ms_per_step": float, "higher_is_better": bool, "scaling": str, "dtype": str, "data": str,
          "config": dict}


def _line(args, timeout):
    r = subprocess.run([sys.executable, "bench.py", *args], cwd=ROOT, capture_output=True, text=True,
                       timeout=timeout)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    for k, t in COMMON.items():
        assert isinstance(d[k], (int, float) if t is float else t), (k, d.get(k))
    assert d["value"] > 0 and d["higher_is_better"] is True and "vs_baseline" in d
    assert d["config"]["workload"].startswith("wave_breaker_991440")
    return d


def _our_config(args):
    """The config our arm prints for the same arguments (built without a GPU)."""
    sys.path.insert(0, ROOT)
    import bench
    old = sys.argv
    try:
        sys.argv = ["bench.py", *args]
        a = bench.parse()
    finally:
        sys.argv = old
    return bench.line_config(a, 1)


def test_reference_arm_line():
    args = ["--impl", "reference", "--steps", "1", "--warmup", "1"]
    d = _line(args, 900)
    assert d["impl"] == "reference"
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # The same config dict as our arm's line for the same workload, naming the CPU sample.
    assert d["config"] == _our_config(args) and "sub-scene" in d["config"]["reference_arm"]
    assert d["iterations_mean"] >= 1 and d["particle_iterations_per_s"] == d["value"] * d["iterations_mean"]
    port = d["port_same_iteration_rule"]
    assert port["kind"] == "port" and port["iterations_mean"] >= 3


@pytest.mark.gpu
def test_library_arm_line():
    d = _line(["--steps", "3", "--warmup", "3", "--train-steps", "5", "--long-steps", "0", "--same-steps", "20"],
              1200)
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3 and d["dtype"] == "f32"
    r = d["roofline"]
    assert r["bound"] in ("hbm", "tensor") and r["unit"] in ("GB/s", "TFLOP/s")
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-3 and r["traffic"] > 0
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    # The end-to-end arm replays the timed steps from their start state and arrives at the
    # same bits as the timed steps.
    assert e["replay_bit_identical"] is True
    assert d["gpu_launches"] > 0
    c = d["clocks"]
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(c) and c["samples"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["value"] > 0
    passes = r["passes"]
    assert {"pci_loop", "neighbors", "nonpressure", "grid_keys", "grid_scan", "grid_scatter",
            "grid_gather"} <= set(passes)
    for v in passes.values():
        assert v["ms_per_step"] > 0 and (v["frac"] is None or 0 < v["frac"] < 2)
    assert d["config"] == _our_config(["--steps", "3", "--warmup", "3", "--train-steps", "5", "--long-steps", "0"])
    ss = d["same_state"]
    assert len(ss) == 2 and all(x["samples"] > 0 for x in ss)
    for x in ss:
        assert x["device_time_ratio"] > 0
        if x["plain"]["qualifying"] == 0:
            assert x["learned_vs_plain_same_state"] is None and not x["target_met"]


def test_same_state_ratio_counts_only_qualifying_steps():
    """learned_vs_plain_same_state is the metric's ratio (steps that met eta per device time),
    so a run where the plain steps never met eta has no ratio, however the times compare."""
    import bench
    assert bench.qualifying_ratio(20, 40.0, 20, 44.0) == pytest.approx(40.0 / 44.0)
    assert bench.qualifying_ratio(10, 40.0, 20, 40.0) == pytest.approx(2.0)
    assert bench.qualifying_ratio(0, 460.0, 0, 250.0) is None
    assert bench.qualifying_ratio(0, 460.0, 5, 250.0) is None
    assert bench.qualifying_ratio(20, 40.0, 0, 44.0) == 0.0

"""The benchmark's host side on CPU: the reference arm's JSON line (it times the
threaded CPU restatement of CAST's CPU kernels, so it runs without a GPU), its
rank handling under a multi-rank launch, and the roofline denominators and
traffic scaling read from committed files."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

REF_ARGS = ["--impl", "reference", "--n", "14", "--cpu-n", "12", "--depth", "4", "--steps", "2",
            "--warmup", "1", "--cpu-budget", "0.1"]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *REF_ARGS], env=env,
                          capture_output=True, text=True, timeout=300)


def test_reference_arm_line_keeps_the_contract():
    r = _run({})
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 1
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["metric"] == "HBM GB/s (fused-gate statevector passes)" and d["unit"] == "GB/s"
    assert d["config"]["workload"] == "brickwork-14q-d4-c128-k4"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert "12-qubit brickwork" in cb["sample"]
    assert cb["build"] in ("-O3 -march=native", "-O3 -march=x86-64-v3")
    assert d["e2e"] == {"value": d["value"], "unit": "GB/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    r = _run({"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_roofline_denominator_and_traffic_scaling():
    peak, kind = bench.measured_peak_hbm()
    assert peak > 0 and kind in ("measured", "fallback")
    with open(os.path.join(ROOT, "profiles", "gate_kernel_traffic.json")) as f:
        entry = json.load(f)["f64_k4"]
    t30 = bench.traffic_from_profile(30, "f64", 4)
    assert t30 == entry["dram_bytes_per_launch"] * (1 << (30 - entry["n_qubits"]))
    # within a few percent of the algorithmic 2 * 2^30 * 16 bytes: no re-reads
    assert 0.9 < t30 / (2 * (1 << 30) * 16) <= 1.05
    assert bench.traffic_from_profile(30, "f64", 9) is None

"""bench.py's one-line JSON contract: the keys, units and types a caller of the
benchmark reads, for the reference arm (CPU only) and for a small run of the
GPU arm."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, timeout=900):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                         capture_output=True, text=True, timeout=timeout)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.strip().splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    d = _run(["--impl", "reference", "--steps", "1", "--warmup", "1", "--cpu-sample", "16",
              "--workload", "gri_32k"])
    assert d["impl"] == "reference" and d["metric"] == "cells_per_sec" and d["unit"] == "cells/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"] == "gri_32k"


def test_reference_arm_default_workload_is_the_1m_cell_batch():
    """The default workload is the 1,048,576-cell GRI-Mech 3.0 configuration;
    the reference arm times a bounded stratified sample of it."""
    d = _run(["--impl", "reference", "--steps", "1", "--warmup", "0", "--cpu-sample", "8"])
    assert d["config"]["workload"] == "gri_1m" and d["config"]["ncells"] == 1048576
    assert d["config"]["sample_cells_per_step"] == 8


@pytest.mark.gpu
def test_gpu_arm_line():
    d = _run(["--steps", "1", "--warmup", "3", "--workload", "gri_32k", "--ncells", "2048", "--no-serving",
              "--no-fp64-step", "--cpu-sample", "64", "--accuracy-cells", "32"])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e",
              "clocks", "gpu_launches"):
        assert k in d, k
    assert d["metric"] == "cells_per_sec" and d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 3
    assert d["scaling"] == "weak" and d["vs_baseline"] is None and d["gpu_launches"] >= 1
    r = d["roofline"]
    assert r["bound"] == "fp64+fp32" and r["unit"] == "TFLOP/s"
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12 and 0 < r["frac"] < 1.5
    assert r["fp64"]["peak_tflops"] > 10 and r["fp32"]["peak_tflops"] > r["fp64"]["peak_tflops"]
    assert r["hbm"]["alg_bytes"] > 0
    a = d["accuracy"]
    assert a["cells"] == 32 and 0 <= a["gpu_vs_cpu_same_tol"]["Y_within_gate"] <= 1
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert "sm_mhz" in d["clocks"] and "reasons" in d["clocks"]
    assert d["cpu_baseline"]["value"] > 0 and d["failed_cells"] == 0
    assert d["cpu_baseline"]["serial"]["value"] > 0 and d["cpu_baseline"]["serial"]["cores"] == 1
    assert d["config"]["workload"] == "gri_32k" and d["config"]["cells_per_gpu"] == 2048

"""The reference arm of bench.py (the oracle's OpenMP restatement of the term
pipeline on the host cores) prints one JSON line with the benchmark's keys,
on the same workload config as the GPU arm.  Runs on the CPU in seconds."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--ref-step-s", "1"], capture_output=True, text=True, timeout=300,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    rt = line["cpu_baseline"]["reference_terms"]
    assert rt["value"] > 0 and "A2_cpu.cpp" in rt["terms"] and "C_cpu.cpp" in rt["terms"]
    sys.path.insert(0, ROOT)
    import bench

    class A:
        queries = 4096

    assert line["config"] == bench.arm_config(A, 1)

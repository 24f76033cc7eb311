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


def test_reference_arm_loads_no_product_library():
    """The CPU arms take alpha(x) from the oracle: the product library is never
    mapped into the reference arm's process."""
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1', "
            "'--ref-step-s', '0.5']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "assert 'libcudapix_b200' not in maps, 'product library loaded'; print('NOLIB')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "NOLIB" in r.stdout


def test_roofline_from_profiles_and_live_spans():
    """The roofline object: the dominant kernel by live CUDA-event time, ALU
    instructions of one launch from its committed ncu profile over the live
    duration, against 2 ALU warp instructions per SM per clock at the sampled
    clock; both committed profiles were taken of the current kernel sources."""
    sys.path.insert(0, ROOT)
    import bench

    class Ctx:
        def sm_count(self):
            return 148

    kern = [{"k_easy": 12.8, "k_hard_shared": 20.5, "k_p2": 2.4}] * 3
    roof, shares = bench.roofline(kern, [21.5] * 3, [1e11] * 3, [37.0] * 3, {"sm_mhz": 1965.0}, Ctx())
    assert roof["bound"] == "alu" and roof["kernel"].startswith("k_hard_shared")
    assert roof["other"]["kernel"].startswith("k_easy")
    for r in (roof, roof["other"]):
        assert r["profile_matches_source"] is True, r["profile"]
        assert 0.3 < r["frac"] < 1.0
        assert abs(r["peak"] - 2.0 * 148 * 1965e6 / 1e9) < 1e-6
    assert abs(shares["k_hard_shared"]["share"] - 20.5 / 37.0) < 1e-9

"""The benchmark's command-line contract, checked on the CPU.

`bench.py --impl reference` times the reference's own solver (the PhAST package
installed under baseline/_ref) on whole load increments on the host cores; its
JSON line must carry the same metric, unit and workload configuration as the
GPU arm, a `cpu_baseline` describing the sample and an `e2e` object with no
host-device traffic.  Invalid warm-up counts are refused.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, timeout=600):
    return subprocess.run([sys.executable, "bench.py", *args], cwd=ROOT, capture_output=True, text=True,
                          timeout=timeout, env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))


def test_reference_arm_json_line():
    out = run_bench("--impl", "reference", "--steps", "1", "--warmup", "3")
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    sys.path.insert(0, ROOT)
    import bench
    assert line["impl"] == "reference"
    if "unavailable" in line:  # the reference package is not installed in this checkout
        assert not os.path.isdir(os.path.join(ROOT, "baseline", "_ref", "phast"))
        return
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["n_gpus"] == 1 and line["steps"] == 1 and line["warmup"] == 3
    assert line["higher_is_better"] is True and line["data"] == "synthetic"
    assert line["config"] == bench.workload_config()
    assert line["timed_increments"]["timed"] == 1 and len(line["timed_increments"]["seconds"]) == 1
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["unit"] == line["unit"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and "phast.solid3d.StaggeredSolver" in cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_warmup_below_three_is_refused():
    out = run_bench("--impl", "reference", "--steps", "1", "--warmup", "2", timeout=120)
    assert out.returncode != 0
    assert "warmup" in (out.stderr + out.stdout)

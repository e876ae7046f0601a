"""bench.py's output contract on the CPU: the reference arm (`--impl
reference`) runs the reference's kernels compiled for the host, so it can be
run here on the small scene (C0) and its one JSON line checked for the keys
the driver reads -- metric, value, unit, impl, steps, warmup, ms_per_step,
higher_is_better, scaling, dtype, config, cpu_baseline (value, unit, cores,
kind, sample) and e2e (value, unit, host/device bytes). Where oracle/_ref is
absent the arm must print its one-line `unavailable` record and exit 0.
"""
import json
import os
import subprocess
import sys

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    d = run_bench("--impl", "reference", "--scene", "C0", "--steps", "2", "--warmup", "1")
    assert d["impl"] == "reference"
    if not oracle.ref_available():
        assert set(d) == {"impl", "unavailable"} and d["unavailable"]
        return
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["steps"] == 2 and d["warmup"] == 1 and d["value"] > 0 and d["higher_is_better"] is True
    assert d["unit"] == "particle-steps/s" and d["scaling"] == "weak"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert abs(d["ms_per_step"] - d["config"]["particles"] * 1e3 / d["value"]) < 1e-6 * d["ms_per_step"]


def test_reference_arm_other_ranks_print_nothing():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--scene", "C0",
                        "--steps", "1", "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600,
                       env=env)
    assert r.returncode == 0 and not r.stdout.strip()

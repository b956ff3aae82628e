"""The benchmark's reference arm (`bench.py --impl reference`, the CPU restatement of the reference timed on the host)
runs without a GPU: its one JSON line carries the keys of the benchmark contract, at a small size."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_line():
    d = _run("--impl", "reference", "--size", "8", "--steps", "2", "--warmup", "1")
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert 1 <= d["steps"] <= 2 and d["steps_requested"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["ms_per_step"] > 0 and "complete factor + solve" in d["cpu_baseline"]["sample"]
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["workload"].startswith("elastic3d-8")
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0

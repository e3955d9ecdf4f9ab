"""bench.py's reference arm on the CPU: the JSON line the benchmark contract
asks of `bench.py --impl reference` (one line from rank 0 with the metric,
value, unit, step counts, config, a cpu_baseline describing the run, and an
e2e block with no host-device bytes), here on the river workload with a few
iterations so it ends in about a second. CPU only: the reference arm times
the oracle on the host cores and launches no kernel."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_reference(*args):
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, check=True).stdout
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out
    return json.loads(lines[0])


def test_reference_arm_line():
    d = run_reference("--workload", "river", "--steps", "3", "--warmup", "3")
    assert d["impl"] == "reference"
    for key in ("metric", "unit", "dtype", "data", "scaling"):
        assert isinstance(d[key], str) and d[key], key
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["unit"] == "DCFR iters/s" and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3
    assert d["vs_baseline"] is None
    assert "river" in d["config"]["workload"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0

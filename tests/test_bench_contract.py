"""bench.py's reference arm on the CPU: one JSON line in the measurement
contract's shape (the driver computes the speed-up ratio from it), on the small
C1 workload so that it runs in seconds; multi-cell workloads get the
`unavailable` line."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                         capture_output=True, text=True, timeout=600, check=True).stdout
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out
    return json.loads(lines[0])


def test_reference_arm_line():
    d = run_bench("--impl", "reference", "--workload", "c1", "--steps", "2", "--warmup", "0")
    assert d["impl"] == "reference" and d["unit"] == "evals/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 2
    assert d["warmup"] >= 3  # the timing rules' minimum
    assert d["config"]["natoms"] == 64
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert set(cb["split_s"]) == {"real_space", "spread", "fft", "gather", "other"}
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_multi_cell_is_unavailable():
    d = run_bench("--impl", "reference", "--workload", "c4", "--steps", "1")
    assert d["impl"] == "reference" and "unavailable" in d

"""bench.py's JSON contract, checked on the CPU through the reference arm
(`--impl reference` times the CPU port on the host cores, no device), with a
small sample: the keys, their types and the reference arm's e2e convention.
The GPU arm's line needs a B200 and is not covered here."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run_bench(*args) -> dict:
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    d = run_bench("--impl", "reference", "--steps", "1", "--warmup", "3", "--cpu-cells", str(1 << 20))
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 3
    assert d["higher_is_better"] is True and d["scaling"] in ("weak", "strong")
    assert d["config"]["workload"] == "uneven-kb-2^30"
    assert d["value"] > 0 and d["unit"] == "cells/s"
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert cb["cpu_model"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_help_lists_the_workloads():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--help"], cwd=ROOT, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0
    for w in ("uneven-kb-2^30", "recursion-bb-48", "single-kb-2^16x64", "fri-kb-2^23", "serving", "open-kb-2^30"):
        assert w in r.stdout, w

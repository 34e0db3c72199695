"""The benchmark's reference arm (bench.py --impl reference) on the host cores: one JSON line
with the contract's keys, the reference's own arithmetic timed on a bounded sample (no GPU)."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "gri-density", "--steps", "1",
                        "--warmup", "1"], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    b = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in b, k
    assert b["impl"] == "reference" and b["value"] > 0 and b["unit"] == "cells/s"
    assert b["e2e"]["value"] == b["value"] and b["e2e"]["h2d_bytes_per_step"] == 0
    assert b["cpu_baseline"]["cores"] >= 1 and b["cpu_baseline"]["kind"] in ("reference", "port")
    assert b["config"]["workload"] == "gri-density"

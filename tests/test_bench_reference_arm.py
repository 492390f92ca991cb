"""bench.py's reference arm runs on the host only: the reference's own run_sim
(oracle/_ref) on a small case prints one JSON line with the fields the bench
line carries, and a rank other than 0 prints nothing and exits 0."""
import json
import os
import subprocess
import sys

import pytest

import helpers as H

BENCH = os.path.join(H.ROOT, "bench.py")
RUN_SIM = os.path.join(H.ROOT, "oracle", "_ref", "run_sim")
needs_ref = pytest.mark.skipif(not os.path.exists(RUN_SIM), reason="oracle/_ref not built here")

ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "0", "--ref-steps", "1", "--ref-procs", "2",
        "--size", "16"]


@needs_ref
def test_reference_arm_line():
    r = subprocess.run([sys.executable, BENCH] + ARGS, capture_output=True, text=True, timeout=300,
                       cwd=H.ROOT, env=dict(os.environ, RANK="0", WORLD_SIZE="1"))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == d["unit"] == "Mcell-steps/s"
    assert d["value"] > 0 and d["steps"] == 1 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] == 2 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["grid"] == 16


@needs_ref
def test_reference_arm_other_ranks_print_nothing():
    r = subprocess.run([sys.executable, BENCH] + ARGS, capture_output=True, text=True, timeout=300,
                       cwd=H.ROOT, env=dict(os.environ, RANK="1", WORLD_SIZE="2"))
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]

"""bench.py's reference arm on the host cores: one JSON line of the bench
contract, timed on the reference's own arithmetic (the harness under
oracle/), built from particles the oracle's initial conditions generate, and
without loading the CUDA library (checked in the process's mappings)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", "c2", "--steps", "2", "--warmup", "1",
            "--cpu-budget-ref", "2"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    if e.code not in (None, 0):
        raise
print("MAPPED_LIBEMU", open("/proc/self/maps").read().count("libemu_b200"))
"""


def test_reference_arm_line():
    from oracle.oracle import have_ref
    if not have_ref(2):
        pytest.skip("reference-arithmetic harness not built")
    r = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert lines[-1] == "MAPPED_LIBEMU 0"
    d = json.loads([l for l in lines if l.startswith("{")][-1])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "dtype", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["warmup"] >= 3
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["particles"] == 10240

"""CPU checks of bench.py's contract: the reference arm prints one JSON line
with the required keys (it needs no GPU), and the option parsing knows every
workload."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, timeout=600):
    env = dict(os.environ, RANK="0", WORLD_SIZE="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True,
                         text=True, cwd=ROOT, timeout=timeout, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("workload,unit", [("lanczos_chain12", "solves/s"), ("spectrum_chain26", "spectra/s")])
def test_reference_arm_line(workload, unit):
    d = run_bench("--impl", "reference", "--workload", workload, "--steps", "1", "--warmup", "3")
    assert d["impl"] == "reference" and d["unit"] == unit
    for key in ("metric", "value", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "dtype",
                "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "lanczos_chain12", "--steps", "1"], capture_output=True, text=True,
                         cwd=ROOT, timeout=120, env=env)
    assert out.returncode == 0 and out.stdout.strip() == ""


def test_unknown_workload_is_refused():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--workload", "nope"],
                         capture_output=True, text=True, cwd=ROOT, timeout=120)
    assert out.returncode != 0

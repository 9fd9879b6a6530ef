"""bench.py's reference arm on the host (no GPU): one JSON line with the contract's keys."""
import json
import os
import subprocess
import sys

import pytest

from oracle import bindings as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not B.ref_available(), reason="needs the reference build (oracle/_ref)")
def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--rows", "2000",
                          "--cols", "4000", "--steps", "1", "--warmup", "1", "--cpu-sample-iters", "20"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] == 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


def test_gpus_2_starts_two_ranks_and_reduces_over_them():
    """`bench.py --gpus 2` without a launcher starts its own two ranks (torch.distributed.run on
    127.0.0.1); the plumbing check runs the process group on gloo here (no GPU) and rank 0 prints
    the maximum of the ranks' stand-in times."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--plumbing-check"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["plumbing_check"] is True and d["n_gpus"] == 2 and d["ranks"] == [0, 1]
    assert d["value"] == 1.25                       # max over ranks of 1 + rank / 4

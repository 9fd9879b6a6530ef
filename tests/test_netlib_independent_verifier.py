"""Netlib solutions against the reference's own independent validator (validator/
independent_verifier.py: its own MPS and .sol parsers; primal feasibility, objective
consistency, dual feasibility and complementary slackness at tolerance 1e-6).

The .sol files under tests/golden/netlib_sol are what the drop-in wrote on a B200 (the
reference's engine with presolve and postsolve, libvajra_pdhg.so through the shim, the
reference's solution writer; tests/golden/netlib_sol/generate.py), for the 21 Netlib models of
the reference's benchmark Suite 1 in both precisions.  The validator is a Python program of the
reference tree, so this check runs where that tree is (it is skipped elsewhere);
tests/test_netlib_gpu.py re-solves the models on the device and runs the reference's C++ file
verifier on the fresh files.
"""
import gzip
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

import pytest

from __graft_entry__ import REFERENCE_TREE
from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden", "netlib_sol")
VALIDATOR = os.path.join(REFERENCE_TREE, "validator", "independent_verifier.py")
MODELS = os.path.join(REFERENCE_TREE, "SOVEREIGN_SOLVER_BLUEPRINT", "test_models")
PRECISIONS = ("mixed", "fp64")

pytestmark = pytest.mark.skipif(not (os.path.exists(VALIDATOR) and os.path.isdir(MODELS)),
                                reason="the reference tree (its validator and Netlib models) is not present")


def fixtures():
    out = []
    for prec in PRECISIONS:
        d = os.path.join(GOLDEN, prec)
        out += [(prec, f[: -len(".sol.gz")]) for f in sorted(os.listdir(d)) if f.endswith(".sol.gz")]
    return out


def test_every_model_has_a_solution_in_both_precisions():
    names = {p: {n for q, n in fixtures() if q == p} for p in PRECISIONS}
    assert len(names["mixed"]) == 21 and names["mixed"] == names["fp64"], names
    for prec in PRECISIONS:
        with open(os.path.join(GOLDEN, prec + ".log")) as f:
            log = f.read()
        assert log.count("PASS ") == 21 and "OK: 0 failure(s)" in log


def test_reference_validator_accepts_every_solution(tmp_path):
    def check(item):
        prec, name = item
        sol = tmp_path / f"{prec}_{name}.sol"
        with gzip.open(os.path.join(GOLDEN, prec, name + ".sol.gz"), "rb") as f:
            sol.write_bytes(f.read())
        p = subprocess.run([sys.executable, VALIDATOR, os.path.join(MODELS, name + ".mps"), str(sol), "1e-6"],
                           capture_output=True, text=True, timeout=600)
        return prec, name, p.returncode, p.stdout[-1500:]

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        results = list(pool.map(check, fixtures()))
    failed = [(prec, name, out) for prec, name, rc, out in results if rc != 0 or "[VERIFIED OPTIMAL]" not in out]
    assert not failed, failed[:3]
    assert len(results) == 42


def test_reference_validator_rejects_a_planted_error(tmp_path):
    """The same check on a copy of one solution with one primal value moved by 1 (planted on the
    CPU): the validator must reject it, so a pass above means something."""
    with gzip.open(os.path.join(GOLDEN, "mixed", "afiro.sol.gz"), "rt") as f:
        lines = f.read().splitlines()
    i = next(k for k, line in enumerate(lines) if line.startswith("X02 "))
    name, value, rest = lines[i].split(" ", 2)
    lines[i] = f"{name} {float(value) + 1.0!r} {rest}"
    sol = tmp_path / "afiro_planted.sol"
    sol.write_text("\n".join(lines) + "\n")
    p = subprocess.run([sys.executable, VALIDATOR, os.path.join(MODELS, "afiro.mps"), str(sol), "1e-6"],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode != 0 and "[FAILED]" in p.stdout, p.stdout[-1500:]

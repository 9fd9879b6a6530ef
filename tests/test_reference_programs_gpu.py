"""The reference's own test programs, compiled unmodified from its tree and linked against the
drop-in (tests/dropin/Makefile), run on the device from the staged model directory:

* tests/test_pdhg.cpp        -- all 11 tests, including [TEST 10], the GPU request through
                                indus::solve (tests/test_pdhg.cpp:405-436);
* tests/test_reliability.cpp -- all 10, including the GPU request of :375-396;
* apps/benchmark_runner.cpp  -- its Suite 2 (:860-1068), which solves five models through
                                indus::gpu::solve_pdhg_gpu and reports get_last_gpu_timing();
* tests/test_benchmark_harness.cpp -- runs, and stops where it asserts that a CPU-only build
                                reports no CUDA device (:80-83): with the B200 backend a device is
                                present, the one deliberate difference (no CPU fallback).
"""
import json
import os
import subprocess

import pytest

from conftest import ROOT

BUILD = os.path.join(ROOT, "tests", "dropin", "_build")
MODELS = os.path.join(BUILD, "models")
needs = pytest.mark.skipif(not os.path.isdir(MODELS), reason="reference programs not built (needs the reference tree)")
pytestmark = [pytest.mark.gpu, needs]


def run(args, timeout=1200):
    p = subprocess.run(args, cwd=MODELS, capture_output=True, text=True, timeout=timeout)
    print(p.stdout[-6000:])
    return p


def test_reference_test_pdhg(cuda):
    p = run([os.path.join(BUILD, "ref_test_pdhg")])
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-2000:]
    assert "ALL 11 PHASE 5 PDHG & GPU TESTS PASSED" in p.stdout
    assert "Available: YES" in p.stdout


def test_reference_test_reliability(cuda):
    p = run([os.path.join(BUILD, "ref_test_reliability")])
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-2000:]
    assert "ALL 10 PHASE 6 RELIABILITY & HARDENING TESTS PASSED" in p.stdout


def test_reference_benchmark_suite_2_measures_gpu_timings(cuda, tmp_path):
    js = tmp_path / "bench.json"
    p = run([os.path.join(BUILD, "indus_benchmark"), "--suite", "cuda", "--quick", "--out-dir", str(tmp_path),
             "--json", str(js), "--csv", str(tmp_path / "bench.csv")])
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-2000:]
    assert "NOT_MEASURED" not in p.stdout
    with open(js) as f:
        rows = json.load(f)["results"]
    assert rows and all(r["suite"] == "cuda" for r in rows)


def test_reference_benchmark_harness_differs_only_in_its_no_device_assertion(cuda):
    p = run([os.path.join(BUILD, "ref_test_benchmark_harness"), os.path.join(BUILD, "indus_benchmark")])
    assert p.returncode != 0
    assert "In CPU-only build, CUDA device must be reported as unavailable" in p.stderr

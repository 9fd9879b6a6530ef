"""The reference engine (indus::solve, compiled from the reference's sources) reaching the
B200 backend through the C++20 drop-in shim: tests/dropin/test_dropin.cpp."""
import os
import subprocess

import pytest

from conftest import ROOT, cuda_device_present

BIN = os.path.join(ROOT, "tests", "dropin", "_build", "test_dropin")
needs_bin = pytest.mark.skipif(not os.path.exists(BIN), reason="drop-in test binary not built (needs the reference tree)")


@needs_bin
@pytest.mark.skipif(cuda_device_present(), reason="checks the no-device path")
def test_engine_without_device_reports_unsupported():
    p = subprocess.run([BIN], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "UNSUPPORTED" in p.stdout


@needs_bin
@pytest.mark.gpu
def test_engine_reference_lps_through_dropin(cuda):
    p = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(p.stdout)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.count("PASS") == 16

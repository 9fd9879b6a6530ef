"""Netlib end to end on the device: the reference's MPS reader (at build time, into binary dumps
under tests/dropin/_build/netlib), its engine with presolve and postsolve, the drop-in shim to
libvajra_pdhg.so, its solution writer and its file verifier; every model OPTIMAL, verified, and
within 1e-6 (relative) of its published optimum (tests/dropin/netlib_e2e.cpp)."""
import json
import os
import subprocess

import pytest

from conftest import ROOT

BIN = os.path.join(ROOT, "tests", "dropin", "_build", "netlib_e2e")
PACK = os.path.join(ROOT, "tests", "dropin", "_build", "netlib")
needs_pack = pytest.mark.skipif(not (os.path.exists(BIN) and os.path.exists(os.path.join(PACK, "optima.json"))),
                                reason="Netlib dumps not built (needs the reference tree at build time)")


@needs_pack
@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_netlib_models_end_to_end(cuda, tmp_path, precision):
    with open(os.path.join(PACK, "optima.json")) as f:
        optima = json.load(f)
    args = [f"{name}={value!r}" for name, value in sorted(optima.items())]
    p = subprocess.run([BIN, "solve", PACK, str(tmp_path), precision] + args, capture_output=True, text=True,
                       timeout=1800)
    print(p.stdout)
    assert p.returncode == 0, p.stdout[-4000:] + p.stderr[-2000:]
    assert p.stdout.count("PASS ") == len(optima)
    for name in optima:
        assert os.path.getsize(os.path.join(tmp_path, name + ".sol")) > 0

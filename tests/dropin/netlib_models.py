"""Build step of the Netlib end-to-end check (run by __graft_entry__.build() where the reference
tree is present): packs the Netlib LP models the reference publishes optima for into binary
dumps with the reference's own MPS reader (tests/dropin/_build/netlib_e2e pack), and records
those optima in tests/dropin/_build/netlib/optima.json.  The outputs are git-ignored build
files; the GPU test (tests/test_netlib_gpu.py) needs nothing from the reference tree.

Published optima, read in place from the reference tree:
* SOVEREIGN_SOLVER_BLUEPRINT/test_models/reference.json  ("published_optimal", from netlib.org)
* apps/benchmark_runner.cpp, its Suite 1 instance table (name, model path, expected objective)
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build", "netlib")
BIN = os.path.join(HERE, "_build", "netlib_e2e")


def published_optima(ref: str) -> dict:
    opt = {}
    with open(os.path.join(ref, "apps", "benchmark_runner.cpp")) as f:
        for m in re.finditer(r'\{"(\w+)",\s*"SOVEREIGN_SOLVER_BLUEPRINT/test_models/(\w+)\.mps",\s*'
                             r'([-+0-9.eE]+),\s*false\}', f.read()):
            opt[m.group(2)] = float(m.group(3))
    with open(os.path.join(ref, "SOVEREIGN_SOLVER_BLUEPRINT", "test_models", "reference.json")) as f:
        for name, inst in json.load(f)["instances"].items():
            opt[name] = float(inst["published_optimal"])      # netlib.org's figure where both list one
    return opt


def main(ref: str) -> int:
    os.makedirs(OUT, exist_ok=True)
    opt = published_optima(ref)
    models = os.path.join(ref, "SOVEREIGN_SOLVER_BLUEPRINT", "test_models")
    names = sorted(n for n in opt if os.path.exists(os.path.join(models, n + ".mps")))
    subprocess.run([BIN, "pack", models, OUT] + names, check=True)
    with open(os.path.join(OUT, "optima.json"), "w") as f:
        json.dump({n: opt[n] for n in names}, f, indent=1, sort_keys=True)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1]))

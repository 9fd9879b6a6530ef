"""Regenerates the Netlib solution fixtures in this folder (needs a CUDA device).

Runs the drop-in's Netlib end-to-end program (tests/dropin/_build/netlib_e2e: the reference's
engine with presolve and postsolve, the shim to libvajra_pdhg.so, the reference's solution
writer) over the binary model dumps in tests/dropin/_build/netlib, in both precisions, and
stores every written .sol file gzipped as <precision>/<model>.sol.gz beside its run log
<precision>.log.  tests/test_netlib_independent_verifier.py then checks the fixtures with the
reference's own validator/independent_verifier.py wherever the reference tree is present.

    python tests/golden/netlib_sol/generate.py
"""
import gzip
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
BIN = os.path.join(ROOT, "tests", "dropin", "_build", "netlib_e2e")
PACK = os.path.join(ROOT, "tests", "dropin", "_build", "netlib")


def main() -> int:
    with open(os.path.join(PACK, "optima.json")) as f:
        optima = json.load(f)
    args = [f"{name}={value!r}" for name, value in sorted(optima.items())]
    rc = 0
    for precision in ("mixed", "fp64"):
        with tempfile.TemporaryDirectory() as tmp:
            p = subprocess.run([BIN, "solve", PACK, tmp, precision] + args, capture_output=True, text=True)
            with open(os.path.join(HERE, precision + ".log"), "w") as f:
                f.write(p.stdout)
            rc |= p.returncode
            out = os.path.join(HERE, precision)
            os.makedirs(out, exist_ok=True)
            for name in sorted(optima):
                src = os.path.join(tmp, name + ".sol")
                if not os.path.exists(src):
                    print(f"{precision} {name}: no solution written", file=sys.stderr)
                    rc = 1
                    continue
                with open(src, "rb") as fi, open(os.path.join(out, name + ".sol.gz"), "wb") as raw, \
                        gzip.GzipFile(filename="", mode="wb", compresslevel=9, fileobj=raw, mtime=0) as fo:
                    shutil.copyfileobj(fi, fo)
        print(p.stdout.strip().splitlines()[-1] if p.stdout.strip() else f"{precision}: no output")
    return rc


if __name__ == "__main__":
    sys.exit(main())

"""The ctypes mirrors of the C ABI structs (vajra_pdhg/_capi.py, vajra_pdhg/autograd.py) against
the header itself: a small C program compiled here prints sizeof and every field's offset, and
each must equal what ctypes computes.  A field added to include/vajra_pdhg.h but not to the
mirror (or the reverse) fails here before any call passes misread options."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from vajra_pdhg import _capi, autograd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = [("vajra_lp", _capi.VajraLp), ("vajra_opts", _capi.VajraOpts), ("vajra_result", _capi.VajraResult),
           ("vajra_device_info", _capi.VajraDeviceInfo), ("vajra_timing", _capi.VajraTiming),
           ("vajra_device_diagnostics", _capi.VajraDeviceDiagnostics),
           ("vajra_unrolled_opts", autograd.VajraUnrolledOpts)]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_header(tmp_path):
    structs = STRUCTS
    lines = ["#include <stdio.h>", "#include <stddef.h>", "#include \"vajra_pdhg.h\"", "int main(void) {"]
    for cname, py in structs:
        lines.append(f'    printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'    printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line.strip():
            cname, field, value = line.split()
            got[(cname, field)] = int(value)
    for cname, py in structs:
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_abi_version_matches_the_header():
    with open(os.path.join(ROOT, "include", "vajra_pdhg.h")) as f:
        text = f.read()
    line = [l for l in text.splitlines() if l.startswith("#define VAJRA_ABI_VERSION")][0]
    assert int(line.split()[2]) == _capi.ABI_VERSION

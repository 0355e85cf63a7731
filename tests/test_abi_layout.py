"""The ctypes mirror (tinypt_b200/_abi.py) against include/tinypt_cuda.h.

A C probe, compiled by the host C compiler from the header itself, prints
every struct's size and every field's offset, and the value of every
constant the mirror defines; the mirror must agree on all of them.  A field
the header does not have fails the probe's compilation.
"""
import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from tinypt_b200 import _abi

HEADER = Path(__file__).resolve().parent.parent / "include" / "tinypt_cuda.h"

STRUCTS = sorted(
    (v for k, v in vars(_abi).items() if k.startswith("tpt_") and isinstance(v, type) and issubclass(v, C.Structure)),
    key=lambda s: s.__name__,
)
CONSTANTS = sorted(k for k, v in vars(_abi).items() if k.startswith("TPT_") and isinstance(v, int))


def _probe_source():
    out = ["#include <stddef.h>", "#include <stdio.h>", f'#include "{HEADER}"', "int main(void) {"]
    for s in STRUCTS:
        n = s.__name__
        out.append(f'    printf("{n} %zu\\n", sizeof({n}));')
        for f in s._fields_:
            out.append(f'    printf("{n}.{f[0]} %zu\\n", offsetof({n}, {f[0]}));')
    for k in CONSTANTS:
        out.append(f'    printf("{k} %lld\\n", (long long)({k}));')
    out += ["    return 0;", "}"]
    return "\n".join(out) + "\n"


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "probe.c", d / "probe"
    src.write_text(_probe_source())
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return dict(line.rsplit(" ", 1) for line in out.splitlines())


def test_mirror_covers_every_header_struct():
    declared = set(re.findall(r"\}\s*(tpt_[a-z_0-9]+)\s*;", HEADER.read_text()))
    assert declared == {s.__name__ for s in STRUCTS}


@pytest.mark.parametrize("struct", STRUCTS, ids=lambda s: s.__name__)
def test_struct_layout_matches_header(c_layout, struct):
    n = struct.__name__
    assert C.sizeof(struct) == int(c_layout[n]), f"sizeof({n})"
    for f in struct._fields_:
        assert getattr(struct, f[0]).offset == int(c_layout[f"{n}.{f[0]}"]), f"offsetof({n}, {f[0]})"


def test_constants_match_header(c_layout):
    assert CONSTANTS
    for k in CONSTANTS:
        assert getattr(_abi, k) == int(c_layout[k]), k

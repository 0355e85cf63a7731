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


# ---- the Rust `extern "C"` binding (include/tinypt_sys.rs) ---------------------

RUST_BINDING = HEADER.parent / "tinypt_sys.rs"
C_EXAMPLE = HEADER.parent / "tinypt_example.c"
_C_BASE = {"int": "i32", "int32_t": "i32", "int64_t": "i64", "uint32_t": "u32", "uint64_t": "u64",
           "double": "f64", "float": "f32", "char": "c_char", "void": "void"}
_RUST_BASE = {"c_int": "i32", "c_double": "f64", "c_char": "c_char", "c_void": "void"}


def _c_type(t):
    """'const double*' -> '*const f64'; 'void**' -> '*mut *mut void'."""
    t = t.strip()
    depth = t.count("*")
    const = t.startswith("const ")
    base = t.replace("const ", "").replace("*", "").strip()
    base = _C_BASE.get(base, base)
    for k in range(depth):
        # only the innermost pointer carries the declared constness
        base = ("*const " if (const and k == 0) else "*mut ") + base
    return base


def _rust_type(t):
    t = " ".join(t.split())
    prefix = ""
    while t.startswith("*"):
        kind, t = t.split(" ", 1)
        prefix += kind + " "
    if t.startswith("Tpt"):
        base = "tpt" + re.sub(r"([A-Z])", lambda m: "_" + m.group(1).lower(), t[3:])
    else:
        base = _RUST_BASE.get(t, t)
    return (prefix + base).strip()


def _param_type(p):
    """'const double dir[3]' -> 'const double*'; 'int32_t* out' -> 'int32_t*'."""
    p = p.strip()
    if p.endswith("]"):
        p = re.sub(r"\s*\b[A-Za-z_0-9]+\s*\[[^]]*\]$", "", p) + "*"
        return p
    return re.sub(r"\b[A-Za-z_0-9]+$", "", p)


def _header_functions(path=HEADER, prefix="tpt_"):
    text = re.sub(r"/\*.*?\*/", "", Path(path).read_text(), flags=re.S)
    out = {}
    pat = r"([A-Za-z_0-9 ]+\**)\s*\b(" + prefix + r"[a-z_0-9]+)\s*\(([^)]*)\)\s*;"
    for ret, name, params in re.findall(pat, text):
        ps = [p.strip() for p in params.split(",") if p.strip() and p.strip() != "void"]
        # a parameter is 'type name'; the type keeps the pointer stars
        types = [_c_type(_param_type(p)) for p in ps]
        r = _c_type(ret.strip())
        out[name] = (types, None if r == "void" else r)
    return out


def _rust_block():
    return RUST_BINDING.read_text()


def _rust_functions():
    out = {}
    body = " ".join(_rust_block().split())
    for name, params, ret in re.findall(r"pub fn (tpt_[a-z_0-9]+)\(([^)]*)\)\s*(?:->\s*([^;]+))?;", body):
        types = [_rust_type(p.split(":", 1)[1]) for p in params.split(",") if p.strip()]
        out[name] = (types, _rust_type(ret) if ret else None)
    return out


def test_rust_binding_declares_every_header_function_with_its_types():
    header, rust = _header_functions(), _rust_functions()
    assert "tpt_render" in header and "tpt_render_resume" in header
    assert set(rust) == set(header)
    for name, sig in header.items():
        assert rust[name] == sig, name


def _rust_size(t, structs):
    t = " ".join(t.split())
    if t.startswith("*"):
        return 8
    m = re.fullmatch(r"\[(.+);\s*(\d+)\]", t)
    if m:
        return _rust_size(m.group(1), structs) * int(m.group(2))
    sizes = {"i32": 4, "u32": 4, "f32": 4, "i64": 8, "u64": 8, "f64": 8}
    return sizes[t] if t in sizes else C.sizeof(structs[t])


def test_rust_structs_match_the_mirror():
    structs = {"Tpt" + "".join(w.title() for w in s.__name__[4:].split("_")): s for s in STRUCTS}
    body = _rust_block()
    found = re.findall(r"pub struct (Tpt[A-Za-z]+)\s*\{(.*?)\}", body, flags=re.S)
    assert {n for n, _ in found} == set(structs)
    for name, fields in found:
        fields = re.sub(r"//[^\n]*", "", fields)
        parsed = [f.split(":", 1) for f in fields.replace("pub ", "").split(",") if f.strip()]
        mirror = structs[name]._fields_
        assert [n.strip() for n, _ in parsed] == [f[0] for f in mirror], name
        for (n, t), f in zip(parsed, mirror):
            assert _rust_size(t, structs) == C.sizeof(f[1]), f"{name}.{n.strip()}"


def test_c_example_compiles_against_the_header(tmp_path):
    """include/tinypt_example.c compiles against include/tinypt_cuda.h."""
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    src = tmp_path / "example.c"
    src.write_text(C_EXAMPLE.read_text().replace('#include "tinypt_cuda.h"', f'#include "{HEADER}"'))
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-c", str(src), "-o", str(tmp_path / "example.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


_CTYPES_BASE = {C.c_int: "i32", C.c_int32: "i32", C.c_int64: "i64", C.c_uint32: "u32", C.c_uint64: "u64",
                C.c_double: "f64", C.c_float: "f32"}


def _ctypes_type(t):
    """A ctypes type as the header form without constness; c_void_p is any pointer."""
    if t is None:
        return None
    if t is C.c_void_p:
        return "*any"
    if t is C.c_char_p:
        return "*c_char"
    if t in _CTYPES_BASE:
        return _CTYPES_BASE[t]
    if hasattr(t, "_type_") and issubclass(t, C._Pointer):
        inner = _ctypes_type(t._type_)
        # a c_void_p pointed to (an out-handle) is a void* in the header
        return "*" + ("*void" if inner == "*any" else inner)
    if issubclass(t, C.Structure):
        return t.__name__
    raise AssertionError(f"unmapped ctypes type {t}")


def _strip_const(t):
    return None if t is None else t.replace("*const ", "*").replace("*mut ", "*")


def _same(ct, ht):
    if ct == "*any":
        return ht is not None and ht.startswith("*")
    return ct == ht


def test_ctypes_signatures_match_the_header():
    header = _header_functions()
    assert set(_abi.SIGNATURES) == set(header)
    for name, (res, args) in _abi.SIGNATURES.items():
        h_args, h_res = header[name]
        assert len(args) == len(h_args), name
        assert _same(_ctypes_type(res), _strip_const(h_res)), f"{name} returns {h_res}"
        for k, (a, h) in enumerate(zip(args, h_args)):
            assert _same(_ctypes_type(a), _strip_const(h)), f"{name} argument {k}: {a} vs {h}"


def test_oracle_ctypes_signatures_match_its_header():
    """The checker's own binding (oracle/oracle.py) against oracle/oracle.h."""
    from oracle import oracle as O

    header = _header_functions(HEADER.parent.parent / "oracle" / "oracle.h", "oracle_")
    lib = O.lib()
    assert "oracle_scene_render" in header and "oracle_env_eval" in header
    for name, (h_args, h_res) in header.items():
        fn = getattr(lib, name)
        assert fn.argtypes is not None, f"{name} has no argtypes"
        assert len(fn.argtypes) == len(h_args), name
        assert _same(_ctypes_type(fn.restype), _strip_const(h_res)), f"{name} returns {h_res}"
        for k, (a, h) in enumerate(zip(fn.argtypes, h_args)):
            assert _same(_ctypes_type(a), _strip_const(h)), f"{name} argument {k}: {a} vs {h}"

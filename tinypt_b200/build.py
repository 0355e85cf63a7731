"""Builds the sm_100a shared library ``tinypt_b200/libtinypt_cuda.so``.

The library is compiled in-tree with nvcc for ``sm_100a`` only.  Each
translation unit gets the floating-point flags its numerics need:

* ``plain_f64.cu``: ``-fmad=false`` so the f64 kernel rounds ``a*b+c`` twice
  like the reference;
* ``bvh_build.cu``: ``-fmad=false`` so the device BVH build's box and SAH
  arithmetic equals the host builder's;
* ``wavefront.cu``, ``adjoint.cu``: FP32 with approximate division/sqrt and
  flush-to-zero (the FP32 form is checked statistically), and no automatic
  FMA contraction (``-fmad=false``; the traversal's slab test writes its
  FMAs out): automatic contraction varied with each kernel instantiation's
  register budget, and batch films, single films and the adjoint must
  follow the same paths bit for bit;
* ``host_scene.cu`` / ``capi.cu`` / ``image_io.cpp`` / ``scene_io.cpp`` /
  ``fp32_tree.cpp``: host
  code with ``-ffp-contract=off`` so the f64 scene quantities (camera basis,
  transforms, BVH boxes, CDFs) match the reference's.

The command-line renderer ``tinypt_b200/bin/tinypt`` (``cli/tinypt.cpp``,
the reference's flags) is linked against the library.

Run ``python -m tinypt_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libtinypt_cuda.so"
CLI = PKG / "bin" / "tinypt"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-Xptxas", "-v"]
UNITS = {
    "host_scene.cu": [],
    "capi.cu": [],
    "plain_f64.cu": ["-fmad=false"],
    "bvh_build.cu": ["-fmad=false"],
    "wavefront.cu": ["-fmad=false", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    "adjoint.cu": ["-fmad=false", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    "image_io.cpp": [],
    "scene_io.cpp": [],
    "checkpoint.cpp": [],
    "fp32_tree.cpp": [],
    "probe.cu": [],
}


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found")
    return exe


def _run(cmd: list[str], log: Path) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    log.write_text(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every translation unit that is older than its sources and
    links the shared library.  Returns the library path."""
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp"))
    headers.append(PKG.parent / "include" / "tinypt_cuda.h")
    newest_header = max(p.stat().st_mtime for p in headers)
    objs = []
    for unit, flags in UNITS.items():
        src = CSRC / unit
        obj = BUILD / (unit + ".o")
        objs.append(obj)
        stale = force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)
        if stale:
            cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", str(src), "-o", str(obj)]
            _run(cmd, BUILD / (unit + ".log"))
            if verbose:
                print((BUILD / (unit + ".log")).read_text())
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        _run(cmd, BUILD / "link.log")
    # the command-line renderer, linked against the library (rpath = its folder)
    cli_src = PKG / "cli" / "tinypt.cpp"
    if force or not CLI.exists() or CLI.stat().st_mtime < max(cli_src.stat().st_mtime, LIB.stat().st_mtime):
        CLI.parent.mkdir(exist_ok=True)
        cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", str(cli_src), "-o", str(CLI), f"-L{PKG}",
               "-ltinypt_cuda", "-Wl,-rpath,$ORIGIN/.."]
        _run(cmd, BUILD / "cli.log")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)

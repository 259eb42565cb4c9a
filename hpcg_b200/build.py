"""Builds libhpcgx.so (the sm_100a kernels and their C ABI) in-tree with nvcc.

The library is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``)
and written next to this file, so that it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libhpcgx.so")
LIB_CHECKED = os.path.join(HERE, "libhpcgx_checked.so")   # -DHPCGX_CHECKED: index-checked kernels
SOURCES = ["kernels.cu", "problem.cu", "noalloc.cu", "general.cu"]
HEADERS = ["common.cuh", "kernels.cuh", "general.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    """Compiles every .cu of csrc/ into libhpcgx.so (checked: libhpcgx_checked.so
    with -DHPCGX_CHECKED) when a source is newer."""
    lib = LIB_CHECKED if checked else LIB
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "hpcgx.h")]
    if not force and not _stale(lib, deps):
        return lib
    objdir = os.path.join(HERE, "_build_checked" if checked else "_build")
    flags = FLAGS + (["-DHPCGX_CHECKED"] if checked else [])
    os.makedirs(objdir, exist_ok=True)
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [NVCC, *ARCH, *flags, "-I", INCLUDE, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                            text=True)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + out)
        if verbose and out:
            print(out)
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-Xlinker",
           "-soname=" + os.path.basename(lib), "-o", lib, *objs]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + out.stdout + out.stderr)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv))

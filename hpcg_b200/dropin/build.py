"""Builds xhpcg_b200: the reference's own benchmark driver (src/main.cpp and
every non-replaceable source file, compiled where they lie) linked with the
drop-in operator files of this directory and libhpcgx.so.

Needs the reference's src/ directory in the environment variable HPCG_REF_SRC;
the binary is written to _build/ next to this file and found by tests through
BINARY.  Without the sources nothing is built.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
REF = os.environ.get("HPCG_REF_SRC", "")
BINARY = os.path.join(HERE, "_build", "xhpcg_b200")
# The files HPCG expects an implementation to replace (src/*.cpp forwarding to
# *_ref); GenerateProblem.cpp is replaced to cut set-up time (same data).
REPLACED = ["CG.cpp", "ComputeSPMV.cpp", "ComputeSYMGS.cpp", "ComputeMG.cpp",
            "ComputeDotProduct.cpp", "ComputeWAXPBY.cpp", "OptimizeProblem.cpp",
            "GenerateProblem.cpp"]


def build(force: bool = False) -> str | None:
    if not REF or not os.path.exists(os.path.join(REF, "main.cpp")):
        return None
    if ROOT not in sys.path:   # run as a script: the package sits two levels up
        sys.path.insert(0, ROOT)
    from hpcg_b200 import build as hb
    lib = hb.build()
    ref_srcs = sorted(p for p in glob.glob(os.path.join(REF, "*.cpp"))
                      if os.path.basename(p) not in REPLACED)
    ours = sorted(glob.glob(os.path.join(HERE, "*.cpp")))
    deps = ref_srcs + ours + glob.glob(os.path.join(HERE, "*.hpp")) + [lib, __file__]
    if (not force and os.path.exists(BINARY)
            and all(os.path.getmtime(d) <= os.path.getmtime(BINARY) for d in deps)):
        return BINARY
    os.makedirs(os.path.dirname(BINARY), exist_ok=True)
    # HPCG_CONTIGUOUS_ARRAYS: the reference's own build option (setup/Make.*,
    # line 101) that allocates each level's rows as one block instead of one
    # allocation per row; it shortens set-up and is honoured alike by
    # GenerateProblem.cpp here and the reference's DeleteMatrix.
    cmd = ["g++", "-O3", "-fno-fast-math", "-ffp-contract=off", "-fopenmp", "-pthread", "-DHPCG_NO_MPI",
           "-DHPCG_CONTIGUOUS_ARRAYS", "-w",
           "-I", REF, "-I", HERE, "-I", os.path.join(ROOT, "include"), "-o", BINARY,
           *ref_srcs, *ours, lib, "-Wl,-rpath,$ORIGIN/../.."]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("drop-in build failed:\n" + " ".join(cmd) + "\n" + out.stderr[-4000:])
    return BINARY


if __name__ == "__main__":
    print(build(force=True))

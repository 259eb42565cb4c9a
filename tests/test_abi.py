"""The C-ABI library loads on a machine without a GPU and exports exactly the
functions include/hpcgx.h declares; without a device it fails with a status
code, never a crash.  No compute call is made here."""
import ctypes as C
import os
import re

import pytest
import torch

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "hpcgx.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(hpcgx_\w+)\s*\(", text))


def status_code(name):
    """The value of a status macro of include/hpcgx.h."""
    m = re.search(r"#define\s+%s\s+(\d+)" % name, open(HEADER).read())
    assert m, name
    return int(m.group(1))


def test_header_declares_the_operator_set():
    names = declared()
    for f in ("hpcgx_cg", "hpcgx_spmv", "hpcgx_symgs", "hpcgx_mg", "hpcgx_dot", "hpcgx_waxpby",
              "hpcgx_residual", "hpcgx_restriction", "hpcgx_prolongation", "hpcgx_create",
              "hpcgx_load_level_rows", "hpcgx_cg_mixed", "hpcgx_adjoint_grad"):
        assert f in names


def test_library_exports_every_declared_symbol():
    from hpcg_b200 import _lib
    h = _lib.lib()
    for name in declared():
        assert hasattr(h, name), name
    assert set(_lib.SIGNATURES) == declared()
    assert h.hpcgx_version() >= 1


def test_checked_library_exports_the_same_symbols():
    """The index-checked build (HPCGX_LIBRARY=checked) is the same ABI."""
    import ctypes
    from hpcg_b200 import _lib
    path = os.path.join(_lib.HERE, "libhpcgx_checked.so")
    if not os.path.exists(path):
        pytest.skip("libhpcgx_checked.so not built")
    h = ctypes.CDLL(path)
    for name in declared():
        assert hasattr(h, name), name


def test_library_is_sm100a_only():
    """The fatbin is built for sm_100a (checked from the build recipe, not by
    reading the binary)."""
    from hpcg_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU error path")
def test_create_without_gpu_returns_status():
    from hpcg_b200 import _lib
    h = C.c_void_p()
    rc = _lib.lib().hpcgx_create(0, 16, 16, 16, 4, C.byref(h))
    assert rc == 2 and not h.value
    assert _lib.lib().hpcgx_last_error()
    assert _lib.lib().hpcgx_init_device(0) == 2


def test_bad_arguments_rejected_before_any_device_work():
    from hpcg_b200 import _lib
    h = C.c_void_p()
    assert _lib.lib().hpcgx_create(0, 15, 16, 16, 4, C.byref(h)) == 1   # odd: cannot coarsen
    assert _lib.lib().hpcgx_create(0, 16, 16, 16, 5, C.byref(h)) == 1   # > 4 levels
    assert _lib.lib().hpcgx_create(0, 0, 16, 16, 1, C.byref(h)) == 1
    assert _lib.lib().hpcgx_spmv(None, 0, None, None) == 1
    assert b"null problem" in _lib.lib().hpcgx_last_error()


def test_product_fails_loudly_without_library(tmp_path, monkeypatch):
    from hpcg_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.lib()


def test_header_compiles_and_links_from_c(tmp_path):
    """include/hpcgx.h is plain C: a C program includes it, links libhpcgx.so
    and calls through it (a bad geometry is refused with HPCGX_EINVAL before
    any device is touched; without a GPU, creation fails with a status)."""
    import shutil
    import subprocess
    from hpcg_b200 import _lib
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    src = tmp_path / "use_hpcgx.c"
    src.write_text(r'''
#include <stdio.h>
#include "hpcgx.h"
int main(void) {
  hpcgx_problem *p = 0;
  if (hpcgx_version() < 1) return 10;
  if (hpcgx_create(0, 0, 16, 16, 4, &p) != HPCGX_EINVAL || p) return 11;
  if (!hpcgx_last_error()[0]) return 12;
  int rc = hpcgx_create(0, 16, 16, 16, 4, &p);
  if (rc == HPCGX_OK) { hpcgx_destroy(p); printf("created\n"); return 0; }
  printf("no device: %d %s\n", rc, hpcgx_last_error());
  return p == 0 ? 0 : 13;
}
''')
    exe = tmp_path / "use_hpcgx"
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", libdir, "-lhpcgx",
                    "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr


def test_dropin_driver_without_device_reports_every_call(tmp_path):
    """The reference's driver linked with the drop-in, on a host without a
    usable CUDA device: OptimizeProblem names the failure, and every replaced
    operator (CG, SpMV, MG, dot) then returns HPCGX_ESTATE to the driver, which
    counts the errors (src/main.cpp:190-192); nothing falls back to the
    reference kernels and no VALID report is written."""
    import glob
    import os
    import subprocess
    from hpcg_b200.dropin.build import BINARY
    if not os.path.exists(BINARY):
        pytest.skip("xhpcg_b200 not built (needs the reference sources at build time)")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="2")
    out = subprocess.run([BINARY, "--nx=16", "--ny=16", "--nz=16", "--rt=0"], cwd=tmp_path,
                         env=env, capture_output=True, text=True, timeout=300)
    # the exit status is the reference driver's own affair (src/main.cpp:317
    # sizes its CG sets by the failed CG's time); the log and report carry the verdict
    del out
    logs = glob.glob(str(tmp_path / "hpcg*T*.txt"))
    assert len(logs) == 1
    log = open(logs[0]).read()
    assert log.splitlines()[0].startswith("OptimizeProblem: hpcgx_create: hpcgx error 2:")
    state = status_code("HPCGX_ESTATE")
    for op in ("CG", "SpMV", "MG", "dot"):
        assert "Error in call to %s: %d." % (op, state) in log, op
    for report in glob.glob(str(tmp_path / "HPCG-Benchmark_3.1_*.txt")):
        assert "VALID with a GFLOP/s rating" not in open(report).read()

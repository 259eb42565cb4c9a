"""The reference's own driver (src/main.cpp with TestCG, TestSymmetry,
TestNorms, the residual-reduction gate and ReportResults) linked with the
drop-in operator files of hpcg_b200/dropin and run on the GPU.  The run must
be reported VALID with every test PASSED and no "Reference version of ...
used" remark, i.e. the benchmark accepted the replacement."""
import glob
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
BINARY = os.path.join(ROOT, "hpcg_b200", "dropin", "_build", "xhpcg_b200")


def run_driver(tmp_path, nx, ny, nz, rt=0, extra_env=None):
    if not os.path.exists(BINARY):
        pytest.skip("xhpcg_b200 not built (needs the reference sources at build time)")
    env = dict(os.environ, OMP_NUM_THREADS=str(min(8, os.cpu_count() or 1)), **(extra_env or {}))
    out = subprocess.run([BINARY, f"--nx={nx}", f"--ny={ny}", f"--nz={nz}", f"--rt={rt}"],
                         cwd=tmp_path, capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    reports = glob.glob(str(tmp_path / "HPCG-Benchmark_3.1_*.txt"))
    assert len(reports) == 1
    kv = {}
    for line in open(reports[0]):
        if "=" in line:
            k, v = line.rstrip("\n").split("=", 1)
            kv[k] = v
    logs = glob.glob(str(tmp_path / "hpcg*T*.txt"))
    return kv, open(logs[0]).read() if logs else ""


@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 32, 32), (32, 24, 16), (64, 64, 64)],
                         ids=lambda d: "x".join(map(str, d)))
def test_reference_driver_accepts_dropin(tmp_path, dims):
    kv, log = run_driver(tmp_path, *dims)
    assert kv["Spectral Convergence Tests::Result"] == "PASSED"
    assert int(kv["Spectral Convergence Tests::Unpreconditioned::Maximum iteration count"]) <= 12
    assert int(kv["Spectral Convergence Tests::Preconditioned::Maximum iteration count"]) <= 2
    sym = "Departure from Symmetry |x'Ay-y'Ax|/(2*||x||*||A||*||y||)/epsilon"
    assert kv[sym + "::Result"] == "PASSED"
    assert float(kv[sym + "::Departure for SpMV"]) <= 1.0
    assert float(kv[sym + "::Departure for MG"]) <= 1.0
    assert kv["Iteration Count Information::Result"] == "PASSED"
    assert kv["Reproducibility Information::Result"] == "PASSED"
    assert "Final Summary::HPCG result is VALID with a GFLOP/s rating of" in kv
    assert not any(k.startswith("Final Summary::Reference version of") for k in kv)
    # A * xexact = b exactly through the drop-in SpMV (src/TestSymmetry.cpp:122-132)
    assert "SpMV call [0] Residual [0]" in log
    assert "hpcgx error" not in log


@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 24, 16)], ids=lambda d: "x".join(map(str, d)))
def test_reference_driver_accepts_general_layout(tmp_path, dims):
    """The same driver with every level on the general-pattern layout
    (HPCGX_DROPIN_GENERAL=1: greedy colouring from the matrix graph, stored
    columns, the driver's own f2c), as a matrix that is not the stencil would
    take: VALID, every test PASSED, no reference operator used."""
    kv, log = run_driver(tmp_path, *dims, extra_env={"HPCGX_DROPIN_GENERAL": "1"})
    assert kv["Spectral Convergence Tests::Result"] == "PASSED"
    sym = "Departure from Symmetry |x'Ay-y'Ax|/(2*||x||*||A||*||y||)/epsilon"
    assert kv[sym + "::Result"] == "PASSED"
    assert kv["Iteration Count Information::Result"] == "PASSED"
    assert kv["Reproducibility Information::Result"] == "PASSED"
    assert "Final Summary::HPCG result is VALID with a GFLOP/s rating of" in kv
    assert not any(k.startswith("Final Summary::Reference version of") for k in kv)
    assert "hpcgx error" not in log

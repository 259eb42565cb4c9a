"""Host-side logic of bench.py that needs no GPU: the reference's iteration
count used to scale its CPU sample, and the JSON contract's helper models."""
import sys

from conftest import ROOT

sys.path.insert(0, ROOT)


def test_reference_iterations_measured_and_extrapolated():
    import bench
    assert bench.reference_iterations(256) == (128, "measured")
    it, basis = bench.reference_iterations(512)
    # one doubling past the last measurement, at the last measured ratio
    assert it == round(128 * 128 / 71) and "extrapolated" in basis
    it2, _ = bench.reference_iterations(1024)
    assert it2 == round(128 * (128 / 71) ** 2)


def test_flop_model_matches_the_reference_report():
    """src/ReportResults.cpp:81-97's flops per iteration at 32^3 (the reference
    report gives 5.96884e8 for 50 iterations of its own run, preamble and
    reference timing included, so only the order is compared here) and the
    nonzero count of the 27-point stencil."""
    import bench
    flops, b64, b32, n0, nnz0 = bench.model((32, 32, 32))
    assert n0 == 32 ** 3 and nnz0 == 830584
    assert 1.0e7 < flops < 1.3e7 and b32 < b64


def test_committed_traffic_names_the_kernels_the_bench_reports():
    """The bench line's `traffic` comes from the small-case ncu capture committed
    in profiles/roofline_traffic_512.json, looked up by the kernel name the
    bench reports: every per-kernel roofline of the bench must find its entry,
    and each entry must say how it was measured."""
    import json
    import os
    import re
    text = open(os.path.join(ROOT, "bench.py")).read()
    names = re.findall(r'roofline\(PROBE_\w+, "([^"]+)"\)', text)
    assert names
    table = json.load(open(os.path.join(ROOT, "profiles", "roofline_traffic_512.json")))
    for name in names:
        if "all modes" in name:
            continue
        assert name in table, name
        entry = table[name]
        assert entry["dram_bytes_per_launch"] > 0 and entry["passes"] == 1
        assert "ncu" in entry["command"] and "--clock-control none" in entry["command"]


def _reference_arm(extra_env=None, *args):
    import json
    import os
    import subprocess
    env = dict(os.environ)
    env.update(extra_env or {})
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--ref-sample", "24", "--ref-sample-it", "2"] + list(args),
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    return [json.loads(l) for l in lines]


def test_reference_arm_prints_one_contract_line():
    """`bench.py --impl reference` runs the reference's CG_ref (oracle/_ref) on
    the host cores, with no GPU, and prints one JSON line on the same metric,
    unit and direction as the product's arm, its e2e equal to its value with no
    host-device bytes, and a cpu_baseline that says what was sampled."""
    import pytest
    from oracle.oracle import RefProblem, build
    build()
    if not RefProblem.available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    import bench
    lines = _reference_arm({"RANK": "0"}, "--steps", "2", "--warmup", "1", "--grid", "64")
    assert len(lines) == 1
    rec = lines[0]
    assert rec["impl"] == "reference" and rec["metric"] == bench.METRIC
    assert rec["unit"] == "s" and rec["higher_is_better"] is False
    assert rec["steps"] == 2 and rec["warmup"] == 1 and rec["n_gpus"] == 1
    assert rec["value"] > 0 and abs(rec["ms_per_step"] - rec["value"] * 1e3) < 1e-9 * rec["value"] * 1e3
    assert rec["e2e"] == {"value": rec["value"], "unit": "s", "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}
    cb = rec["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == rec["value"] and cb["cores"] >= 1
    assert "24^3" in cb["sample"] and cb["sample_grid"] == [24, 24, 24]
    # 64^3 is a measured iteration count, so nothing about it is extrapolated
    assert cb["extrapolation"]["iterations"] == bench.REF_NATURAL_ITERS[64]
    assert cb["extrapolation"]["iterations_basis"] == "measured"
    assert abs(cb["extrapolation"]["rows_factor"] - (64 / 24) ** 3) < 1e-12
    assert rec["config"]["grid"] == [64, 64, 64]


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun the reference arm runs on rank 0 alone; the other ranks
    print nothing and exit 0."""
    assert _reference_arm({"RANK": "1"}, "--steps", "1", "--warmup", "0") == []


def test_reference_arm_unavailable_line(monkeypatch, capsys):
    """Without the reference build the arm prints its one-line `unavailable`
    record and returns normally."""
    import argparse
    import json
    import bench
    from oracle import oracle as orc
    monkeypatch.setattr(orc.RefProblem, "available", classmethod(lambda cls: False))
    monkeypatch.setenv("RANK", "0")
    args = argparse.Namespace(gpus=1, steps=1, warmup=0, ref_sample=24, ref_sample_it=1)
    bench.run_reference(args, (64, 64, 64))
    out = [l for l in capsys.readouterr().out.splitlines() if l.strip()]
    assert len(out) == 1
    rec = json.loads(out[0])
    assert rec["impl"] == "reference" and "unavailable" in rec


def test_reference_iteration_table_against_the_reference():
    """The measured entries of bench.REF_NATURAL_ITERS that run in seconds
    (32^3, 64^3): CG_ref of the reference build on the bench's system
    (b = A u, u ~ U(-1, 1) seed 1, x0 = 0) to 1e-10 takes that many
    iterations.  The table scales the CPU baseline to the benchmark grid."""
    import numpy as np
    import pytest
    import bench
    from oracle.oracle import Oracle, RefProblem, build
    build()
    if not RefProblem.available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    for n in (32, 64):
        ref = RefProblem(n, n, n)
        try:
            u = Oracle.uniform(bench.SEED_U, ref.rows(0), -1.0, 1.0)
            b = ref.spmv(0, u)
            _, k, nr, nr0, _ = ref.cg(b, np.zeros(ref.rows(0)), 500, bench.TOL)
        finally:
            ref.close()
        assert k == bench.REF_NATURAL_ITERS[n] and nr <= bench.TOL * nr0, (n, k)

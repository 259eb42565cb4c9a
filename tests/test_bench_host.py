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

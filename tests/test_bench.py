"""The bench's host-side logic (no GPU): the iteration counts its CPU arms
scale their timed samples by, and the reference arm's line for a workload
without a converged solve to scale by."""
import json
import os
import subprocess
import sys

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_counts_come_from_the_oracle_fixture_when_it_exists():
    counts, source = bench.iteration_counts("hubbard8")
    with open(os.path.join(ROOT, "tests", "golden", "fp64_hubbard8.json")) as f:
        fixture = json.load(f)
    assert counts["outer_iterations"] == fixture["outer_iterations"]
    assert counts["cg_iterations"] == fixture["cg_iterations"]
    assert "oracle" in source


def test_counts_fall_back_to_the_device_solve():
    if bench.fp64_reference("df20") is not None:
        counts, source = bench.iteration_counts("df20")
        assert "oracle" in source
        return
    counts, source = bench.iteration_counts("df20")
    assert counts == bench.DEVICE_COUNTS["df20"] and "device" in source


def test_no_counts_for_an_unconverged_workload():
    assert bench.iteration_counts("hubbard4x4") == (None, None)


def test_reference_arm_reports_unavailable_without_counts():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "hubbard4x4", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line


def test_cg_traffic_scales_with_iterations():
    per = bench.CG_DRAM_BYTES_PER_ITERATION["df20"]
    # one ncu capture: 14.26 GB over 142 CG iterations and the initial residual
    assert abs(per * 143 - 14.26e9) < 1e6

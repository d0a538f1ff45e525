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


def test_fp64_fixtures_describe_the_bench_problems():
    """Each committed CPU-oracle fixture is a converged solve of the problem
    its workload names: the same primal and dual sizes as the oracle builds
    for it, and errors below the thresholds it was run at."""
    from oracle.maps import OracleProblem
    for name in ("hubbard8", "df20"):
        ref = bench.fp64_reference(name)
        if ref is None:
            continue
        w = bench.WORKLOADS[name]
        kind, ham = bench.hamiltonian(w)
        kw = dict(hubbard=ham) if kind == "hubbard" else dict(h=ham[0], g=ham[1])
        o = OracleProblem(w["nmo"], w["nalpha"], w["nbeta"], w["positivity"], True, True, **kw)
        assert (ref["n_primal"], ref["n_dual"]) == (o.n_primal, o.n_dual), name
        assert ref["converged"] and ref["eps_p"] < 1e-6 and ref["eps_d"] < 1e-6, name
        assert abs(ref["energy"] - ref["dual_energy"]) < 1e-6, name

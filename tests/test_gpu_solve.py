"""Full boundary-point solves on the B200 against the numpy oracle and known answers.

Energies agree with the FP64 oracle to |dE| <= 1e-6 Eh at the same thresholds."""
import numpy as np
import pytest

import hilbert_b200 as hb
from oracle.bpsdp import SDPOptions, run_v2rdm
from oracle.fci import hubbard_fci
from oracle.maps import OracleProblem

pytestmark = pytest.mark.gpu

E_TOL = 1e-6


def hubbard_options(L, U, r=1e-6, e=1e-6, maxiter=100000, muf=500):
    return hb.Options({"HUBBARD_HAMILTONIAN": True, "N_HUBBARD_SITES": L, "N_HUBBARD_SPINS": L,
                       "HUBBARD_T": 1.0, "HUBBARD_U": U, "R_CONVERGENCE": r, "E_CONVERGENCE": e,
                       "MAXITER": maxiter, "MU_UPDATE_FREQUENCY": muf})


def test_two_site_hubbard_exact(cuda_device):
    helper = hb.v2RDMHelper(None, hubbard_options(2, 4.0))
    e = helper.compute_energy()
    assert helper.stats["converged"]
    assert abs(e - (2.0 - np.sqrt(8.0))) <= E_TOL
    assert helper.variables["CURRENT ENERGY"] == e
    assert abs(np.trace(helper.get_opdm()) - 2.0) <= 1e-5


def test_four_site_hubbard_matches_oracle_and_bounds_fci(cuda_device):
    helper = hb.v2RDMHelper(None, hubbard_options(4, 4.0))
    e = helper.compute_energy()
    assert helper.stats["converged"]
    o = OracleProblem(4, 2, 2, "DQG", True, True, hubbard=(1.0, 4.0))
    xo, so = run_v2rdm(o, o.guess("random"), SDPOptions(1e-6, 1e-6, 1e-9, 10000, 100000), 500)
    assert so.is_converged()
    assert abs(e - float(o.c @ xo)) <= E_TOL
    assert e <= hubbard_fci(4, 4, 1.0, 4.0) + E_TOL


def test_external_triplet_matches_oracle(cuda_device):
    n, na, nb = 3, 2, 1
    rng = np.random.default_rng(11)
    h = rng.standard_normal((n, n)); h = 0.5 * (h + h.T)
    b = rng.standard_normal((n, n, 2)) * 0.3
    g = np.einsum("ijq,klq->ijkl", b, b)
    opts = hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": 100000,
                       "MU_UPDATE_FREQUENCY": 500})
    helper = hb.v2RDMHelper(na, nb, n, h.ravel(), g.ravel(), opts)
    e = helper.compute_energy()
    assert helper.stats["converged"]
    o = OracleProblem(n, na, nb, "DQG", True, True, h=h, g=g)
    xo, so = run_v2rdm(o, o.guess("random"), SDPOptions(1e-6, 1e-6, 1e-9, 10000, 100000), 500)
    assert so.is_converged()
    assert abs(e - float(o.c @ xo)) <= E_TOL


def test_host_callback_solver_matches_device_solve(cuda_device):
    """libsdp-shaped solver with host callbacks (hilbert's evaluate_Au / evaluate_ATu).
    Both solves converge to 1e-7 so that their energies agree to 1e-6."""
    o = OracleProblem(4, 2, 2, "DQG", True, True, hubbard=(1.0, 2.0))
    opts = hb.Options({"R_CONVERGENCE": 1e-7, "E_CONVERGENCE": 1e-7, "MAXITER": 100000})
    s = hb.BPSDPSolver(o.n_primal, o.n_dual, opts)
    x = o.guess("random")
    while not s.is_converged() and s.oiter_total() < 100000:
        s.solve(x, o.b, o.c, o.dims, 500, o.Au, o.ATu)
    assert s.is_converged()
    p = hb.V2RDMProblem(4, 2, 2, hubbard_multiplicity=True)
    xd, st = p.solve(o.guess("random"), o.b, o.c, hb.Options({"R_CONVERGENCE": 1e-7,
                                                               "E_CONVERGENCE": 1e-7,
                                                               "MAXITER": 100000,
                                                               "MU_UPDATE_FREQUENCY": 500}))
    assert st["converged"]
    assert abs(float(o.c @ x) - st["energy"]) <= E_TOL
    # state accessors of the libsdp surface
    assert s.get_y().shape == (o.n_dual,) and s.get_z().shape == (o.n_primal,)
    assert s.iiter_total() > 0 and s.get_mu() > 0


def test_monitor_protocol(cuda_device):
    """mu is fixed inside one solve() call of MU_UPDATE_FREQUENCY iterations and
    becomes mu * eps_p / eps_d afterwards (tests/mcpdft/output.ref:495-506)."""
    rows = []
    p = hb.V2RDMProblem(4, 2, 2, hubbard_multiplicity=True)
    opts = hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": 60,
                       "MU_UPDATE_FREQUENCY": 20})
    p.solve(p.guess("RANDOM"), p.b(), p.c_hubbard(1.0, 4.0), opts,
            monitor=lambda pl, oi, ii, ep, ed, mu, erp, erd, d: rows.append((oi, mu, erp, erd)))
    assert [r[0] for r in rows] == list(range(60))
    assert rows[0][1] == pytest.approx(0.1)
    assert all(r[1] == rows[0][1] for r in rows[:20])
    assert rows[20][1] == pytest.approx(rows[19][1] * rows[19][2] / rows[19][3], rel=1e-12)


def test_large_block_trajectory_matches_oracle(cuda_device):
    """100 boundary-point iterations of a 9-site ring (G2aa block of 162 rows, past the
    shared-memory Jacobi limit, so the cluster kernel runs) follow the numpy oracle."""
    from oracle.bpsdp import BPSDPSolver
    n = 9
    o = OracleProblem(n, 4, 4, "DQG", True, True, hubbard=(1.0, 4.0))
    assert max(o.dims) > 160
    so = BPSDPSolver(o.n_primal, o.n_dual, SDPOptions(1e-12, 1e-12, 1e-9, 10000, 100))
    xo = o.guess("random")
    so.solve(xo, o.b, o.c, o.dims, 100, o.Au, o.ATu)
    p = hb.V2RDMProblem(n, 4, 4, hubbard_multiplicity=True)
    opts = hb.Options({"R_CONVERGENCE": 1e-12, "E_CONVERGENCE": 1e-12, "MAXITER": 100,
                       "MU_UPDATE_FREQUENCY": 100})
    xg, st = p.solve(o.guess("random"), o.b, o.c, opts)
    assert st["oiter"] == 100
    assert np.max(np.abs(xg - xo)) <= 1e-6
    assert abs(float(o.c @ xg) - float(o.c @ xo)) <= 1e-7


def test_dqgt2_trajectory_matches_oracle_on_reference_maps(cuda_device):
    """60 boundary-point iterations with the T2 condition (DQGT2, 4-site ring:
    T2aaa/bbb blocks of 88 rows, T2aab/bba of 24) follow the numpy oracle driven
    by hilbert's own compiled maps (t2.cc through oracle/_ref)."""
    from oracle.bpsdp import BPSDPSolver
    from oracle.maps import RefProblem, ref_available
    if not ref_available():
        pytest.skip("oracle/_ref not built")
    n = 4
    r = RefProblem(n, 2, 2, "DQGT2", True, True, hubbard=(1.0, 4.0))
    so = BPSDPSolver(r.n_primal, r.n_dual, SDPOptions(1e-12, 1e-12, 1e-9, 10000, 60))
    xo = r.x0.copy()
    so.solve(xo, r.b, r.c, r.dims, 60, r.Au, r.ATu)
    p = hb.V2RDMProblem(n, 2, 2, "DQGT2", hubbard_multiplicity=True)
    opts = hb.Options({"R_CONVERGENCE": 1e-12, "E_CONVERGENCE": 1e-12, "MAXITER": 60,
                       "MU_UPDATE_FREQUENCY": 100})
    xg, st = p.solve(r.x0, r.b, r.c, opts)
    assert st["oiter"] == 60
    assert np.max(np.abs(xg - xo)) <= 1e-6
    assert abs(float(r.c @ xg) - float(r.c @ xo)) <= 1e-7


def test_dqgt2_energy_between_dqg_and_fci(cuda_device):
    """The T2 condition tightens the DQG lower bound: E(DQG) <= E(DQGT2) <= E(FCI)."""
    e = {}
    for pos in ("DQG", "DQGT2"):
        o = hubbard_options(4, 4.0)
        o.set("POSITIVITY", pos)
        helper = hb.v2RDMHelper(None, o)
        e[pos] = helper.compute_energy()
        assert helper.stats["converged"], pos
    assert e["DQG"] <= e["DQGT2"] + E_TOL
    assert e["DQGT2"] <= hubbard_fci(4, 4, 1.0, 4.0) + E_TOL


def test_t1_tightens_dqg_below_fci(cuda_device):
    """A device solve through the T1 maps (hilbert's t1.cc family) keeps
    E(DQG) <= E(DQGT1) <= E(FCI) on the 4-site ring at U/t = 4."""
    e = {}
    for pos in ("DQG", "DQGT1"):
        o = hubbard_options(4, 4.0)
        o.set("POSITIVITY", pos)
        helper = hb.v2RDMHelper(None, o)
        e[pos] = helper.compute_energy()
        assert helper.stats["converged"], pos
    assert e["DQG"] <= e["DQGT1"] + E_TOL
    assert e["DQGT1"] <= hubbard_fci(4, 4, 1.0, 4.0) + E_TOL


def test_d3_trajectory_matches_oracle_on_reference_maps(cuda_device):
    """60 boundary-point iterations with the D3 condition (DQG+D3, 4-site
    ring) follow the numpy oracle driven by hilbert's own compiled maps
    (d3.cc through oracle/_ref).  (A DQG+D3 solve of this ring does not
    reach 1e-6 within 100,000 outer iterations, on the device as in the
    oracle, which stands at eps_p = eps_d = 1.3e-6 there: the check is on
    the trajectory.)"""
    from oracle.bpsdp import BPSDPSolver
    from oracle.maps import RefProblem, ref_available
    if not ref_available():
        pytest.skip("oracle/_ref not built")
    n = 4
    r = RefProblem(n, 2, 2, "DQG+D3", True, True, hubbard=(1.0, 4.0))
    so = BPSDPSolver(r.n_primal, r.n_dual, SDPOptions(1e-12, 1e-12, 1e-9, 10000, 60))
    xo = r.x0.copy()
    so.solve(xo, r.b, r.c, r.dims, 60, r.Au, r.ATu)
    p = hb.V2RDMProblem(n, 2, 2, "DQG+D3", hubbard_multiplicity=True)
    opts = hb.Options({"R_CONVERGENCE": 1e-12, "E_CONVERGENCE": 1e-12, "MAXITER": 60,
                       "MU_UPDATE_FREQUENCY": 100})
    xg, st = p.solve(r.x0, r.b, r.c, opts)
    assert st["oiter"] == 60
    assert np.max(np.abs(xg - xo)) <= 1e-6
    assert abs(float(r.c @ xg) - float(r.c @ xo)) <= 1e-7


def test_profiling_timers_leave_the_solve_unchanged(cuda_device):
    """Kernel-class events, projection phases and the CG kernel's own phase
    clock: all populated, consistent with each other, and the solve with them
    on is bit-identical to the solve without."""
    opts = hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": 60,
                       "MU_UPDATE_FREQUENCY": 20})
    runs = []
    for on in (0, 2):
        p = hb.V2RDMProblem(6, 3, 3, hubbard_multiplicity=True)
        p.set_profiling(on)
        x, st = p.solve(p.guess("RANDOM"), p.b(), p.c_hubbard(1.0, 4.0), opts)
        runs.append((p, x, st))
    assert np.array_equal(runs[0][1], runs[1][1])
    p = runs[1][0]
    classes, cg, phases = p.profile(), p.cg_profile(), p.projection_profile()
    assert classes["cg_kernel"][1] == 60
    assert all(v >= 0.0 for v in cg.values())
    assert cg["transpose_gather"] > 0.0 and cg["gather_update"] > 0.0
    # barrier-to-barrier phases lie inside the kernels' event-timed span
    assert sum(cg.values()) <= 1.05 * classes["cg_kernel"][0] + 0.5
    assert phases["gemm"][1] > 0


def test_synthetic_runner_prints_one_capped_solve(cuda_device, capsys):
    """python -m hilbert_b200.synthetic: one solve of a small DF active
    space, capped at MAXITER outer iterations, reported as one JSON line."""
    import json

    from hilbert_b200.synthetic import main
    main(["--n", "4", "--naux", "30", "--max-outer", "3"])
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert out["outer_iterations"] == 3 and not out["converged"]
    assert out["cg_iterations"] > 0 and out["kernel_launches"] > 0
    assert np.isfinite(out["energy"])

"""v2RDM-DOCI (hilbert's src/v2rdm_doci) on the CPU: the oracle against the
reference's compiled code and its golden fixture, and the product library's
host-side problem (sizes, b, c, guess, packed A and A^T) against both."""
import itertools
import os
import types

import numpy as np
import pytest

from conftest import ROOT
import hilbert_b200 as hb
from hilbert_b200 import _capi
from oracle.doci import DociOracle, DociRef, ref_available, seniority_zero_ci, symmetric_integrals
from test_host_problem import operator, packed_apply

GOLDEN = os.path.join(ROOT, "tests", "golden", "doci_maps.npz")
POSITIVITIES = ["D", "DQ", "DG", "DQG", "DQGT1", "DQGT2", "DQGT1T2"]
needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


def golden_cases():
    with np.load(GOLDEN) as z:
        names = sorted({k.split("/")[0] for k in z.files})
        return {name: {k.split("/")[1]: z[k] for k in z.files if k.startswith(name + "/")}
                for name in names}


def d3_scaled_rows(n, positivity):
    """Dual rows of the seniority-3 D3 condition (d3.cc:131-145), the one
    family whose A.x the packed rows round differently (a partial sum
    scaled by 1/6 as a whole)."""
    pos, *extras = positivity.split("+")
    if "D3" not in extras:
        return np.zeros(0, np.int64)
    pairs = n * (n - 1) // 2
    start = 3 + 3 * n + n * n
    if pos in ("DQ", "DQG", "DQGT1", "DQGT2", "DQGT1T2"):
        start += pairs + n * n
    if pos in ("DG", "DQG", "DQGT1", "DQGT2", "DQGT1T2"):
        start += 4 * pairs + n * n
    return np.arange(start, start + n * (n - 1))


def assert_Au_matches(got, want, n, positivity, x):
    """Bit-exact except the scaled D3 rows, which hold to a few ulps of their
    terms (6(n-2) + 1 of them, each |1/6 x| or |(N/2 - 2) x|)."""
    rows = d3_scaled_rows(n, positivity)
    other = np.setdiff1d(np.arange(len(want)), rows)
    assert np.array_equal(got[other], want[other])
    if len(rows):
        bound = 8 * n * np.finfo(float).eps * (1.0 + n) * np.abs(x).max()
        assert np.max(np.abs(got[rows] - want[rows])) <= bound


def product(n, na, nb, positivity):
    return hb.DOCIProblem(n, na, nb, positivity)


# ---------------------------------------------------------------- oracle pins
def test_doci_oracle_matches_golden():
    """The C restatement against the fixture made from hilbert's compiled DOCI code."""
    for name, case in golden_cases().items():
        n, na, nb = (int(v) for v in case["meta"])
        pos = str(case["positivity"])
        o = DociOracle(n, na, nb, pos)
        assert np.array_equal(o.dims, case["dims"]), name
        assert np.array_equal(o.b(), case["b"]), name
        assert np.array_equal(o.c(case["h"], case["g"]), case["c"]), name
        assert np.array_equal(o.guess(), case["x0"]), name
        assert np.array_equal(o.Au(case["x"]), case["Ax"]), name
        assert np.array_equal(o.ATu(case["y"]), case["ATy"]), name


@needs_ref
def test_doci_oracle_matches_reference_grid():
    """Every POSITIVITY with and without D3, n = 2..5, open and closed shells."""
    rng = np.random.default_rng(7)
    for pos, d3, n in itertools.product(POSITIVITIES, ["", "+D3"], [2, 3, 4, 5]):
        for na, nb in [(n // 2, n // 2), (min(n, n // 2 + 1), n // 2), (1, 1)]:
            h, g = symmetric_integrals(rng, n)
            r = DociRef(n, na, nb, pos + d3, h=h, g=g)
            o = DociOracle(n, na, nb, pos + d3)
            assert (o.n_primal, o.n_dual) == (r.n_primal, r.n_dual)
            assert np.array_equal(o.dims, r.dims)
            assert np.array_equal(o.b(), r.b) and np.array_equal(o.guess(), r.x0)
            assert np.array_equal(o.c(h, g), r.c)
            x, y = rng.standard_normal(r.n_primal), rng.standard_normal(r.n_dual)
            assert np.array_equal(o.Au(x), r.Au(x)) and np.array_equal(o.ATu(y), r.ATu(y))


# ------------------------------------------------------- product host problem
def test_doci_host_problem_matches_golden():
    for name, case in golden_cases().items():
        n, na, nb = (int(v) for v in case["meta"])
        pos = str(case["positivity"])
        p = product(n, na, nb, pos)
        assert list(p.dims) == list(case["dims"]), name
        assert np.array_equal(p.b(), case["b"]), name
        assert np.array_equal(p.c_external(case["h"], case["g"]), case["c"]), name
        assert np.array_equal(p.guess("RANDOM"), case["x0"]), name
        rp, ent, pal = operator(p, False)
        assert_Au_matches(packed_apply(rp, ent, pal, case["x"]), case["Ax"], n, pos, case["x"])
        rp, ent, pal = operator(p, True)
        assert np.array_equal(packed_apply(rp, ent, pal, case["y"]), case["ATy"]), name
        p.close()


@pytest.mark.parametrize("pos", POSITIVITIES + ["DQG+D3", "DQGT1T2+D3"])
def test_doci_host_problem_matches_oracle(pos):
    rng = np.random.default_rng(11)
    for n in (2, 3, 4, 6):
        na = nb = n // 2
        h, g = symmetric_integrals(rng, n)
        o, p = DociOracle(n, na, nb, pos), product(n, na, nb, pos)
        assert (p.n_primal, p.n_dual) == (o.n_primal, o.n_dual) and list(p.dims) == list(o.dims)
        assert np.array_equal(p.b(), o.b()) and np.array_equal(p.c_external(h, g), o.c(h, g))
        assert np.array_equal(p.guess("RANDOM"), o.guess())
        x, y = rng.standard_normal(o.n_primal), rng.standard_normal(o.n_dual)
        rp, ent, pal = operator(p, False)
        assert len(pal) <= 16
        assert_Au_matches(packed_apply(rp, ent, pal, x), o.Au(x), n, pos, x)
        rp, ent, pal = operator(p, True)
        assert np.array_equal(packed_apply(rp, ent, pal, y), o.ATu(y))
        p.close()


@pytest.mark.parametrize("pos", ["DQGT1T2+D3", "DQG"])
def test_doci_packed_operators_are_adjoint(pos):
    rng = np.random.default_rng(3)
    p = product(5, 2, 2, pos)
    x, y = rng.standard_normal(p.n_primal), rng.standard_normal(p.n_dual)
    rp, ent, pal = operator(p, False)
    ax = packed_apply(rp, ent, pal, x)
    rp, ent, pal = operator(p, True)
    aty = packed_apply(rp, ent, pal, y)
    assert abs(ax @ y - x @ aty) <= 1e-12 * max(1.0, abs(ax @ y))


def test_doci_refusals():
    """What DOCI does not have is an error, not a silent v2RDM answer."""
    with pytest.raises(ValueError):
        hb.DOCIProblem(4, 2, 2, "DQG+E3")
    lib = _capi.load()
    import ctypes
    h = ctypes.c_void_p()
    for code in (3 | _capi.V2B_CONSTRAIN_Q3, 3 | _capi.V2B_CONSTRAIN_D4, 7, -1):
        assert lib.v2b_doci_problem_create(4, 2, 2, code, ctypes.byref(h)) == _capi.V2B_BAD_ARG
    assert lib.v2b_doci_problem_create(1, 1, 1, 3 | _capi.V2B_CONSTRAIN_D3, ctypes.byref(h)) == _capi.V2B_BAD_ARG
    p = product(4, 2, 2, "DQG")
    with pytest.raises(_capi.V2BError):
        p.guess("HF")
    with pytest.raises(_capi.V2BError):
        p.c_hubbard(1.0, 4.0)
    p.close()


def test_doci_layout_packs_like_the_reference():
    """The DOCI spin blocks of v2rdm_layout, packed by hilbert's own v2RDM
    PackSpatialDensity, give what hilbert's DOCI PackSpatialDensity gives
    (the device packing of DOCI runs the v2RDM kernel on that layout)."""
    if not (ref_available() and os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libv2rdm_ref.so"))):
        pytest.skip("oracle/_ref not built")
    from oracle.maps import RefProblem
    rng = np.random.default_rng(23)
    for n, pos in itertools.product([1, 2, 3, 4, 5], ["D", "DQG", "DQGT1T2+D3"]):
        if n < 2 and pos.endswith("D3"):
            continue
        na = max(1, n // 2)
        d = DociRef(n, na, na, pos)
        x = rng.standard_normal(d.n_primal)
        want_d2, want_d1 = d.pack_spatial_density(x)
        p = product(n, na, na, pos)
        layout = p.v2rdm_layout(x)
        r = RefProblem(n, na, na, "D", False, True, h=np.zeros((n, n)), g=np.zeros((n,) * 4))
        full = np.zeros(r.n_primal)
        for block, v in layout.items():
            full[r.offsets[block]:r.offsets[block] + len(v)] = v
        got_d2, got_d1 = r.pack_spatial_density(full)
        assert np.array_equal(got_d2, want_d2) and np.array_equal(got_d1, want_d1), (n, pos)
        p.close()


# --------------------------------------------------------------- oracle solve
def pair_hamiltonian(h, g):
    """One electron pair in seniority zero: <pp'|H|qq'> = d_pq (2 h_pp + (pp|pp)) + (1 - d_pq) (pq|pq)."""
    n = h.shape[0]
    H = np.array([[g[p, q, p, q] for q in range(n)] for p in range(n)])
    H[np.diag_indices(n)] += 2.0 * np.diag(h)
    return H


def oracle_solve(o, h, g, r_conv=1e-7, e_conv=1e-7, maxiter=20000):
    from oracle.bpsdp import SDPOptions, run_v2rdm
    prob = types.SimpleNamespace(n_primal=o.n_primal, n_dual=o.n_dual, b=o.b(), c=o.c(h, g),
                                 dims=[int(d) for d in o.dims], Au=o.Au, ATu=o.ATu)
    opts = SDPOptions(sdp_objective_convergence=e_conv, sdp_error_convergence=r_conv,
                      cg_convergence=1e-10, cg_maxiter=10000, maxiter=maxiter)
    x, solver = run_v2rdm(prob, o.guess(), opts, mu_update_frequency=500)
    return float(prob.c @ x), solver


def test_doci_one_pair_is_exact():
    """For one electron pair the D condition alone is exact: the energy is the
    lowest eigenvalue of the seniority-zero pair Hamiltonian."""
    rng = np.random.default_rng(2)
    h, g = symmetric_integrals(rng, 4)
    e, solver = oracle_solve(DociOracle(4, 1, 1, "D"), h, g)
    assert solver.is_converged()
    exact = np.linalg.eigvalsh(pair_hamiltonian(h, g))[0]
    assert abs(exact - seniority_zero_ci(h, g, 1)) < 1e-12
    assert abs(e - exact) < 1e-6


def df_integrals(n, naux=12, seed=5):
    """h with a spread diagonal, (ij|kl) = sum_Q B_ij^Q B_kl^Q (positive semidefinite)."""
    rng = np.random.default_rng(seed)
    h = 0.1 * rng.standard_normal((n, n))
    h = h + h.T + np.diag(np.linspace(-2.0, 1.0, n))
    B = 0.3 * rng.standard_normal((n, n, naux))
    B = B + B.transpose(1, 0, 2)
    return h, np.einsum("ijq,klq->ijkl", B, B)


def test_doci_relaxations_bound_exact_doci():
    """Each set of conditions is a relaxation of seniority-zero CI, and adding
    Q and G tightens it: E(D) <= E(DQG) <= E(DOCI)."""
    h, g = df_integrals(4)
    exact = seniority_zero_ci(h, g, 2)
    e_d, s_d = oracle_solve(DociOracle(4, 2, 2, "D"), h, g)
    e_dqg, s_dqg = oracle_solve(DociOracle(4, 2, 2, "DQG"), h, g)
    assert s_d.is_converged() and s_dqg.is_converged()
    assert e_d <= e_dqg + 1e-6 and e_dqg <= exact + 1e-6
    assert exact - e_dqg < 0.5   # DQG recovers most of the gap left by D (2.85 Eh here)


def oracle_schedule_solver(n, npair, positivity="DQG", frequency=500, r_conv=1e-5, e_conv=1e-6,
                           maxiter=100000):
    """hilbert's v2RDM-DOCI schedule on the CPU chain (v2rdm_doci_solver.cc:1111-1137):
    one oracle BPSDPSolver whose state (x, y, z, mu) carries over from one
    solve(ORBOPT_FREQUENCY) call to the next while the orbitals change, the
    densities packed by hilbert's compiled DOCI PackSpatialDensity."""
    import torch
    from oracle.bpsdp import BPSDPSolver, SDPOptions
    o = DociOracle(n, npair, npair, positivity)
    ref = DociRef(n, npair, npair, positivity)
    dims = [int(d) for d in o.dims]
    solver = BPSDPSolver(o.n_primal, o.n_dual, SDPOptions(e_conv, r_conv, 1e-9, 10000, maxiter))
    state = {"x": o.guess()}

    def solve(h_act, g_act):
        c = o.c(h_act.cpu().numpy(), g_act.cpu().numpy())
        solver.solve(state["x"], o.b(), c, dims, frequency, o.Au, o.ATu)
        d2p, d1p = ref.pack_spatial_density(state["x"])
        return float(c @ state["x"]), torch.from_numpy(d2p), torch.from_numpy(d1p), solver.is_converged()

    solve.solver = solver
    return solve


def doci_schedule_energy(n=4, npair=2, g_conv=1e-3, e_conv=1e-6):
    """(final energy, rounds, info) of the CPU chain under hilbert's schedule
    on the 4-orbital DF fixture."""
    import torch
    import hilbert_b200.orbital as ho
    h_mo, B_mo, *_ = ho.casscf_df_problem(nbf=n, naux=10, ncore=0, nact=n)
    info = {}
    E, gn, _, _ = ho.doci_casscf(torch.from_numpy(h_mo), torch.from_numpy(B_mo), npair, npair,
                                 solve_active=oracle_schedule_solver(n, npair), macro_iterations=200,
                                 g_conv=g_conv, e_conv=e_conv, info=info)
    return E, gn, info


@needs_ref
def test_doci_orbital_optimisation_on_hilbert_schedule():
    """doci_casscf on the CPU with hilbert's interleaved schedule: the SDP
    state carries over between solve(500) calls while focas steps the
    orbitals (all active, active-active rotations on).  The loop ends once
    the SDP has converged and the orbital step met the thresholds; the energy
    falls from -28.31 to -33.5749 Eh and the orbital gradient below 1e-3."""
    E, gn, info = doci_schedule_energy()
    assert info["sdp_converged"] and info["orbitals_converged"]
    assert info["rounds"] < 40
    assert E[1] < E[0] - 1.0
    assert abs(info["final_energy"] - (-33.57490517)) <= 1e-6
    assert gn[-1] < 1e-3 and gn[-1] < 1e-3 * gn[0]


@needs_ref
def test_doci_rdm_entries_match_the_reference_writer():
    """What v2RDM-DOCI's WriteTPDM writes (D2aa, D2bb, D2ab and their
    metadata), byte for byte; DOCI writes no spin-free D2 and no 1-RDM files."""
    rng = np.random.default_rng(29)
    for n, pos in itertools.product([1, 2, 3, 4, 5], ["D", "DQG+D3"]):
        if n < 2 and pos.endswith("D3"):
            continue
        na = max(1, n // 2)
        r = DociRef(n, na, na, pos)
        x = rng.standard_normal(r.n_primal)
        want = r.write_tpdm(x)
        p = product(n, na, na, pos)
        got = p.rdm_entries(x)
        assert set(got) == {"D2aa", "D2bb", "D2ab"}
        for name, entries in want.items():
            assert got[name] == entries, (n, pos, name)
        p.close()


def test_doci_helper_builds_the_problem_its_options_name():
    """v2RDM_DOCIHelper: POSITIVITY / CONSTRAIN_D3 pick the conditions, c from
    h and (ij|kl) or from the DF factors, ORBOPT_FREQUENCY sets the mu period;
    without a GPU compute_energy fails loudly."""
    rng = np.random.default_rng(8)
    n = 4
    h, g = symmetric_integrals(rng, n)
    helper = hb.v2RDM_DOCIHelper(2, 2, n, h, g, {"POSITIVITY": "DQG", "CONSTRAIN_D3": True,
                                                 "ORBOPT_FREQUENCY": 250})
    o = DociOracle(n, 2, 2, "DQG+D3")
    assert helper.problem.n_primal == o.n_primal
    assert np.array_equal(helper.b, o.b()) and np.array_equal(helper.c, o.c(h, g))
    assert helper._sdp_options().get("MU_UPDATE_FREQUENCY") == 250
    B = 0.3 * rng.standard_normal((6, n, n))
    B = B + B.transpose(0, 2, 1)
    from_b = hb.v2RDM_DOCIHelper(2, 2, n, h, None, {"POSITIVITY": "DQ"}, B=B)
    assert np.allclose(from_b.c, DociOracle(n, 2, 2, "DQ").c(h, np.einsum("Qij,Qkl->ijkl", B, B)))
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        with pytest.raises(_capi.V2BError):
            helper.compute_energy()


@needs_ref
def test_doci_one_orbital_edge_cases():
    """n = 1 (no pairs: Q2s2, G2s2 and the T2 3x3 blocks are empty), zero and
    one pair, against the reference; the oracle and the product agree."""
    rng = np.random.default_rng(13)
    for pos, na in itertools.product(["D", "DQ", "DG", "DQG", "DQGT2"], [0, 1]):
        h, g = symmetric_integrals(rng, 1)
        r = DociRef(1, na, na, pos, h=h, g=g)
        o, p = DociOracle(1, na, na, pos), product(1, na, na, pos)
        assert list(p.dims) == list(r.dims) and np.array_equal(o.dims, r.dims)
        assert np.array_equal(p.b(), r.b) and np.array_equal(o.b(), r.b)
        assert np.array_equal(p.c_external(h, g), r.c) and np.array_equal(o.c(h, g), r.c)
        x, y = rng.standard_normal(r.n_primal), rng.standard_normal(r.n_dual)
        assert np.array_equal(packed_apply(*operator(p, False), x), r.Au(x))
        assert np.array_equal(packed_apply(*operator(p, True), y), r.ATu(y))
        assert np.array_equal(o.Au(x), r.Au(x)) and np.array_equal(o.ATu(y), r.ATu(y))
        p.close()

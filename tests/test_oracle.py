"""The C restatement (oracle) against the reference's golden vectors and,
where oracle/_ref is built, against hilbert's own compiled map code."""
import itertools

import numpy as np
import pytest

from conftest import case_kwargs
from oracle.maps import OracleProblem, RefProblem, ref_available


def same(a, b):
    """equal as float64 values (the sign of a zero is not compared)"""
    return a.shape == b.shape and np.array_equal(a, b)


def test_golden_cases_present(golden):
    assert len(golden) >= 8


@pytest.mark.parametrize("name", ["hub2_dqg", "hub4_dqg", "hub4_d_nospin", "ext3_dqg_triplet",
                                  "ext4_dq_nosz", "ext4_dg_doublet", "ext5_dqg", "ext1_dqg",
                                  "hub3_dqgt2", "ext3_dqgt2_doublet", "hub4_dqgt1",
                                  "ext4_dqgt1t2_doublet", "hub4_dqg_d3", "ext3_d_d3_nosz_doublet",
                                  "ext3_dqg_q3_doublet", "hub3_d_e3", "ext3_d_f3_doublet",
                                  "ext4_d_d4_quartet"])
def test_oracle_matches_golden(golden, name):
    case = golden[name]
    kw = case_kwargs(case)
    o = OracleProblem(**kw)
    assert list(o.dims) == list(case["dims"])
    bas_ab, ibas_ab, bas_aa, ibas_aa = o.tables()
    assert np.array_equal(bas_ab, case["bas_ab"]) and np.array_equal(ibas_ab, case["ibas_ab"])
    assert np.array_equal(bas_aa, case["bas_aa"]) and np.array_equal(ibas_aa, case["ibas_aa"])
    assert same(o.b, case["b"])
    assert same(o.c, case["c"])
    assert same(o.guess("random"), case["x_random"])
    assert same(o.guess("hf"), case["x_hf"])
    # bit-exact maps
    assert same(o.Au(case["x"]), case["Ax"])
    assert same(o.ATu(case["y"]), case["ATy"])


def test_sizes_match_reference_counts():
    # the reference prints n_primal / n_dual only for its molecular (D2h)
    # decks, so the C1 formula is pinned on the sizes of the workloads
    o = OracleProblem(8, 4, 4, "DQG", True, True, hubbard=(1.0, 4.0))
    assert (o.n_primal, o.n_dual) == (40256, 47028)
    o = OracleProblem(20, 10, 10, "DQG", True, True, h=np.zeros((20, 20)), g=np.zeros((20,) * 4))
    assert (o.n_primal, o.n_dual) == (1586000, 1856304)
    assert sorted(set(o.dims)) == [20, 190, 400, 800]
    # tests/v2rdm3 (H3 doublet, POSITIVITY D + CONSTRAIN_D3) prints 623 primal
    # variables (output.ref:363); its C1 formula gives the same
    assert OracleProblem(3, 2, 1, "D+D3", True, True, h=np.zeros((3, 3)), g=np.zeros((3,) * 4)).n_primal == 623
    # the half-filled Hubbard rings of the 64-instance batch, L = 6 .. 14
    for L, sizes, big in ((6, (12708, 14863), 72), (14, (379652, 443895), 392)):
        o = OracleProblem(L, L // 2, L // 2, "DQG", True, True, hubbard=(1.0, 4.0))
        assert (o.n_primal, o.n_dual) == sizes and max(o.dims) == big
    # config 5: the 4x4 Hubbard lattice with T2 (80 M primal variables)
    o = OracleProblem(16, 8, 8, "DQGT2", True, True, hubbard=(1.0, 4.0))
    assert (o.n_primal, o.n_dual) == (80405760, 80515780)
    assert sorted(set(o.dims)) == [16, 120, 256, 512, 1920, 6016]


def test_adjoint_identity():
    rng = np.random.default_rng(7)
    for n, na, nb, pos, spin, sz in [(4, 2, 2, "DQG", 1, 1), (5, 3, 2, "DQG", 1, 0), (3, 1, 1, "DG", 0, 1),
                                     (3, 2, 1, "DQGT2", 1, 1), (4, 2, 2, "DQGT2", 0, 1)]:
        o = OracleProblem(n, na, nb, pos, spin, sz, h=rng.standard_normal((n, n)),
                          g=rng.standard_normal((n,) * 4))
        x = rng.standard_normal(o.n_primal)
        y = rng.standard_normal(o.n_dual)
        lhs = float(o.Au(x) @ y)
        rhs = float(x @ o.ATu(y))
        assert abs(lhs - rhs) <= 1e-11 * max(1.0, abs(lhs))


def test_hf_guess_satisfies_d_constraints():
    # a pure determinant satisfies the trace, D1+Q1=I and partial-trace rows exactly
    o = OracleProblem(6, 3, 3, "DQG", True, True, hubbard=(1.0, 4.0))
    x = o.guess("hf")
    r = o.Au(x) - o.b
    n, gab, gaa = 6, 36, 15
    n_d_rows = 3 + 2 * gaa * gaa + gab * gab + 2 * n * n + 4 * n * n
    assert np.max(np.abs(r[:n_d_rows])) == 0.0


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_oracle_bit_exact_against_reference_grid():
    rng = np.random.default_rng(3)
    for n, na, nb, pos, spin, sz in itertools.product([1, 2, 3, 4], [0, 1, 2], [0, 1, 2],
                                                      ["D", "DQ", "DG", "DQG", "DQGT2", "DQGT1",
                                                       "DQGT1T2", "DQG+D3", "D+D3", "DQG+Q3", "D+E3", "D+F3",
                                                       "DQGT1T2+D3+Q3+E3+F3"], [0, 1], [0, 1]):
        if na > n or nb > n:
            continue
        kw = dict(h=rng.standard_normal((n, n)), g=rng.standard_normal((n,) * 4))
        r = RefProblem(n, na, nb, pos, spin, sz, **kw)
        o = OracleProblem(n, na, nb, pos, spin, sz, **kw)
        assert (r.n_primal, r.n_dual) == (o.n_primal, o.n_dual)
        assert list(r.dims) == list(o.dims)
        assert r.offsets == o.offsets
        x = rng.standard_normal(r.n_primal)
        y = rng.standard_normal(r.n_dual)
        assert same(r.Au(x), o.Au(x)) and same(r.ATu(y), o.ATu(y))
        assert same(r.b, o.b) and same(r.c, o.c)


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("pos", ["DQGT2", "DQGT1", "DQGT1T2", "DQGT1T2+D3", "DQGT2+Q3"])
def test_oracle_triplet_guesses_bit_exact_against_reference_grid(pos):
    """The T1 / T2 parts of the HF guess (t1.cc:45-419, t2.cc:1845-2452) and
    the random guess with those blocks present, against hilbert's compiled code."""
    rng = np.random.default_rng(11)
    for n, na, nb, spin, sz in itertools.product([1, 2, 3, 4], [0, 1, 2], [0, 1, 2], [0, 1], [0, 1]):
        if na > n or nb > n:
            continue
        kw = dict(h=rng.standard_normal((n, n)), g=rng.standard_normal((n,) * 4))
        o = OracleProblem(n, na, nb, pos, spin, sz, **kw)
        for kind in ("random", "hf"):
            r = RefProblem(n, na, nb, pos, spin, sz, guess=kind, **kw)
            assert same(r.x0, o.guess(kind)), (n, na, nb, spin, sz, kind)


def test_t2_blocks_and_rows_follow_the_triplet_counts():
    """T2aaa / T2bbb have n^2 (n - 1) / 2 + n^3 rows, T2aab / T2bba
    n^2 (n - 1) / 2 (v2rdm_solver.cc:3879-3906); the T2 rows are zero in b."""
    n = 4
    o = OracleProblem(n, 2, 2, "DQGT2", True, True, hubbard=(1.0, 4.0))
    d = OracleProblem(n, 2, 2, "DQG", True, True, hubbard=(1.0, 4.0))
    ta, tb = n * n * (n - 1) // 2, n ** 3
    assert list(o.dims[len(d.dims):]) == [ta + tb, ta + tb, ta, ta]
    assert o.n_primal - d.n_primal == 2 * (ta + tb) ** 2 + 2 * ta * ta
    assert o.n_dual - d.n_dual == o.n_primal - d.n_primal
    assert not np.any(o.b[d.n_dual:])


@pytest.mark.parametrize("n", [3, 4])
def test_d3_is_exact_for_three_electrons(n):
    """Known answer (the reference's tests/v2rdm3 deck compares D + D3 with
    FCI for H3): with the 3-RDM positive and contracting to the 2-RDM, three
    electrons reach the full-CI energy of their Ms sector, while D alone lies
    far below it."""
    from oracle.bpsdp import SDPOptions, run_v2rdm
    from oracle.fci import fci_energy
    rng = np.random.default_rng(7)
    h = rng.standard_normal((n, n))
    h = 0.5 * (h + h.T)
    B = rng.standard_normal((6, n, n))
    B = 0.5 * (B + B.transpose(0, 2, 1))
    g = np.einsum("Qij,Qkl->ijkl", B, B)
    e_fci = fci_energy(h, g, 2, 1)
    o = OracleProblem(n, 2, 1, "D+D3", False, True, h=h, g=g)
    x, so = run_v2rdm(o, o.guess("random"), SDPOptions(1e-8, 1e-8, 1e-10, 10000, 200000), 500)
    assert so.is_converged()
    assert abs(float(o.c @ x) - e_fci) <= 1e-6
    o = OracleProblem(n, 2, 1, "D", False, True, h=h, g=g)
    x, so = run_v2rdm(o, o.guess("random"), SDPOptions(1e-8, 1e-8, 1e-10, 10000, 200000), 500)
    assert float(o.c @ x) < e_fci - 1.0


def test_q3_without_q2_and_g2_is_refused():
    """The Q3 rows read Q2 and G2 elements: with POSITIVITY D they would read
    blocks that do not exist, so the combination is refused."""
    with pytest.raises(ValueError):
        OracleProblem(3, 1, 1, "D+Q3", True, True, h=np.eye(3), g=np.zeros((3,) * 4))


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_oracle_d4_bit_exact_against_reference_grid():
    """CONSTRAIN_D4 (d4.cc) with every electron-count gate of its families
    (n = 1..5, nalpha, nbeta = 0..4), and every family of the reference at
    once; the reference's dual count includes the aabb family twice, and so
    does the oracle's (empty trailing rows)."""
    rng = np.random.default_rng(91)
    for pos in ("D+D4", "DQGT1T2+Q3+E3+F3+D4"):
        for n, na, nb, spin, sz in itertools.product([1, 2, 3, 4, 5], range(5), range(5), [0, 1], [0, 1]):
            if na > n or nb > n or (pos != "D+D4" and (n > 4 or spin != sz)):
                continue
            kw = dict(h=rng.standard_normal((n, n)), g=rng.standard_normal((n,) * 4))
            r = RefProblem(n, na, nb, pos, spin, sz, **kw)
            o = OracleProblem(n, na, nb, pos, spin, sz, **kw)
            assert (r.n_primal, r.n_dual) == (o.n_primal, o.n_dual) and list(r.dims) == list(o.dims)
            x, y = rng.standard_normal(r.n_primal), rng.standard_normal(r.n_dual)
            assert same(r.Au(x), o.Au(x)) and same(r.ATu(y), o.ATu(y))


def test_fp32_eigenvectors_with_an_fp64_rayleigh_ritz_step_keep_the_solve():
    """The precision study of the mixed projection at n = 4 (a (4e, 4o)
    synthetic DF problem): FP32 eigenvectors followed by one FP64
    Rayleigh-Ritz step converge in the outer iterations of the FP64
    projection (to 1%) and to its energy within 1e-7 Eh."""
    from oracle.precision_study import run
    a, b = run(4, "fp64"), run(4, "fp32rr")
    assert a["converged"] and b["converged"]
    assert abs(a["outer_iterations"] - b["outer_iterations"]) <= 0.01 * a["outer_iterations"]
    assert abs(a["energy"] - b["energy"]) <= 1e-7


def test_normal_equations_cg_step_keeps_the_solve():
    """The device CG's step length r.r / ||A^T p||^2 (with its extrapolated
    start) against the p.(A A^T p) form on a (4e, 4o) synthetic DF problem:
    the same solution within 1e-8 Eh, in outer iterations within 1%."""
    from hilbert_b200.synthetic import df_hamiltonian
    from oracle.bpsdp import BPSDPSolver, SDPOptions
    h, g = df_hamiltonian(4, 400, 4, 5)
    o = OracleProblem(4, 2, 2, "DQG", True, True, h=h, g=g)
    out = {}
    for step in ("pq", "normal"):
        s = BPSDPSolver(o.n_primal, o.n_dual, SDPOptions(1e-6, 1e-6, 1e-9, 10000, 200000),
                        cg_start="extrapolate", cg_step=step)
        x = o.guess("random")
        while not s.is_converged() and s.oiter_total() < 200000:
            s.solve(x, o.b, o.c, [int(d) for d in o.dims], 500, o.Au, o.ATu)
        assert s.is_converged()
        out[step] = (float(o.c @ x), s.oiter_total(), s.iiter_total())
    (ea, na, _), (eb, nb, _) = out["pq"], out["normal"]
    assert abs(ea - eb) <= 1e-8
    assert abs(na - nb) <= 0.01 * na

"""The product library's host-side problem (sizes, b, c, guesses, packed
operator) through the C ABI, without a GPU, against the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, case_kwargs
import hilbert_b200 as hb
from hilbert_b200 import _capi
from oracle.maps import OracleProblem


def packed_apply(rp, ent, pal, x):
    """Test-side replay of the packed rows: left-to-right sum, second partial for flagged terms."""
    out = np.zeros(len(rp) - 1)
    col = (ent & ((1 << 27) - 1)).astype(np.int64)
    code = ((ent >> 27) & 15).astype(np.int64)
    grp = (ent >> 31).astype(bool)
    for r in range(len(rp) - 1):
        a0 = 0.0
        a1 = 0.0
        g = False
        for k in range(rp[r], rp[r + 1]):
            v = pal[code[k]] * x[col[k]]
            g = g or grp[k]
            if g:
                a1 = a1 + v
            else:
                a0 = a0 + v
        out[r] = a0 + a1 if g else a0
    return out


def operator(prob, transposed):
    lib = prob._lib
    nrows, nnz, npal = ctypes.c_long(), ctypes.c_long(), ctypes.c_int()
    _capi.check(lib.v2b_problem_operator_size(prob._h, int(transposed), ctypes.byref(nrows),
                                              ctypes.byref(nnz), ctypes.byref(npal)))
    rp = np.zeros(nrows.value + 1, np.uint32)
    ent = np.zeros(max(nnz.value, 1), np.uint32)
    pal = np.zeros(max(npal.value, 1))
    _capi.check(lib.v2b_problem_operator(
        prob._h, int(transposed), rp.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
        ent.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
        pal.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return rp.astype(np.int64), ent[:nnz.value], pal


def product_problem(kw):
    return hb.V2RDMProblem(kw["n"], kw["na"], kw["nb"], kw["positivity"], kw["constrain_spin"],
                           kw["constrain_sz"], hubbard_multiplicity="hubbard" in kw)


def test_header_symbols_exported():
    header = open(os.path.join(ROOT, "include", "v2rdm_b200.h")).read()
    declared = set(re.findall(r"\b(v2b_[A-Za-z0-9_]+)\s*\(", header))
    declared -= {"v2b_sdp_callback", "v2b_sdp_monitor"}
    lib = _capi.load()
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(_capi.EXPORTS)


@pytest.mark.parametrize("name", ["hub2_dqg", "hub4_dqg", "hub4_d_nospin", "ext3_dqg_triplet",
                                  "ext4_dq_nosz", "ext4_dg_doublet", "ext1_dqg", "hub3_dqgt2",
                                  "ext3_dqgt2_doublet", "hub4_dqgt1", "ext4_dqgt1t2_doublet",
                                  "hub4_dqg_d3", "ext3_d_d3_nosz_doublet", "ext3_dqg_q3_doublet",
                                  "hub3_d_e3", "ext3_d_f3_doublet", "ext4_d_d4_quartet"])
def test_host_problem_matches_golden(golden, name):
    case = golden[name]
    kw = case_kwargs(case)
    p = product_problem(kw)
    assert list(p.dims) == list(case["dims"])
    assert np.array_equal(p.b(), case["b"])
    if "hubbard" in kw:
        c = p.c_hubbard(*kw["hubbard"])
    else:
        c = p.c_external(kw["h"], kw["g"])
    assert np.array_equal(c, case["c"])
    assert np.array_equal(p.guess("RANDOM"), case["x_random"])
    assert np.array_equal(p.guess("HF"), case["x_hf"])
    rp, ent, pal = operator(p, False)
    assert len(pal) <= 16
    assert np.array_equal(packed_apply(rp, ent, pal, case["x"]), case["Ax"])
    rp, ent, pal = operator(p, True)
    assert np.array_equal(packed_apply(rp, ent, pal, case["y"]), case["ATy"])


def test_layout_helper_matches_library():
    for args in [(4, 2, 2, "DQG", True), (3, 2, 1, "DQG", True), (4, 2, 2, "D", False),
                 (4, 2, 1, "DG", True), (3, 2, 1, "DQGT2", True), (4, 2, 2, "DQGT1", True),
                 (4, 2, 1, "DQGT1T2", True), (3, 1, 1, "DQGT", False), (4, 2, 2, "DQG+D3", True),
                 (3, 2, 1, "D+D3", False), (3, 2, 1, "DQG+Q3", True), (3, 1, 1, "DQGT1+D3+Q3", True),
                 (3, 2, 1, "D+E3", True), (3, 2, 1, "DQGT1T2+Q3+E3+F3", True), (5, 4, 3, "DQG+D4", True),
                 (4, 2, 2, "DQGT1T2+D4", False)]:
        p = hb.V2RDMProblem(args[0], args[1], args[2], args[3], args[4])
        assert [d for _, d in hb.block_layout(*args)] == list(p.dims)


def test_bad_arguments_are_rejected():
    with pytest.raises(hb.V2BError):
        hb.V2RDMProblem(4, 5, 2)
    with pytest.raises(hb.V2BError):
        hb.V2RDMProblem(0, 0, 0)
    with pytest.raises(ValueError):
        hb.V2RDMProblem(4, 2, 2, positivity="3POS")
    with pytest.raises(hb.V2BError):
        hb.V2RDMProblem(3, 1, 1, positivity="D+Q3")   # Q3 reads Q2 and G2


def test_device_calls_fail_loudly_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = hb.V2RDMProblem(2, 1, 1, "DQG", True, True, True)
    x = np.zeros(p.n_primal)
    with pytest.raises(hb.V2BError) as e:
        p.solve(x, p.b(), p.c_hubbard(1.0, 4.0), hb.Options())
    assert e.value.code == _capi.V2B_NO_DEVICE


def test_config5_sizes_match_the_oracle():
    """4x4 Hubbard lattice, DQG + T2: the product's host tables give the
    reference's sizes and block dimensions (T2 blocks of 1920 and 6016 rows)."""
    p = hb.V2RDMProblem(16, 8, 8, "DQGT2", True, True, hubbard_multiplicity=True)
    assert (p.n_primal, p.n_dual) == (80405760, 80515780)
    assert sorted(set(int(d) for d in p.dims)) == [16, 120, 256, 512, 1920, 6016]


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libv2rdm_ref.so")),
                    reason="oracle/_ref not built")
@pytest.mark.parametrize("pos", ["DQGT1T2", "DQG+D3", "DQGT2+Q3", "DQG+E3", "DQGT1T2+D3+Q3+E3+F3",
                                 "DQG+D4"])
def test_triplet_families_bit_exact_against_reference_grid(pos):
    """T1 and T2 together (DQGT1T2), and D3 (CONSTRAIN_D3): sizes, b, c, both
    guesses and the packed A / A^T, against hilbert's compiled code, n = 1..3."""
    import itertools
    from oracle.maps import RefProblem
    rng = np.random.default_rng(31)
    for n, na, nb, spin, sz in itertools.product([1, 2, 3], [0, 1, 2], [0, 1, 2], [0, 1], [0, 1]):
        if na > n or nb > n:
            continue
        h, g = rng.standard_normal((n, n)), rng.standard_normal((n,) * 4)
        r = RefProblem(n, na, nb, pos, spin, sz, h=h, g=g)
        rh = RefProblem(n, na, nb, pos, spin, sz, h=h, g=g, guess="hf")
        p = hb.V2RDMProblem(n, na, nb, pos, bool(spin), bool(sz))
        assert (p.n_primal, p.n_dual) == (r.n_primal, r.n_dual) and list(p.dims) == list(r.dims)
        assert np.array_equal(p.b(), r.b) and np.array_equal(p.c_external(h, g), r.c)
        assert np.array_equal(p.guess("RANDOM"), r.x0) and np.array_equal(p.guess("HF"), rh.x0)
        x, y = rng.standard_normal(r.n_primal), rng.standard_normal(r.n_dual)
        rp, ent, pal = operator(p, False)
        assert np.array_equal(packed_apply(rp, ent, pal, x), r.Au(x))
        rp, ent, pal = operator(p, True)
        assert np.array_equal(packed_apply(rp, ent, pal, y), r.ATu(y))


def test_positivity_bits_are_checked_at_the_abi():
    """v2b_problem_create takes POSITIVITY in the low four bits and the
    CONSTRAIN_D3 / _Q3 / _E3 / _F3 / _D4 flags above; anything else is
    BAD_ARG, and every flag brings the D3 blocks with it."""
    lib = _capi.load()
    h = ctypes.c_void_p()
    assert lib.v2b_problem_create(3, 1, 1, 3 | 512, 1, 1, 0, ctypes.byref(h)) == _capi.V2B_BAD_ARG
    assert lib.v2b_problem_create(3, 1, 1, 7, 1, 1, 0, ctypes.byref(h)) == _capi.V2B_BAD_ARG
    assert lib.v2b_problem_create(3, 1, 1, -1, 1, 1, 0, ctypes.byref(h)) == _capi.V2B_BAD_ARG
    for flag, name in ((_capi.V2B_CONSTRAIN_Q3, "q3"), (_capi.V2B_CONSTRAIN_E3, "e3"),
                       (_capi.V2B_CONSTRAIN_F3, "f3"), (_capi.V2B_CONSTRAIN_D4, "d4")):
        assert lib.v2b_problem_create(4, 2, 2, 3 | flag, 1, 1, 0, ctypes.byref(h)) == _capi.V2B_OK
        names = [b for b, _ in hb.block_layout(4, 2, 2, "DQG+" + name.upper(), True)]
        assert "d3aaa" in names and any(b.startswith(name) for b in names)
        lib.v2b_problem_destroy(h)


@pytest.mark.parametrize("pos,n,na,nb,spin,sz", [
    ("DQGT1T2+D3+Q3+E3+F3+D4", 4, 3, 2, True, True), ("DQG+D4", 5, 4, 4, True, False),
    ("D+E3+F3", 4, 2, 1, False, True), ("DQGT2+Q3", 3, 2, 2, True, True)])
def test_packed_operators_are_adjoint(pos, n, na, nb, spin, sz):
    """<A x, y> = <x, A^T y> for the packed A and A^T the library builds,
    with every constraint family combination it supports."""
    p = hb.V2RDMProblem(n, na, nb, pos, spin, sz)
    rng = np.random.default_rng(n * 10 + na)
    x, y = rng.standard_normal(p.n_primal), rng.standard_normal(p.n_dual)
    rp, ent, pal = operator(p, False)
    ax = packed_apply(rp, ent, pal, x)
    rp, ent, pal = operator(p, True)
    aty = packed_apply(rp, ent, pal, y)
    lhs, rhs = float(ax @ y), float(x @ aty)
    assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs))


def test_helper_options_select_the_constraint_families():
    """hilbert's CONSTRAIN_D3 / _Q3 / _E3 / _F3 / _D4 options reach the problem
    through v2RDMHelper, as set_constraints reads them."""
    n = 4
    h, g = np.eye(n), np.zeros((n,) * 4)
    o = hb.Options({"POSITIVITY": "DQGT1", "CONSTRAIN_Q3": True, "CONSTRAIN_D4": True})
    helper = hb.v2RDMHelper(2, 2, n, h, g, o)
    want = [d for _, d in hb.block_layout(n, 2, 2, "DQGT1+Q3+D4", True)]
    assert list(helper.problem.dims) == want
    names = [b for b, _ in hb.block_layout(n, 2, 2, "DQGT1+Q3+D4", True)]
    assert {"t1aaa", "q3aab", "d3bbb", "d4aabb"} <= set(names) and "e3aaa" not in names


def test_new_entry_points_refuse_bad_arguments():
    """NULL handles, wrong problem kinds and bad values give V2B_BAD_ARG."""
    lib = _capi.load()
    bad = _capi.V2B_BAD_ARG
    out = ctypes.c_void_p()
    counts = np.zeros(6, np.int64)
    size = ctypes.c_long()
    n = ctypes.c_int()
    assert lib.v2b_batch_problem_create(None, 1, ctypes.byref(out)) == bad
    assert lib.v2b_batch_problem_create((ctypes.c_void_p * 1)(None), 1, ctypes.byref(out)) == bad
    assert lib.v2b_problem_rdm_counts(None, 0, counts.ctypes.data) == bad
    assert lib.v2b_problem_palette(None, 0, None, ctypes.byref(n)) == bad
    assert lib.v2b_doci_v2rdm_layout(None, None, None, ctypes.byref(size)) == bad
    p = hb.V2RDMProblem(3, 1, 1, "DQG")
    assert lib.v2b_doci_v2rdm_layout(p._h, None, None, ctypes.byref(size)) == bad   # not DOCI
    y, z = np.zeros(p.n_dual), np.zeros(p.n_primal)
    dp = ctypes.POINTER(ctypes.c_double)
    for mu in (0.0, -1.0, float("nan"), float("inf")):
        assert lib.v2b_problem_set_state(p._h, mu, y.ctypes.data_as(dp), z.ctypes.data_as(dp)) == bad
    assert lib.v2b_problem_set_state(p._h, 0.5, None, z.ctypes.data_as(dp)) == bad
    assert lib.v2b_problem_rdm_records(p._h, 0, None, None, None, None, None, None, None) == bad
    assert lib.v2b_problem_rdm_counts(p._h, -1, counts.ctypes.data) == bad
    p.close()


@pytest.mark.parametrize("kind,n,pos", [("doci", 20, "DQGT1T2+D3"), ("v2rdm", 8, "DQGT1T2+D3+Q3+E3+F3+D4"),
                                        ("v2rdm", 20, "DQG")])
def test_packed_A_and_AT_are_exact_transposes(kind, n, pos):
    """At sizes beyond the reference grid: the (row, column, coefficient)
    triples of A^T, duplicates summed, are exactly those of A transposed
    (both emitters visit the same terms)."""
    import scipy.sparse as sp

    def csr(rp, ent, pal, shape):
        rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
        m = sp.coo_matrix((pal[(ent >> 27) & 15], (rows, (ent & ((1 << 27) - 1)).astype(np.int64))),
                          shape=shape).tocsr()
        m.sum_duplicates()
        m.eliminate_zeros()
        return m

    p = (hb.DOCIProblem(n, n // 2, n // 2, pos) if kind == "doci"
         else hb.V2RDMProblem(n, n // 2, n // 2, pos))
    A = csr(*operator(p, False), (p.n_dual, p.n_primal))
    AT = csr(*operator(p, True), (p.n_primal, p.n_dual))
    diff = A.T.tocsr() - AT
    diff.eliminate_zeros()
    assert diff.nnz == 0
    p.close()


def test_helpers_refuse_other_sdp_solvers():
    """SDP_SOLVER RRSDP is hilbert's other libsdp solver; it is not built, so
    asking for it is an error, not a BPSDP solve."""
    n = 2
    h, g = np.eye(n), np.zeros((n,) * 4)
    with pytest.raises(NotImplementedError):
        hb.v2RDMHelper(1, 1, n, h.ravel(), g.ravel(), {"SDP_SOLVER": "RRSDP"})
    with pytest.raises(NotImplementedError):
        hb.v2RDM_DOCIHelper(1, 1, n, h, g, {"SDP_SOLVER": "RRSDP"})
    with pytest.raises(NotImplementedError):
        hb.v2RDMHelper(1, 1, n, h.ravel(), g.ravel(), {"GPC_CONSTRAINTS": "1RDM"})
    hb.v2RDMHelper(1, 1, n, h.ravel(), g.ravel(), {"SDP_SOLVER": "BPSDP", "GPC_CONSTRAINTS": "NONE"})


def test_helper_refuses_restart_files_as_the_reference_does():
    """RESTART_FROM_CHECKPOINT_FILE is an error for Hubbard and external
    Hamiltonians in hilbert (v2rdm_solver.cc:958-959, 1081-1082)."""
    with pytest.raises(ValueError, match="Hubbard"):
        hb.v2RDMHelper(None, {"HUBBARD_HAMILTONIAN": True, "RESTART_FROM_CHECKPOINT_FILE": "ck"})
    with pytest.raises(ValueError, match="external"):
        hb.v2RDMHelper(1, 1, 2, np.eye(2).ravel(), np.zeros(16), {"RESTART_FROM_CHECKPOINT_FILE": "ck"})


def test_helper_mu_period_follows_the_reference():
    """For Hubbard and external Hamiltonians hilbert solves in calls of
    MU_UPDATE_FREQUENCY iterations even when OPTIMIZE_ORBITALS asks for
    ORBOPT_FREQUENCY (v2rdm_solver.cc:1298-1301); v2RDM-DOCI always uses
    ORBOPT_FREQUENCY (v2rdm_doci_solver.cc:1116)."""
    h, g = np.eye(2).ravel(), np.zeros(16)
    for orbopt in (True, False):
        helper = hb.v2RDMHelper(1, 1, 2, h, g, {"OPTIMIZE_ORBITALS": orbopt, "MU_UPDATE_FREQUENCY": 700})
        assert helper._sdp_options().get("MU_UPDATE_FREQUENCY") == 700
    doci = hb.v2RDM_DOCIHelper(1, 1, 2, np.eye(2), np.zeros((2,) * 4), {"MU_UPDATE_FREQUENCY": 700})
    assert doci._sdp_options().get("MU_UPDATE_FREQUENCY") == 500

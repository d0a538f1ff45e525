"""Orbital side of v2RDM-CASSCF on the host: hilbert's PackSpatialDensity
restated in the oracle and pinned to the reference's compiled function; the
density unpacking, the rotated-orbital energy and its hand-written adjoint
(hilbert_b200.orbital) against the energy of the v2RDM solution, the focas
gradient formulas and central finite differences (step 1e-5)."""
import numpy as np
import pytest
import torch

from hilbert_b200 import orbital as ho
from oracle import orbital as oo
from oracle.bpsdp import SDPOptions, run_v2rdm
from oracle.maps import RefProblem, ref_available

needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
FD_TOL = 1e-6      # dE/dkappa against central differences
FOCAS_TOL = 1e-10  # against the focas gradient formulas


@needs_ref
@pytest.mark.parametrize("n,na,nb", [(2, 1, 1), (3, 2, 1), (4, 2, 2), (5, 3, 2)])
def test_pack_spatial_density_restatement_is_bit_exact(n, na, nb):
    rng = np.random.default_rng(40 + n)
    h = rng.standard_normal((n, n)); h = h + h.T
    g = rng.standard_normal((n, n, n, n))
    r = RefProblem(n, na, nb, "DQG", True, True, h=h, g=g)
    x = rng.standard_normal(r.n_primal)
    d2r, d1r = r.pack_spatial_density(x)
    _, ibas_ab, _, ibas_aa = r.tables()
    off = {k: r.offsets[k] for k in ("d2ab", "d2aa", "d2bb", "d1a", "d1b")}
    d2, d1 = oo.pack_spatial_density(x, n, off, lambda i, j: int(ibas_ab[i, j]),
                                     lambda i, j: int(ibas_aa[i, j]))
    assert np.array_equal(d2, d2r)
    assert np.array_equal(d1, d1r)


@pytest.fixture(scope="module")
def small_casscf():
    """2 core + (4e, 4o) + 2 virtual, synthetic DF integrals, 2000 oracle iterations of the
    active v2RDM (the identities checked hold for any iterate: its D2 blocks are Hermitian
    to the primal error)."""
    if not ref_available():
        pytest.skip("oracle/_ref not built")
    nc, na_, nv = 2, 4, 2
    h_mo, B_mo, h_act, g_act, e_core = ho.casscf_df_problem(nbf=8, naux=12, ncore=nc, nact=na_)
    r = RefProblem(na_, 2, 2, "DQG", True, True, h=h_act, g=g_act)
    x, so = run_v2rdm(r, r.x0, SDPOptions(1e-6, 1e-6, 1e-9, 10000, 2000), 500)
    d2p, d1p = r.pack_spatial_density(x)
    return dict(nc=nc, na=na_, nv=nv, h=h_mo, B=B_mo, e=e_core + float(r.c @ x), d2p=d2p, d1p=d1p)


def test_unpack_and_energy(small_casscf):
    s = small_casscf
    Da, Ga = ho.unpack_densities(torch.from_numpy(s["d2p"]), torch.from_numpy(s["d1p"]), s["na"])
    Dn, Gn = oo.unpack_active(s["d2p"], s["d1p"], s["na"])
    assert np.array_equal(Da.numpy(), Dn)
    assert np.allclose(Ga.numpy(), Gn, rtol=0, atol=1e-15)
    D, G = ho.full_densities(Da, Ga, s["nc"], s["nv"])
    n = s["h"].shape[0]
    E = ho.rotated_energy(torch.zeros((n, n), dtype=torch.float64), torch.from_numpy(s["h"]),
                          torch.from_numpy(s["B"]), D, G)
    assert abs(E.item() - s["e"]) <= 1e-10


def test_adjoint_matches_focas_and_finite_differences(small_casscf):
    s = small_casscf
    nc, na_, nv = s["nc"], s["na"], s["nv"]
    Da, Ga = ho.unpack_densities(torch.from_numpy(s["d2p"]), torch.from_numpy(s["d1p"]), na_)
    D, G = ho.full_densities(Da, Ga, nc, nv)
    h, B = torch.from_numpy(s["h"]), torch.from_numpy(s["B"])
    pairs = ho.rotation_pairs(nc, na_, nv, active_active=True)
    _, g = ho.orbital_gradient(h, B, D, G, pairs)
    gf = oo.focas_gradient(s["h"], s["B"], Da.numpy(), Ga.numpy(), nc, na_, active_active=True)
    for k, pq in enumerate(pairs):
        assert abs(g[k].item() - gf[pq]) <= FOCAS_TOL, pq
    n = nc + na_ + nv
    for K0 in (torch.zeros((n, n), dtype=torch.float64),
               (lambda a: a - a.T)(torch.from_numpy(np.random.default_rng(9).normal(0, 0.1, (n, n))))):
        K = K0.clone().requires_grad_(True)
        (gk,) = torch.autograd.grad(ho.rotated_energy(K, h, B, D, G), K)
        for p, q in pairs:
            dK = torch.zeros((n, n), dtype=torch.float64)
            dK[p, q], dK[q, p] = 1e-5, -1e-5
            fd = (ho.rotated_energy(K0 + dK, h, B, D, G).item()
                  - ho.rotated_energy(K0 - dK, h, B, D, G).item()) / 2e-5
            assert abs(fd - (gk[p, q] - gk[q, p]).item()) <= FD_TOL, (p, q)


def test_orbital_step_lowers_energy_at_fixed_densities(small_casscf):
    s = small_casscf
    nc, na_, nv = s["nc"], s["na"], s["nv"]
    Da, Ga = ho.unpack_densities(torch.from_numpy(s["d2p"]), torch.from_numpy(s["d1p"]), na_)
    D, G = ho.full_densities(Da, Ga, nc, nv)
    h, B = torch.from_numpy(s["h"]), torch.from_numpy(s["B"])
    pairs = ho.rotation_pairs(nc, na_, nv)
    U, e_opt, g0, g1 = ho.optimize_orbitals(h, B, D, G, pairs)
    n = h.shape[0]
    assert torch.allclose(U.T @ U, torch.eye(n, dtype=torch.float64), atol=1e-13)
    assert e_opt < s["e"] - 1e-3 and g0 > 1e-2
    assert g1 <= 1e-3 * g0   # (near-)stationary over the rotation pairs
    # the rotated integrals give the optimised energy at kappa = 0
    e2, _ = ho.orbital_gradient(U.T @ h @ U, U.T @ B @ U, D, G, pairs)
    assert abs(e2.item() - e_opt) <= 1e-10


def test_diagonal_hessian_matches_focas_and_second_differences(small_casscf):
    """focas's exact diagonal Hessian: the product's contraction form against
    the literal restatement of orbopt_hessian.cc (after focas's 2/m rescale
    of the packed d2), and both against central second differences of E."""
    s = small_casscf
    nc, na_, nv = s["nc"], s["na"], s["nv"]
    Da, Ga = ho.unpack_densities(torch.from_numpy(s["d2p"]), torch.from_numpy(s["d1p"]), na_)
    h, B = torch.from_numpy(s["h"]), torch.from_numpy(s["B"])
    pairs = ho.rotation_pairs(nc, na_, nv)
    H = ho.diagonal_hessian(h, B, Da, Ga, nc, na_).numpy()
    Hf = oo.focas_diagonal_hessian(s["h"], s["B"], s["d2p"], s["d1p"], nc, na_)
    Hf = np.array([Hf[pq] for pq in pairs])
    assert np.max(np.abs(H - Hf)) <= 1e-12 * np.max(np.abs(Hf))
    D, G = ho.full_densities(Da, Ga, nc, nv)
    n = h.shape[0]
    E0 = ho.rotated_energy(torch.zeros((n, n), dtype=torch.float64), h, B, D, G).item()
    st = 2e-4
    for k, (p, q) in enumerate(pairs):
        dK = torch.zeros((n, n), dtype=torch.float64)
        dK[p, q], dK[q, p] = st, -st
        fd = (ho.rotated_energy(dK, h, B, D, G).item() - 2.0 * E0
              + ho.rotated_energy(-dK, h, B, D, G).item()) / st ** 2
        assert abs(fd - H[k]) <= 1e-5 * max(1.0, abs(H[k])), (p, q, fd, H[k])


def _check_focas_trajectory(h, B, s, maxiter, g_conv=1e-4, e_conv=1e-8):
    nc, na_ = s["nc"], s["na"]
    Da, Ga = ho.unpack_densities(torch.from_numpy(s["d2p"]), torch.from_numpy(s["d1p"]), na_)
    U, E, hist = ho.optimize_orbitals_focas(torch.from_numpy(h), torch.from_numpy(B), Da, Ga, nc, na_,
                                            maxiter=maxiter, g_conv=g_conv, e_conv=e_conv)
    _, _, Uo, histo = oo.focas_optimize(h, B, s["d2p"], s["d1p"], nc, na_, maxiter=maxiter,
                                        g_conv=g_conv, e_conv=e_conv)
    assert len(hist) == len(histo)
    for a, b in zip(hist, histo):
        assert abs(a[0] - b[0]) <= 1e-9 and a[3] == b[3]   # energies; identical trust factors
    assert np.max(np.abs(U.numpy() - Uo)) <= 1e-9
    return U, E, hist


def test_focas_step_follows_the_oracle_with_rejections(small_casscf):
    """From the fixture's random orbitals (|g| ~ 9): one accepted step, then
    rejected ones (Update_r, Update_kappa), and Restore_last_step at the end
    returns to the accepted point; the product and the restated loop take the
    same path."""
    s = small_casscf
    U, E, hist = _check_focas_trajectory(s["h"], s["B"], s, maxiter=10)
    assert hist[0][1] < 0.0 and any(rec[1] > 0.0 for rec in hist)
    assert abs(E - hist[0][0]) <= 1e-9          # restored to the accepted step
    assert E < s["e"] - 1e-2


def test_focas_step_converges_near_a_minimum(small_casscf):
    """Near stationary orbitals (L-BFGS optimum rotated by ~0.02 rad) the
    accepted focas steps lower the energy and the gradient."""
    s = small_casscf
    nc, na_, nv = s["nc"], s["na"], s["nv"]
    Da, Ga = ho.unpack_densities(torch.from_numpy(s["d2p"]), torch.from_numpy(s["d1p"]), na_)
    D, G = ho.full_densities(Da, Ga, nc, nv)
    h, B = torch.from_numpy(s["h"]), torch.from_numpy(s["B"])
    pairs = ho.rotation_pairs(nc, na_, nv)
    Ul, _, _, _ = ho.optimize_orbitals(h, B, D, G, pairs, max_iter=500, gtol=1e-12)
    theta = torch.from_numpy(np.random.default_rng(3).normal(0.0, 0.02, len(pairs)))
    Up = Ul @ torch.linalg.matrix_exp(ho._pair_kappa(theta, pairs, h.shape[0]))
    h1, B1 = (Up.T @ h @ Up).numpy(), (Up.T @ B @ Up).numpy()
    E1, g1 = ho.orbital_gradient(torch.from_numpy(h1), torch.from_numpy(B1), D, G, pairs)
    U, E, hist = _check_focas_trajectory(h1, B1, s, maxiter=30, g_conv=1e-6, e_conv=1e-12)
    assert E < E1.item()
    assert hist[-1][2] < 0.5 * float(g1.norm())


def test_active_active_hessian_block_and_step_follow_the_oracle(small_casscf):
    """ComputeH_diag_aa (orbopt_hessian.cc:465-827), used with
    ORBOPT_ACTIVE_ACTIVE_ROTATIONS: the contraction form equals the literal
    restatement, and the focas loop with active-active pairs follows the
    oracle's.  (This block is focas's approximation, not the exact second
    derivative, so it is pinned to the restatement alone.)"""
    s = small_casscf
    nc, na_, nv = s["nc"], s["na"], s["nv"]
    Da, Ga = ho.unpack_densities(torch.from_numpy(s["d2p"]), torch.from_numpy(s["d1p"]), na_)
    h, B = torch.from_numpy(s["h"]), torch.from_numpy(s["B"])
    pairs = ho.rotation_pairs(nc, na_, nv, active_active=True)
    H = ho.diagonal_hessian(h, B, Da, Ga, nc, na_, active_active=True).numpy()
    Hf = oo.focas_diagonal_hessian(s["h"], s["B"], s["d2p"], s["d1p"], nc, na_, active_active=True)
    Hf = np.array([Hf[pq] for pq in pairs])
    assert len(H) == len(pairs)
    assert np.max(np.abs(H - Hf)) <= 1e-12 * np.max(np.abs(Hf))
    U, E, hist = ho.optimize_orbitals_focas(h, B, Da, Ga, nc, na_, maxiter=10, active_active=True)
    _, _, Uo, histo = oo.focas_optimize(s["h"], s["B"], s["d2p"], s["d1p"], nc, na_, maxiter=10,
                                        active_active=True)
    assert len(hist) == len(histo)
    assert all(abs(a[0] - b[0]) <= 1e-9 and a[3] == b[3] for a, b in zip(hist, histo))
    assert np.max(np.abs(U.numpy() - Uo)) <= 1e-9


@needs_ref
def test_casscf_macro_iterations_with_the_focas_step():
    """casscf(..., orbital_step="focas") on the CPU with the oracle's active
    solve (hilbert's compiled maps + the numpy BPSDP): the orbital step lowers
    the energy the next SDP solve starts from."""
    nc, na_ = 2, 4
    h_mo, B_mo, *_ = ho.casscf_df_problem(nbf=8, naux=12, ncore=nc, nact=na_)

    def solve_active(h_act, g_act):
        r = RefProblem(na_, 2, 2, "DQG", True, True, h=h_act.numpy(), g=g_act.numpy())
        x, _ = run_v2rdm(r, r.x0, SDPOptions(1e-6, 1e-6, 1e-9, 10000, 2000), 500)
        d2p, d1p = r.pack_spatial_density(x)
        return float(r.c @ x), torch.from_numpy(d2p), torch.from_numpy(d1p)

    E, gn, h1, B1 = ho.casscf(torch.from_numpy(h_mo), torch.from_numpy(B_mo), nc, na_, solve_active,
                              macro_iterations=2, orbital_step="focas")
    assert E[1] < E[0] - 0.5
    n = h_mo.shape[0]
    # the rotated integrals stay those of an orthogonal transformation
    assert abs(float(torch.linalg.eigvalsh(h1).sum()) - float(np.trace(h_mo))) <= 1e-9 * n


def test_eri_factors_reproduce_4_index_integrals():
    """Factors of (pq|rs) give back the integrals, and the DF orbital energy
    on them equals the energy on the original factors."""
    rng = np.random.default_rng(12)
    n, naux = 5, 9
    B = rng.standard_normal((naux, n, n))
    B = torch.from_numpy(0.5 * (B + B.transpose(0, 2, 1)))
    g = torch.einsum("Qpq,Qrs->pqrs", B, B)
    F = ho.eri_factors(g)
    assert F.shape[0] <= n * (n + 1) // 2
    assert torch.allclose(torch.einsum("Qpq,Qrs->pqrs", F, F), g, atol=1e-11)
    h = torch.from_numpy(rng.standard_normal((n, n)))
    h = h + h.T
    D = torch.eye(n, dtype=torch.float64)
    G = torch.einsum("pq,rs->pqrs", D, D).reshape(n * n, n * n)
    K = torch.zeros((n, n), dtype=torch.float64)
    K[0, 1], K[1, 0] = 0.3, -0.3
    e1 = ho.rotated_energy(K, h, B, D, G)
    e2 = ho.rotated_energy(K, h, F, D, G)
    assert abs(float(e1 - e2)) < 1e-10
    with pytest.raises(ValueError):
        ho.eri_factors(-g)


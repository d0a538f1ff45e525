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

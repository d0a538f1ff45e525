"""The orbital step against focas itself: hilbert's C++ orbital optimizer
(src/focas/C_files/*.cc) compiled from the reference sources by
oracle/build_ref.sh and driven through oracle/focas.py.  On the 2 core +
(4e, 4o) + 2 virtual synthetic DF fixture, the product's energy, orbital
gradient and exact diagonal Hessian (in focas's rotation order) equal the
compiled ones to 1e-12 relative, and a full optimize_orbitals call takes the
same path: iteration count, energy change, final gradient norm, and the
transformation matrix (focas stores its transpose)."""
import numpy as np
import pytest
import torch

from hilbert_b200 import orbital as ho
from oracle import focas
from oracle.bpsdp import SDPOptions, run_v2rdm
from oracle.maps import RefProblem, ref_available

pytestmark = pytest.mark.skipif(not (ref_available() and focas.available()),
                                reason="oracle/_ref (reference build) not built")
REL = 1e-12


@pytest.fixture(scope="module")
def fixture():
    nc, na_, nv, naux = 2, 4, 2, 12
    h_mo, B_mo, h_act, g_act, e_core = ho.casscf_df_problem(nbf=8, naux=naux, ncore=nc, nact=na_)
    r = RefProblem(na_, 2, 2, "DQG", True, True, h=h_act, g=g_act)
    x, _ = run_v2rdm(r, r.x0, SDPOptions(1e-6, 1e-6, 1e-9, 10000, 1000), 500)
    d2p, d1p = r.pack_spatial_density(x)
    return dict(nc=nc, na=na_, nv=nv, naux=naux, h=h_mo, B=B_mo, d2p=d2p, d1p=d1p)


def product_side(s, active_active):
    Da, Ga = ho.unpack_densities(torch.from_numpy(s["d2p"]), torch.from_numpy(s["d1p"]), s["na"])
    D, G = ho.full_densities(Da, Ga, s["nc"], s["nv"])
    h, B = torch.from_numpy(s["h"]), torch.from_numpy(s["B"])
    pairs = ho.rotation_pairs(s["nc"], s["na"], s["nv"], active_active)
    E, g = ho.orbital_gradient(h, B, D, G, pairs)
    H = ho.diagonal_hessian(h, B, Da, Ga, s["nc"], s["na"], active_active)
    return float(E), g.numpy(), H.numpy(), (h, B, Da, Ga)


@pytest.mark.parametrize("active_active", [False, True])
def test_gradient_and_diagonal_hessian_equal_compiled_focas(fixture, active_active):
    s = fixture
    f = focas.Focas(s["nc"], s["na"], s["nv"], s["naux"], active_active=active_active)
    E, g, hd, gn = f.gradient_hessian(s["h"], s["B"], s["d2p"], s["d1p"])
    Ep, gp, Hp, _ = product_side(s, active_active)
    assert abs(Ep - E) <= REL * abs(E)
    assert g.shape == gp.shape
    assert np.max(np.abs(gp - g)) <= REL * np.max(np.abs(g))
    assert abs(np.linalg.norm(gp) - gn) <= REL * gn
    if active_active:
        # ComputeH_diag_aa is focas's approximation (Shepard's Eq. B27): the
        # product restates it term by term
        assert np.max(np.abs(Hp - hd)) <= 1e-11 * np.max(np.abs(hd))
    else:
        assert np.max(np.abs(Hp - hd)) <= REL * np.max(np.abs(hd))


@pytest.mark.parametrize("active_active", [False, True])
def test_orbital_step_takes_compiled_focas_path(fixture, active_active):
    s = fixture
    f = focas.Focas(s["nc"], s["na"], s["nv"], s["naux"], active_active=active_active)
    Uf, dEf, gnf, itf = f.optimize(s["h"], s["B"], s["d2p"], s["d1p"])
    E0, _, _, (h, B, Da, Ga) = product_side(s, active_active)
    U, E, hist = ho.optimize_orbitals_focas(h, B, Da, Ga, s["nc"], s["na"], active_active=active_active)
    assert len(hist) == itf
    assert abs((E - E0) - dEf) <= 1e-10
    assert abs(hist[-1][2] - gnf) <= 1e-10 * gnf
    assert np.max(np.abs(U.numpy().T - Uf)) <= 1e-10

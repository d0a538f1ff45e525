"""Orbital side of v2RDM-CASSCF on the B200: hilbert's PackSpatialDensity as a
device kernel, bit-exact against the reference's compiled function, and the
orbital gradient of the synthetic DF CASSCF problem (nbf 40, naux 160, 5 core +
(10e, 10o) active, 25 virtual; 425 rotations) from the device v2RDM solution,
against the focas gradient formulas and central finite differences."""
import numpy as np
import pytest

import hilbert_b200 as hb
from hilbert_b200 import orbital as ho
from oracle import orbital as oo
from oracle.maps import RefProblem, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]


@pytest.mark.parametrize("n,na,nb", [(2, 1, 1), (3, 2, 1), (4, 2, 2), (6, 3, 3), (10, 5, 5)])
def test_pack_kernel_bit_exact(cuda_device, n, na, nb):
    import torch
    rng = np.random.default_rng(70 + n)
    h = rng.standard_normal((n, n)); h = h + h.T
    g = rng.standard_normal((n, n, n, n))
    r = RefProblem(n, na, nb, "DQG", True, True, h=h, g=g)
    x = rng.standard_normal(r.n_primal)
    d2r, d1r = r.pack_spatial_density(x)
    p = hb.V2RDMProblem(n, na, nb)
    d2, d1 = p.pack_spatial_density(torch.from_numpy(x).to(cuda_device))
    assert np.array_equal(d2.cpu().numpy(), d2r)
    assert np.array_equal(d1.cpu().numpy(), d1r)


def test_df_casscf_orbital_gradient(cuda_device):
    import torch
    nc, na_, nv = 5, 10, 25
    h_mo, B_mo, h_act, g_act, e_core = ho.casscf_df_problem(40, 160, nc, na_)
    p = hb.V2RDMProblem(na_, 5, 5)
    b, c = p.b(), p.c_external(h_act, g_act)
    dev = cuda_device
    dx = torch.from_numpy(p.guess("RANDOM")).to(dev)
    opts = hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": 100000,
                       "MU_UPDATE_FREQUENCY": 500})
    st = p.solve_device(dx, torch.from_numpy(b).to(dev), torch.from_numpy(c).to(dev), opts)
    assert st["converged"]
    d2p, d1p = p.pack_spatial_density(dx)
    Da, Ga = ho.unpack_densities(d2p, d1p, na_)
    D, G = ho.full_densities(Da, Ga, nc, nv)
    h, B = torch.from_numpy(h_mo).to(dev), torch.from_numpy(B_mo).to(dev)
    pairs = ho.rotation_pairs(nc, na_, nv)
    assert len(pairs) == 425
    E, g = ho.orbital_gradient(h, B, D, G, pairs)
    assert abs(E.item() - (e_core + float(c @ dx.cpu().numpy()))) <= 1e-9 * max(1.0, abs(E.item()))
    gf = oo.focas_gradient(h_mo, B_mo, Da.cpu().numpy(), Ga.cpu().numpy(), nc, na_)
    g = g.cpu().numpy()
    for k, pq in enumerate(pairs):
        assert abs(g[k] - gf[pq]) <= 1e-9 * max(1.0, abs(gf[pq])), pq
    n = nc + na_ + nv
    for k, (pp, qq) in enumerate(pairs):
        dK = torch.zeros((n, n), dtype=torch.float64, device=dev)
        dK[pp, qq], dK[qq, pp] = 1e-5, -1e-5
        fd = (ho.rotated_energy(dK, h, B, D, G).item() - ho.rotated_energy(-dK, h, B, D, G).item()) / 2e-5
        assert abs(fd - g[k]) <= 1e-6, (pp, qq, fd, g[k])


def test_df_casscf_macro_iterations(cuda_device):
    """v2RDM-CASSCF on the synthetic DF problem: each macro-iteration solves the
    active v2RDM on the device, optimises the orbitals at its densities and
    rotates the integrals; the energy falls and the orbital gradient shrinks."""
    import torch
    nc, na_ = 5, 10
    h_mo, B_mo, *_ = ho.casscf_df_problem(40, 160, nc, na_)
    p = hb.V2RDMProblem(na_, 5, 5)
    b = torch.from_numpy(p.b()).to(cuda_device)
    x0 = torch.from_numpy(p.guess("RANDOM")).to(cuda_device)
    opts = hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": 100000,
                       "MU_UPDATE_FREQUENCY": 500})

    def solve_active(h_act, g_act):
        c = torch.from_numpy(p.c_external(h_act.cpu().numpy(), g_act.cpu().numpy())).to(cuda_device)
        x = x0.clone()
        st = p.solve_device(x, b, c, opts)
        assert st["converged"]
        d2p, d1p = p.pack_spatial_density(x)
        return float(c @ x), d2p, d1p

    E, gn, _, _ = ho.casscf(torch.from_numpy(h_mo).to(cuda_device), torch.from_numpy(B_mo).to(cuda_device),
                            nc, na_, solve_active, macro_iterations=4)
    for a, b_ in zip(E, E[1:]):
        assert b_ <= a + 1e-6
    assert E[-1] < E[0] - 1e-2
    assert gn[-1] < 0.1 * gn[0]


def test_df_casscf_on_hilbert_schedule(cuda_device):
    """v2RDM-CASSCF (config 2: nbf 40, naux 160, 5 core + (10e, 10o)) on
    hilbert's schedule: solve(ORBOPT_FREQUENCY = 500) calls on the device
    that carry x, y, z and mu over while the orbitals change between them
    (v2rdm_solver.cc:1330-1361).  After a few rounds the SDP state is still
    the one solve's (the iteration count only grows by the calls), the
    energy has fallen below the first round's, and the orbital gradient has
    shrunk."""
    import torch
    nc, na_ = 5, 10
    h_mo, B_mo, *_ = ho.casscf_df_problem(40, 160, nc, na_)
    p = hb.V2RDMProblem(na_, 5, 5)
    opts = hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": 100000})
    solve = ho.active_solver(p, opts, frequency=500)
    info = {}
    E, gn, _, _ = ho.casscf(torch.from_numpy(h_mo).to(cuda_device), torch.from_numpy(B_mo).to(cuda_device),
                            nc, na_, solve, macro_iterations=6, info=info)
    assert info["rounds"] == 6 and solve.oiter <= 6 * 500
    assert not solve.exhausted
    assert E[-1] < E[0] - 1e-2
    assert gn[-1] < 0.1 * gn[0]


@pytest.mark.parametrize("n,count", [(40, 160), (13, 7), (80, 3), (1, 2)])
def test_df_transform_kernels_match_torch(cuda_device, n, count):
    """The library's FP64 tensor-core transform B'_Q = U^T B_Q U and its
    adjoint sum_Q (B_Q U M_Q^T + B_Q^T U M_Q) against torch's FP64 GEMMs, to
    1e-13 relative (the products differ only in summation order)."""
    import torch
    g = torch.Generator().manual_seed(n * 1000 + count)
    U = torch.linalg.qr(torch.randn(n, n, generator=g, dtype=torch.float64))[0].to(cuda_device)
    B = torch.randn(count, n, n, generator=g, dtype=torch.float64).to(cuda_device)
    M = torch.randn(count, n, n, generator=g, dtype=torch.float64).to(cuda_device)
    Bp = ho.df_transform(U, B)
    ref = U.T @ B @ U
    assert torch.allclose(Bp, ref, rtol=0, atol=1e-13 * float(ref.abs().max()))
    dU = ho.df_transform_adjoint(U, B, M)
    ref = (B @ U @ M.transpose(1, 2)).sum(0) + (B.transpose(1, 2) @ U @ M).sum(0)
    assert torch.allclose(dU, ref, rtol=0, atol=1e-13 * float(ref.abs().max()) * count)


def test_df_transform_rejects_too_many_orbitals(cuda_device):
    import torch
    from hilbert_b200 import _capi
    U = torch.eye(81, dtype=torch.float64, device=cuda_device)
    with pytest.raises(_capi.V2BError) as e:
        ho.df_transform(U, U.unsqueeze(0))
    assert e.value.code == _capi.V2B_BAD_ARG and "at most 80" in str(e.value)

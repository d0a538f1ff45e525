"""v2RDM-DOCI on the B200: the device maps against the fixture made from
hilbert's compiled DOCI code, and device solves against the exact one-pair
answer and the numpy oracle (|dE| <= 1e-6)."""
import numpy as np
import pytest

import hilbert_b200 as hb
from oracle.doci import DociOracle, seniority_zero_ci, symmetric_integrals
from test_doci import (assert_Au_matches, df_integrals, doci_schedule_energy, golden_cases, oracle_solve,
                       pair_hamiltonian)

pytestmark = pytest.mark.gpu

E_TOL = 1e-6


@pytest.mark.parametrize("name", sorted(golden_cases()))
def test_doci_device_maps_golden(cuda_device, name):
    import torch
    case = golden_cases()[name]
    n, na, nb = (int(v) for v in case["meta"])
    pos = str(case["positivity"])
    p = hb.DOCIProblem(n, na, nb, pos)
    x = torch.from_numpy(case["x"]).to(cuda_device)
    y = torch.from_numpy(case["y"]).to(cuda_device)
    assert_Au_matches(p.Au(x).cpu().numpy(), case["Ax"], n, pos, case["x"])
    assert np.array_equal(p.ATu(y).cpu().numpy(), case["ATy"])
    d2, d1 = p.pack_spatial_density(x)
    assert np.array_equal(d2.cpu().numpy(), case["pd2"]) and np.array_equal(d1.cpu().numpy(), case["pd1"])
    p.close()


def device_solve(p, h, g, r=1e-7, e=1e-7):
    import torch
    dev = torch.device("cuda", 0)
    b, c = p.b(), p.c_external(h, g)
    x = torch.from_numpy(p.guess("RANDOM")).to(dev)
    opts = hb.Options({"R_CONVERGENCE": r, "E_CONVERGENCE": e, "MAXITER": 200000,
                       "MU_UPDATE_FREQUENCY": 500})
    st = p.solve_device(x, torch.from_numpy(b).to(dev), torch.from_numpy(c).to(dev), opts)
    return float(c @ x.cpu().numpy()), st


def test_doci_device_one_pair_is_exact(cuda_device):
    rng = np.random.default_rng(2)
    h, g = symmetric_integrals(rng, 4)
    p = hb.DOCIProblem(4, 1, 1, "D")
    e, st = device_solve(p, h, g)
    p.close()
    assert st["converged"]
    assert abs(e - np.linalg.eigvalsh(pair_hamiltonian(h, g))[0]) <= E_TOL


@pytest.mark.parametrize("pos", ["DQG", "DQGT1T2+D3"])
def test_doci_device_solve_matches_oracle(cuda_device, pos):
    """Six orbitals, three pairs, seeded density-fitted integrals."""
    n = 6
    h, g = df_integrals(n)
    p = hb.DOCIProblem(n, 3, 3, pos)
    e, st = device_solve(p, h, g)
    p.close()
    assert st["converged"]
    eo, so = oracle_solve(DociOracle(n, 3, 3, pos), h, g)
    assert so.is_converged()
    assert abs(e - eo) <= E_TOL
    assert e <= seniority_zero_ci(h, g, 3) + E_TOL


def test_doci_casscf_on_the_device(cuda_device):
    """doci_casscf with the device DOCI solve and packing follows the CPU
    chain (oracle solve, hilbert's compiled DOCI packing) of test_doci."""
    import torch
    import hilbert_b200.orbital as ho
    n, npair = 4, 2
    h_mo, B_mo, *_ = ho.casscf_df_problem(nbf=n, naux=10, ncore=0, nact=n)
    E, gn, _, _ = ho.doci_casscf(torch.from_numpy(h_mo).to(cuda_device), torch.from_numpy(B_mo).to(cuda_device),
                                 npair, npair, macro_iterations=3)
    assert all(b <= a + 1e-6 for a, b in zip(E, E[1:]))
    assert abs(E[0] - (-28.3102401)) <= 1e-5 and abs(E[2] - (-33.5748761)) <= 1e-4
    assert gn[2] < 0.01 * gn[0]


# options of hilbert's v2RDM-DOCI deck (tests/v2rdm_doci/input.dat: MAXITER
# 100000, ORBOPT_FREQUENCY 500) with thresholds a small fixture reaches in
# a few tens of rounds
ORBITAL_OPTS = {"POSITIVITY": "DQG", "OPTIMIZE_ORBITALS": True, "MAXITER": 100000,
                "ORBOPT_FREQUENCY": 500, "R_CONVERGENCE": 1e-5, "E_CONVERGENCE": 1e-6,
                "ORBOPT_GRADIENT_CONVERGENCE": 1e-3, "ORBOPT_ENERGY_CONVERGENCE": 1e-6}


def test_doci_helper_energy(cuda_device):
    """v2RDM_DOCIHelper with fixed orbitals gives the oracle's DOCI energy."""
    import hilbert_b200.orbital as ho
    n, npair = 4, 2
    h_mo, B_mo, *_ = ho.casscf_df_problem(nbf=n, naux=10, ncore=0, nact=n)
    g = np.einsum("Qij,Qkl->ijkl", B_mo, B_mo)
    opts = {"POSITIVITY": "DQG", "OPTIMIZE_ORBITALS": False, "R_CONVERGENCE": 1e-7,
            "E_CONVERGENCE": 1e-7, "MAXITER": 200000}
    helper = hb.v2RDM_DOCIHelper(npair, npair, n, h_mo, g, opts)
    e = helper.compute_energy()
    eo, so = oracle_solve(DociOracle(n, npair, npair, "DQG"), h_mo, g)
    assert so.is_converged() and abs(e - eo) <= E_TOL
    assert helper.variables["v2RDM-DOCI TOTAL ENERGY"] == e
    assert abs(helper.occupations.sum() - 2 * npair) <= 1e-5


def test_doci_helper_follows_hilbert_schedule(cuda_device):
    """With OPTIMIZE_ORBITALS the helper runs hilbert's loop on the device:
    solve(ORBOPT_FREQUENCY) calls that continue the SDP state, each followed
    by a focas orbital step, until both have converged.  The energy is the
    CPU chain's under the same schedule (oracle BPSDP + hilbert's compiled
    DOCI packing) to 5e-5 Eh: the two stop after different rounds of a
    slowly converging orbital loop (the stopping energies of the thresholds
    1e-3 and 1e-4 differ by 5e-6 Eh on this fixture)."""
    n, npair = 4, 2
    import hilbert_b200.orbital as ho
    h_mo, B_mo, *_ = ho.casscf_df_problem(nbf=n, naux=10, ncore=0, nact=n)
    helper = hb.v2RDM_DOCIHelper(npair, npair, n, h_mo, None, ORBITAL_OPTS, B=B_mo)
    e = helper.compute_energy(macro_iterations=400)
    st = helper.stats
    assert st["converged"] and st["sdp_converged"] and st["orbitals_converged"]
    assert st["rounds"] < 100
    assert st["energies"][0] > st["energies"][-1] + 1.0
    _, _, info = doci_schedule_energy()
    assert abs(e - info["final_energy"]) <= 5e-5
    assert helper.variables["v2RDM-DOCI TOTAL ENERGY"] == e


def test_doci_helper_optimises_orbitals_from_4_index_integrals(cuda_device):
    """Given (ij|kl) alone, the helper factors it exactly and optimises the
    orbitals: the same energies as from the DF factors themselves."""
    import hilbert_b200.orbital as ho
    n, npair = 4, 2
    h_mo, B_mo, *_ = ho.casscf_df_problem(nbf=n, naux=10, ncore=0, nact=n)
    g = np.einsum("Qij,Qkl->ijkl", B_mo, B_mo)
    h_g = hb.v2RDM_DOCIHelper(npair, npair, n, h_mo, g, ORBITAL_OPTS)
    e_g = h_g.compute_energy(macro_iterations=400)
    h_b = hb.v2RDM_DOCIHelper(npair, npair, n, h_mo, None, ORBITAL_OPTS, B=B_mo)
    e_b = h_b.compute_energy(macro_iterations=400)
    assert h_g.stats["converged"] and h_b.stats["converged"]
    # both loops stop at R_CONVERGENCE = 1e-5 on their own rounding paths:
    # the energies agree to that tolerance's scale, as with the oracle above
    assert abs(e_g - e_b) <= 5e-5


def test_doci_torch_ops_and_their_adjoint(cuda_device):
    """torch.ops.v2rdm.doci_Au equals the device map, and autograd through it
    gives doci_ATu (d<A x, w>/dx = A^T w)."""
    import torch
    import hilbert_b200.torch_ops  # noqa: F401  (registers the operators)
    spec = (4, 2, 2, "DQG+D3")
    p = hb.DOCIProblem(*spec)
    rng = np.random.default_rng(9)
    x = torch.from_numpy(rng.standard_normal(p.n_primal)).to(cuda_device).requires_grad_(True)
    w = torch.from_numpy(rng.standard_normal(p.n_dual)).to(cuda_device)
    ax = torch.ops.v2rdm.doci_Au(x, *spec)
    assert torch.equal(ax.detach(), p.Au(x.detach()))
    (ax * w).sum().backward()
    assert torch.equal(x.grad, p.ATu(w))
    p.close()

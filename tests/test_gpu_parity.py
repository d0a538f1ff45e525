"""Solver parity at the benchmark sizes: the device solve to convergence
against the CPU oracle's FP64 solve of the same workload (hilbert's compiled
maps driven by the numpy boundary-point restatement; fixtures made by
tests/golden/make_fp64_energies.py), |dE| <= 1e-6 Eh, both at
R_CONVERGENCE = E_CONVERGENCE = 1e-6, with the device's primal and dual
errors below the threshold (the device solve's own convergence test)."""
import json
import os

import pytest

import hilbert_b200 as hb
from conftest import ROOT

pytestmark = pytest.mark.gpu

E_TOL = 1e-6


def fixture(name):
    path = os.path.join(ROOT, "tests", "golden", f"fp64_{name}.json")
    if not os.path.exists(path):
        pytest.skip(f"no FP64 CPU solve fixture {path}")
    with open(path) as f:
        return json.load(f)


def device_solve(p, b, c, cuda_device):
    import torch
    opts = hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "CG_CONVERGENCE": 1e-9,
                       "MAXITER": 400000, "MU_UPDATE_FREQUENCY": 500})
    x = torch.from_numpy(p.guess("RANDOM")).to(cuda_device)
    st = p.solve_device(x, torch.from_numpy(b).to(cuda_device), torch.from_numpy(c).to(cuda_device), opts)
    return float(c @ x.cpu().numpy()), st


def test_hubbard8_matches_the_cpu_oracle(cuda_device):
    """Config 1: the 8-site periodic Hubbard ring, 8 electrons, t = 1, U = 4."""
    ref = fixture("hubbard8")
    assert ref["converged"]
    p = hb.V2RDMProblem(8, 4, 4, "DQG", hubbard_multiplicity=True)
    b, c = p.b(), p.c_hubbard(1.0, 4.0)
    e, st = device_solve(p, b, c, cuda_device)
    assert st["converged"]
    assert abs(e - ref["energy"]) <= E_TOL, (e, ref["energy"])


def test_df20_matches_the_cpu_oracle(cuda_device):
    """Config 4: (20e, 20o) on the synthetic density-fitted integrals."""
    from hilbert_b200.synthetic import df_hamiltonian
    ref = fixture("df20")
    assert ref["converged"]
    p = hb.V2RDMProblem(20, 10, 10, "DQG")
    b, c = p.b(), p.c_external(*df_hamiltonian(20, 400, 4, 5))
    e, st = device_solve(p, b, c, cuda_device)
    assert st["converged"]
    assert abs(e - ref["energy"]) <= E_TOL, (e, ref["energy"])

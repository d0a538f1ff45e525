"""Checkpoint and restart of a device solve (WriteCheckpointFile /
ReadFromCheckpointFile, checkpoint.cc:48-124): a solve stopped early,
checkpointed and resumed in a new problem ends at the uninterrupted energy."""
import os

import numpy as np
import pytest

import hilbert_b200 as hb
from hilbert_b200 import checkpoint as ck

pytestmark = pytest.mark.gpu


def ring(n=6):
    p = hb.V2RDMProblem(n, n // 2, n // 2, "DQG", True, True, hubbard_multiplicity=True)
    return p, p.b(), p.c_hubbard(1.0, 4.0)


def solve(p, x, b, c, maxiter):
    import torch
    dev = torch.device("cuda", 0)
    xd = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    opts = hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": maxiter,
                       "MU_UPDATE_FREQUENCY": 500})
    st = p.solve_device(xd, torch.from_numpy(b).to(dev), torch.from_numpy(c).to(dev), opts)
    return xd, st


def test_restart_reaches_the_uninterrupted_energy(cuda_device, tmp_path):
    p, b, c = ring()
    x_full, st_full = solve(p, p.guess("RANDOM"), b, c, 100000)
    assert st_full["converged"]
    e_full = float(c @ x_full.cpu().numpy())

    x_part, st_part = solve(p, p.guess("RANDOM"), b, c, 2000)
    assert not st_part["converged"]
    path = os.path.join(tmp_path, "ring6.ck.npz")
    ck.write_checkpoint(path, p, x_part)
    saved = ck.load_checkpoint(path)
    assert saved["MU"] == p.get_mu() != 0.1
    p.close()

    q, _, _ = ring()
    x0 = ck.restart(q, path)
    x_rest, st_rest = solve(q, x0, b, c, 100000)
    assert st_rest["converged"]
    assert abs(float(c @ x_rest.cpu().numpy()) - e_full) <= 1e-6
    # the restart continues rather than starting over
    assert st_rest["oiter"] < st_full["oiter"]
    q.close()


def test_helper_writes_the_checkpoint_entries(cuda_device):
    """WRITE_CHECKPOINT_FILE: the helper leaves MU, PRIMAL, DUAL 1 and DUAL 2
    of its solve (v2rdm_solver.cc:1514-1516)."""
    opts = {"HUBBARD_HAMILTONIAN": True, "N_HUBBARD_SITES": 4, "N_HUBBARD_SPINS": 4, "HUBBARD_U": 4.0,
            "R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": 100000, "MU_UPDATE_FREQUENCY": 500,
            "WRITE_CHECKPOINT_FILE": True}
    helper = hb.v2RDMHelper(None, opts)
    helper.compute_energy()
    ck_entries = helper.files["CHECKPOINT"]
    assert set(ck_entries) == {"MU", "PRIMAL", "DUAL 1", "DUAL 2"}
    assert np.frombuffer(ck_entries["PRIMAL"], np.float64).tolist() == helper.x.tolist()
    assert np.frombuffer(ck_entries["MU"], np.float64)[0] == helper.problem.get_mu()
    assert len(np.frombuffer(ck_entries["DUAL 1"], np.float64)) == helper.problem.n_dual

"""Checkpoint files (the entries of hilbert's WriteCheckpointFile) and the
restart state of a device problem, on the CPU."""
import os

import numpy as np
import pytest

import hilbert_b200 as hb
from hilbert_b200 import checkpoint as ck


def test_checkpoint_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    x, y, z, U = rng.standard_normal(7), rng.standard_normal(5), rng.standard_normal(7), rng.standard_normal((3, 3))
    path = os.path.join(tmp_path, "v2rdm.ck.npz")
    ck.save_checkpoint(path, 14.719, x, y, z, mo_to_mo=U)
    got = ck.load_checkpoint(path)
    assert set(got) == {"MU", "PRIMAL", "DUAL 1", "DUAL 2", "MO TO MO' TRANSFORMATION MATRIX"}
    assert got["MU"] == 14.719
    for key, want in (("PRIMAL", x), ("DUAL 1", y), ("DUAL 2", z), ("MO TO MO' TRANSFORMATION MATRIX", U)):
        assert np.array_equal(got[key], want)


def test_restart_checks_sizes_and_mu(tmp_path):
    """set_state keeps a host copy until the next solve: its checks need no GPU."""
    p = hb.V2RDMProblem(3, 1, 1, "DQG")
    path = os.path.join(tmp_path, "ck.npz")
    ck.save_checkpoint(path, 0.5, np.zeros(p.n_primal), np.zeros(p.n_dual), np.zeros(p.n_primal))
    x = ck.restart(p, path)
    assert x.shape == (p.n_primal,) and p.get_mu() == 0.5
    ck.save_checkpoint(path, 0.5, np.zeros(p.n_primal + 1), np.zeros(p.n_dual), np.zeros(p.n_primal))
    with pytest.raises(ValueError):
        ck.restart(p, path)
    with pytest.raises(ValueError):
        p.set_state(0.5, np.zeros(p.n_dual - 1), np.zeros(p.n_primal))
    with pytest.raises(hb.V2BError):
        p.set_state(0.0, np.zeros(p.n_dual), np.zeros(p.n_primal))
    p.close()


def test_doci_restart_uses_the_same_entries(tmp_path):
    p = hb.DOCIProblem(4, 2, 2, "DQG")
    path = os.path.join(tmp_path, "doci.ck.npz")
    rng = np.random.default_rng(3)
    x = rng.standard_normal(p.n_primal)
    ck.save_checkpoint(path, 2.5, x, rng.standard_normal(p.n_dual), rng.standard_normal(p.n_primal))
    assert np.array_equal(ck.restart(p, path), x) and p.get_mu() == 2.5
    p.close()

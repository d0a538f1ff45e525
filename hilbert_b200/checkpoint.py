"""Checkpoint and restart of a device v2RDM solve.

The file holds the entries hilbert's WriteCheckpointFile writes
(src/v2rdm_casscf/checkpoint.cc:48-88), with the same names and contents:
"MU" (the penalty after the last solve), "PRIMAL" (x), "DUAL 1" (y),
"DUAL 2" (z) and, for an orbital-optimised run, "MO TO MO' TRANSFORMATION
MATRIX" and "SO TO MO TRANSFORMATION MATRIX".  v2RDM-DOCI writes the same
entries (src/v2rdm_doci/checkpoint.cc:48-86), so a DOCIProblem restarts the
same way.  The container is one .npz
archive (the reference's is a Psi4 PSIO file).  A restart is
ReadFromCheckpointFile (checkpoint.cc:90-124): mu, y and z seed the next
solve, and x is its starting point.
"""
import numpy as np

MU, PRIMAL, DUAL_Y, DUAL_Z = "MU", "PRIMAL", "DUAL 1", "DUAL 2"
MO_TO_MO = "MO TO MO' TRANSFORMATION MATRIX"
SO_TO_MO = "SO TO MO TRANSFORMATION MATRIX"


def save_checkpoint(path, mu, x, y, z, mo_to_mo=None, so_to_mo=None):
    entries = {MU: np.float64(mu), PRIMAL: np.asarray(x, np.float64),
               DUAL_Y: np.asarray(y, np.float64), DUAL_Z: np.asarray(z, np.float64)}
    if mo_to_mo is not None:
        entries[MO_TO_MO] = np.asarray(mo_to_mo, np.float64)
    if so_to_mo is not None:
        entries[SO_TO_MO] = np.asarray(so_to_mo, np.float64)
    with open(path, "wb") as f:
        np.savez(f, **entries)


def load_checkpoint(path):
    """{entry: array}; "MU" as a float."""
    with np.load(path) as z:
        out = {k: z[k] for k in z.files}
    out[MU] = float(out[MU])
    return out


def write_checkpoint(path, problem, x, mo_to_mo=None, so_to_mo=None):
    """After a device solve of `problem` that left x (host or CUDA): its mu,
    x, y and z."""
    xh = x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)
    save_checkpoint(path, problem.get_mu(), xh, problem.get_y(), problem.get_z(), mo_to_mo, so_to_mo)


def restart(problem, path):
    """Seeds the next solve of `problem` with the checkpoint's mu, y and z
    and returns its x (host array) to start that solve from."""
    ck = load_checkpoint(path)
    if ck[PRIMAL].shape != (problem.n_primal,):
        raise ValueError(f"checkpoint holds {ck[PRIMAL].size} primal values, the problem {problem.n_primal}")
    problem.set_state(ck[MU], ck[DUAL_Y], ck[DUAL_Z])
    return ck[PRIMAL].copy()

"""Generate tests/golden/fp64_<workload>.json: the CPU oracle's converged FP64
solve of a benchmark workload, the reference energy the device solves are
compared with.

The oracle here is hilbert's own constraint maps compiled from its sources
(oracle/_ref/libv2rdm_ref.so, built by oracle/build_ref.sh with OpenMP) driven
by the numpy boundary-point restatement (oracle/bpsdp.py, LAPACK eigh per
block), with the benchmark's options: R_CONVERGENCE = E_CONVERGENCE = 1e-6,
CG_CONVERGENCE = 1e-9, MU_UPDATE_FREQUENCY = 500, from the reference's random
guess (srand(0), v2rdm_solver.cc:1799-1806).  hilbert's outer protocol for
Hubbard and external Hamiltonians (v2rdm_solver.cc:1296-1361): solve() calls
of MU_UPDATE_FREQUENCY iterations until converged.

Workloads (the same definitions as bench.py):
  hubbard8  1D periodic Hubbard ring, 8 sites, 8 electrons, t = 1, U = 4
  df20      (20e, 20o) synthetic density-fitted integrals (naux 400, seeds 4, 5)

The df20 solve takes hours (5.4 h on 7 threads for the committed fixture,
with the extrapolated CG start).  --state PATH saves the iteration state
(x, y, z, mu, counters) after every solve() call and resumes from it.  Run
from the repository root:

    OMP_NUM_THREADS=8 python tests/golden/make_fp64_energies.py hubbard8
    OMP_NUM_THREADS=8 python tests/golden/make_fp64_energies.py df20 --state /tmp/df20.npz \
        --cg-start extrapolate
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import maps  # noqa: E402
from oracle.bpsdp import BPSDPSolver, SDPOptions  # noqa: E402

WORKLOADS = {
    "hubbard8": dict(nmo=8, nalpha=4, nbeta=4, hubbard=(1.0, 4.0)),
    "df20": dict(nmo=20, nalpha=10, nbeta=10, df=dict(n=20, naux=400, seed_b=4, seed_h=5)),
}
MUF = 500


def problem(w):
    if "hubbard" in w:
        return maps.RefProblem(w["nmo"], w["nalpha"], w["nbeta"], "DQG", True, True, hubbard=w["hubbard"])
    from hilbert_b200.synthetic import df_hamiltonian
    h, g = df_hamiltonian(**w["df"])
    return maps.RefProblem(w["nmo"], w["nalpha"], w["nbeta"], "DQG", True, True, h=h, g=g)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=sorted(WORKLOADS))
    ap.add_argument("--state", default=None, help="checkpoint file for a resumable run")
    ap.add_argument("--max-outer", type=int, default=400000)
    ap.add_argument("--cg-start", choices=("last", "extrapolate"), default="last",
                    help="CG starting point (oracle/bpsdp.py): the last y, or the extrapolation "
                         "through the last solutions, which the device solve uses")
    a = ap.parse_args()
    w = WORKLOADS[a.workload]
    P = problem(w)
    opts = SDPOptions(1e-6, 1e-6, 1e-9, 10000, a.max_outer)
    s = BPSDPSolver(P.n_primal, P.n_dual, opts, cg_start=a.cg_start)
    x = P.x0.copy()
    wall = 0.0
    if a.state and os.path.exists(a.state):
        st = np.load(a.state)
        x, s.y, s.z, s.mu = st["x"].copy(), st["y"].copy(), st["z"].copy(), float(st["mu"])
        s._oiter_total, s._iiter_total, wall = int(st["oiter"]), int(st["iiter"]), float(st["wall"])
        print(f"resumed at outer iteration {s.oiter_total()}", flush=True)
    while not s.is_converged() and s.oiter_total() < a.max_outer:
        t0 = time.perf_counter()
        s.solve(x, P.b, P.c, P.dims, min(MUF, a.max_outer - s.oiter_total()), P.Au, P.ATu)
        wall += time.perf_counter() - t0
        print(f"oiter {s.oiter_total()} iiter {s.iiter_total()} E {float(P.c @ x):.12f} "
              f"eps_p {s.primal_error:.3e} eps_d {s.dual_error:.3e} mu {s.mu:.4g} wall {wall:.0f} s",
              flush=True)
        if a.state:
            np.savez(a.state + ".tmp.npz", x=x, y=s.y, z=s.z, mu=s.mu, oiter=s.oiter_total(),
                     iiter=s.iiter_total(), wall=wall)
            os.replace(a.state + ".tmp.npz", a.state)
    out = {"workload": a.workload, "energy": float(P.c @ x), "dual_energy": float(P.b @ s.y),
           "eps_p": s.primal_error, "eps_d": s.dual_error, "converged": bool(s.is_converged()),
           "outer_iterations": s.oiter_total(), "cg_iterations": s.iiter_total(),
           "n_primal": int(P.n_primal), "n_dual": int(P.n_dual),
           "options": {"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "CG_CONVERGENCE": 1e-9,
                       "MU_UPDATE_FREQUENCY": MUF, "TPDM_GUESS": "RANDOM"},
           "maps": "hilbert's compiled maps (oracle/_ref)", "solver": "oracle/bpsdp.py",
           "cg_start": a.cg_start,
           "omp_threads": int(os.environ.get("OMP_NUM_THREADS", "0") or 0), "wall_s": round(wall, 1)}
    path = os.path.join(ROOT, "tests", "golden", f"fp64_{a.workload}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()

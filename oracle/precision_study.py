"""ORACLE -- test infrastructure only.

The precision study behind the mixed-precision projection: the boundary-point
iteration of oracle/bpsdp.py on a synthetic (n e, n o) DF problem
(hilbert_b200.synthetic.df_hamiltonian, seeds 4 and 5, the bench workload's
generator), solved to R_CONVERGENCE = E_CONVERGENCE = 1e-6 once with the FP64
projection and once with FP32 eigenvectors followed by one FP64
Rayleigh-Ritz step (project_blocks(..., "fp32rr")).  Prints one JSON line per
precision: outer and CG iterations, energy, errors; the energies' difference
and the outer iteration counts are what the study compares.  Run from the
repository root:

    OMP_NUM_THREADS=1 python oracle/precision_study.py 8
"""
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from oracle.bpsdp import BPSDPSolver, SDPOptions  # noqa: E402
from oracle.maps import OracleProblem  # noqa: E402


def run(n, precision, maxiter=200000, muf=500):
    from hilbert_b200.synthetic import df_hamiltonian
    h, g = df_hamiltonian(n, 400, 4, 5)
    o = OracleProblem(n, n // 2, n // 2, "DQG", True, True, h=h, g=g)
    s = BPSDPSolver(o.n_primal, o.n_dual, SDPOptions(1e-6, 1e-6, 1e-9, 10000, maxiter), precision=precision)
    x = o.guess("random")
    t0 = time.perf_counter()
    while not s.is_converged() and s.oiter_total() < maxiter:
        s.solve(x, o.b, o.c, [int(d) for d in o.dims], muf, o.Au, o.ATu)
    return {"n": n, "precision": precision, "converged": s.is_converged(), "outer_iterations": s.oiter_total(),
            "cg_iterations": s.iiter_total(), "energy": float(o.c @ x), "eps_p": s.primal_error,
            "eps_d": s.dual_error, "seconds": round(time.perf_counter() - t0, 1)}


if __name__ == "__main__":
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 8
    out = [run(n, p) for p in ("fp64", "fp32rr")]
    for r in out:
        print(json.dumps(r))
    print(json.dumps({"n": n, "abs_dE": abs(out[0]["energy"] - out[1]["energy"])}))

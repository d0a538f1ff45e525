"""Seeded synthetic Hamiltonians for the benchmark workloads.

No molecular integrals are available without Psi4, so the large-active-space
workload uses density-fitted-like integrals drawn from fixed seeds:
B^Q_pq ~ N(0, 0.05) symmetrised over (p, q) with naux = 400 (seed 4),
h = diag(linspace(-2, -0.1, n)) + N(0, 0.02) symmetrised off-diagonal (seed 5),
(pq|rs) = sum_Q B^Q_pq B^Q_rs, passed through the external-Hamiltonian path
(hilbert's v2rdm_solver.cc:147-195).
"""
import numpy as np


def df_hamiltonian(n=20, naux=400, seed_b=4, seed_h=5):
    """(h[n, n], g[n, n, n, n] in (pq|rs) order) for an (n e, n o) active space."""
    rb = np.random.default_rng(seed_b)
    B = rb.normal(0.0, 0.05, size=(naux, n, n))
    B = 0.5 * (B + B.transpose(0, 2, 1))
    rh = np.random.default_rng(seed_h)
    off = rh.normal(0.0, 0.02, size=(n, n))
    off = 0.5 * (off + off.T)
    np.fill_diagonal(off, 0.0)
    h = np.diag(np.linspace(-2.0, -0.1, n)) + off
    Bm = B.reshape(naux, n * n)
    g = (Bm.T @ Bm).reshape(n, n, n, n)
    return h, g


def hubbard_2d(lx=4, ly=4, t=1.0, U=8.0):
    """(h, g) of the periodic lx x ly Hubbard lattice for the external-
    Hamiltonian path (hilbert's own Hubbard path is the 1D ring only):
    h_ij = -t for the lattice neighbours of site i = x + lx y (left, right,
    up, down with wrap-around, each pair once), g_pppp = U, (pq|rs) order."""
    n = lx * ly
    h = np.zeros((n, n))
    for y in range(ly):
        for x in range(lx):
            i = x + lx * y
            for j in ((x + 1) % lx + lx * y, x + lx * ((y + 1) % ly)):
                if j != i:
                    h[i, j] = h[j, i] = -t
    g = np.zeros((n, n, n, n))
    for p in range(n):
        g[p, p, p, p] = U
    return h, g


def main(argv=None):
    """One solve of a synthetic DF active space on cuda:0 through the public
    API, printed as one JSON line: the small, bounded command that profilers
    and quick checks run.

        python -m hilbert_b200.synthetic --n 20 --naux 400 --max-outer 2
    """
    import argparse
    import json

    import torch

    import hilbert_b200 as hb
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--n", type=int, default=20, help="active orbitals (n electrons, singlet)")
    ap.add_argument("--naux", type=int, default=400)
    ap.add_argument("--positivity", default="DQG")
    ap.add_argument("--max-outer", type=int, default=2, help="MAXITER of the solve")
    ap.add_argument("--projection", default="refine", choices=("refine", "jacobi", "mixed"))
    a = ap.parse_args(argv)
    if a.n % 2:
        raise SystemExit("--n must be even (n electrons in n orbitals, singlet)")
    dev = torch.device("cuda", 0)
    p = hb.V2RDMProblem(a.n, a.n // 2, a.n // 2, a.positivity, True, True)
    h, g = df_hamiltonian(n=a.n, naux=a.naux)
    b, c, x0 = p.b(), p.c_external(h, g), p.guess("RANDOM")
    p.set_projection_mode(a.projection)
    opts = hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "CG_CONVERGENCE": 1e-9,
                       "MAXITER": a.max_outer, "MU_UPDATE_FREQUENCY": 500})
    x = torch.from_numpy(x0).to(dev)
    st = p.solve_device(x, torch.from_numpy(b).to(dev), torch.from_numpy(c).to(dev), opts)
    torch.cuda.synchronize()
    print(json.dumps({"n": a.n, "naux": a.naux, "positivity": a.positivity, "n_primal": int(x0.size),
                      "n_dual": int(b.size), "outer_iterations": st["oiter"], "cg_iterations": st["iiter"],
                      "converged": st["converged"], "energy": float(c @ x.cpu().numpy()),
                      "kernel_launches": p.kernel_launches()}))


if __name__ == "__main__":
    main()

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

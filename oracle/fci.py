"""ORACLE -- test infrastructure only.

Exact (full CI) ground-state energies of small Hamiltonians in the same
convention as hilbert's external / Hubbard input, used as known answers:
a DQG lower bound must satisfy E_DQG <= E_FCI, and for two electrons the
D condition alone is exact.
"""
import itertools

import numpy as np


def hubbard_ring_h(n, t):
    """One-electron matrix of hilbert's Hubbard ring (src/v2rdm_casscf/oei.cc:76-95)."""
    h = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            d = abs(i - j)
            if d == 1 or d == n - 1:
                h[i, j] = -t
    return h


def _strings(n, k):
    return [sum(1 << i for i in c) for c in itertools.combinations(range(n), k)]


def _single_excitations(s, n):
    """(j_from, i_to, sign, new) for a+_i a_j acting on bit string s."""
    out = []
    for j in range(n):
        if not (s >> j) & 1:
            continue
        s1 = s & ~(1 << j)
        sj = (-1) ** bin(s & ((1 << j) - 1)).count("1")
        for i in range(n):
            if (s1 >> i) & 1:
                continue
            si = (-1) ** bin(s1 & ((1 << i) - 1)).count("1")
            out.append((j, i, sj * si, s1 | (1 << i)))
    return out


def fci_energy(h, g, na, nb):
    """Lowest eigenvalue of H = sum_ij h_ij E_ij + 1/2 sum_ijkl (ij|kl) (E_ij E_kl - d_jk E_il)."""
    n = h.shape[0]
    A, B = _strings(n, na), _strings(n, nb)
    ia = {s: k for k, s in enumerate(A)}
    ib = {s: k for k, s in enumerate(B)}
    dim = len(A) * len(B)
    H = np.zeros((dim, dim))
    # E_ij on each spin string set (including diagonal i == j)
    def ops(strs, idx):
        m = {}
        for s in strs:
            for j, i, sg, t in _single_excitations(s, n):
                m.setdefault((i, j), []).append((idx[s], idx[t], sg))
        return m
    ea, eb = ops(A, ia), ops(B, ib)
    nA, nB = len(A), len(B)

    def E(i, j):
        M = np.zeros((dim, dim))
        for (a_from, a_to, sg) in ea.get((i, j), []):
            for bk in range(nB):
                M[a_to * nB + bk, a_from * nB + bk] += sg
        for (b_from, b_to, sg) in eb.get((i, j), []):
            for ak in range(nA):
                M[ak * nB + b_to, ak * nB + b_from] += sg
        return M

    Es = {(i, j): E(i, j) for i in range(n) for j in range(n)}
    for i in range(n):
        for j in range(n):
            if h[i, j] != 0.0:
                H += h[i, j] * Es[(i, j)]
    for i, j, k, l in itertools.product(range(n), repeat=4):
        v = g[i, j, k, l]
        if v == 0.0:
            continue
        H += 0.5 * v * (Es[(i, j)] @ Es[(k, l)])
        if j == k:
            H -= 0.5 * v * Es[(i, l)]
    return float(np.linalg.eigvalsh(H)[0])


def hubbard_fci(n, nelec, t, U):
    h = hubbard_ring_h(n, t)
    g = np.zeros((n, n, n, n))
    for i in range(n):
        g[i, i, i, i] = U
    return fci_energy(h, g, nelec // 2, nelec // 2)

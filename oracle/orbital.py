"""CPU restatements for the orbital-optimisation side of v2RDM-CASSCF (test
infrastructure: the checker for hilbert_b200.orbital and the packing kernel,
never the measured path).

* pack_spatial_density: hilbert's PackSpatialDensity
  (src/v2rdm_casscf/v2rdm_solver.cc:3110-3219) for C1 active spaces.
  Pinned bit-exactly to the reference's own compiled function
  (oracle/_ref, tests/test_orbital.py).
* focas_gradient: the orbital gradient of focas (src/focas/C_files/
  orbopt_gradient.cc:26-147 with Fi 863-1130, Fa 450-860, Q 223-449,
  Z 189-222) restated on dense matrices from the same definitions: inactive
  Fock Fi, active Fock Fa, Q and Z, gradient blocks
  ed = 4 (Fi + Fa), ea = 2 (Q + Z), ad = 4 (Fi + Fa) - 2 (Q + Z), aa
  (optional) = 2 (Q + Z - (Q + Z)^T).
"""
import numpy as np


def tri(i, j):
    """hilbert's INDEX(i, j): lower-triangle index"""
    return i * (i + 1) // 2 + j if i >= j else j * (j + 1) // 2 + i


def pack_spatial_density(x, n, off, iab, iaa):
    """(d2 packed over the n(n+1)/2 "00" geminals, d1 packed) from a primal x.

    off: block offsets ("d2ab", "d2aa", "d2bb", "d1a", "d1b"); iab(i, j) and
    iaa(i, j): geminal numbers.  Loops, sums and overwrites follow
    v2rdm_solver.cc:3116-3196 (C1: every geminal in irrep 0)."""
    gab, gaa = n * n, n * (n - 1) // 2
    g00 = n * (n + 1) // 2
    d2 = np.zeros(g00 * (g00 + 1) // 2)
    X = x
    for ij in range(gab):
        i, j = ij % n, ij // n
        ij_ab, ji_ab = iab(i, j), iab(j, i)
        ij_aa = iaa(i, j) if i != j else None
        for kl in range(gab):
            k, l = kl % n, kl // n
            kl_ab, lk_ab = iab(k, l), iab(l, k)
            kl_aa = iaa(k, l) if k != l else None
            ik, jl = tri(i, k), tri(j, l)
            kj_ab, il_ab, jk_ab, li_ab = iab(k, j), iab(i, l), iab(j, k), iab(l, i)
            dlj = 1.0 - float(l == j)
            dik = 1.0 - float(i == k)
            ab = off["d2ab"]
            val = 0.0
            val += 0.5 * X[ab + ij_ab * gab + kl_ab]
            val += 0.5 * X[ab + kj_ab * gab + il_ab] * dlj
            val += 0.5 * X[ab + il_ab * gab + kj_ab] * dik
            val += 0.5 * X[ab + kl_ab * gab + ij_ab] * dlj * dik
            val += 0.5 * X[ab + ji_ab * gab + lk_ab]
            val += 0.5 * X[ab + jk_ab * gab + li_ab] * dlj
            val += 0.5 * X[ab + li_ab * gab + jk_ab] * dik
            val += 0.5 * X[ab + lk_ab * gab + ji_ab] * dlj * dik
            if i != j and k != l:
                sij = 1 if i < j else -1
                skl = 1 if k < l else -1
                aa, bb = off["d2aa"], off["d2bb"]
                val += 0.5 * sij * skl * X[aa + ij_aa * gaa + kl_aa]
                val += 0.5 * sij * skl * X[aa + kl_aa * gaa + ij_aa] * dlj * dik
                val += 0.5 * sij * skl * X[bb + ij_aa * gaa + kl_aa]
                val += 0.5 * sij * skl * X[bb + kl_aa * gaa + ij_aa] * dlj * dik
            if k != j and i != l:
                skj = 1 if k < j else -1
                sil = 1 if i < l else -1
                kj_aa, il_aa = iaa(k, j), iaa(i, l)
                aa, bb = off["d2aa"], off["d2bb"]
                val += 0.5 * skj * sil * X[aa + kj_aa * gaa + il_aa] * dlj
                val += 0.5 * skj * sil * X[aa + il_aa * gaa + kj_aa] * dik
                val += 0.5 * skj * sil * X[bb + kj_aa * gaa + il_aa] * dlj
                val += 0.5 * skj * sil * X[bb + il_aa * gaa + kj_aa] * dik
            if ik != jl:
                val *= 2.0
            d2[tri(ik, jl)] = val
    d1 = np.zeros(n * (n + 1) // 2)
    for i in range(n):
        for j in range(i, n):
            d1[tri(i, j)] = X[off["d1a"] + i * n + j] + X[off["d1b"] + i * n + j]
    return d2, d1


def unpack_active(d2p, d1p, n):
    """Dense spin-summed active densities from the packed ones: D[t, u] and
    G[t, u, v, w] with E_act = sum h_tu D_tu + 1/2 sum (tu|vw) G_tuvw.

    A packed element holds half the sum of G over the orbit of its index under
    t <-> u, v <-> w and (tu) <-> (vw) (v2rdm_solver.cc:3152-3185: the
    first-electron and second-electron permutations, and the factor 2 for
    tu != vw), so that E_act,2 = sum over packed tu >= vw of (tu|vw) d2[tu, vw]."""
    D = np.zeros((n, n))
    for t in range(n):
        for u in range(n):
            D[t, u] = d1p[tri(t, u)]
    G = np.zeros((n, n, n, n))
    for t in range(n):
        for u in range(n):
            tu = tri(t, u)
            for v in range(n):
                for w in range(n):
                    vw = tri(v, w)
                    m = (2 if t != u else 1) * (2 if v != w else 1) * (2 if tu != vw else 1)
                    G[t, u, v, w] = 2.0 * d2p[tri(tu, vw)] / m
    return D, G


def full_densities(D_act, G_act, ncore):
    """Dense spin-summed densities over core + active orbitals (core doubly occupied)."""
    na = D_act.shape[0]
    n = ncore + na
    D = np.zeros((n, n))
    G = np.zeros((n, n, n, n))
    c = np.arange(ncore)
    a = slice(ncore, n)
    D[c, c] = 2.0
    D[a, a] = D_act
    G[a, a, a, a] = G_act
    for i in range(ncore):
        for j in range(ncore):
            G[i, i, j, j] += 4.0
            G[i, j, j, i] -= 2.0
        G[i, i, a, a] += 2.0 * D_act
        G[a, a, i, i] += 2.0 * D_act
        G[i, a, a, i] -= D_act.T
        G[a, i, i, a] -= D_act
    return D, G


def energy(h, eri, D, G):
    return float(np.einsum("pq,pq->", h, D) + 0.5 * np.einsum("pqrs,pqrs->", eri, G))


def focas_gradient(h, B, D_act, G_act, ncore, nact, active_active=False):
    """focas's orbital gradient on dense matrices (see module docstring).

    h: (nmo, nmo) one-electron integrals; B: (naux, nmo, nmo) DF factors,
    (pq|rs) = sum_Q B[Q,p,q] B[Q,r,s]; D_act, G_act: dense spin-summed active
    densities.  Returns {(p, q): g} for the rotation pairs p > q of different
    classes (core 0, active 1, virtual 2), focas's sign convention."""
    nmo = h.shape[0]
    core = list(range(ncore))
    act = list(range(ncore, ncore + nact))
    eri = np.einsum("Qpq,Qrs->pqrs", B, B)
    # inactive Fock: Fi_pq = h_pq + sum_i 2 (pq|ii) - (pi|iq)
    Fi = h.copy()
    for i in core:
        Fi += 2.0 * eri[:, :, i, i] - eri[:, i, i, :]
    # active Fock: Fa_pq = sum_tu D_tu [ (pq|tu) - 1/2 (pt|uq) ]
    Fa = np.zeros((nmo, nmo))
    for ti, t in enumerate(act):
        for ui, u in enumerate(act):
            Fa += D_act[ti, ui] * (eri[:, :, t, u] - 0.5 * eri[:, t, u, :])
    # Q_tp = sum_uvw G_tuvw (pu|vw);  Z_tp = sum_u D_tu Fi_pu
    A = np.ix_(act, act, act)
    Qm = np.zeros((nact, nmo))
    for ti in range(nact):
        for p in range(nmo):
            Qm[ti, p] = np.einsum("uvw,uvw->", G_act[ti], eri[p][A])
    Zm = np.zeros((nact, nmo))
    for ti in range(nact):
        for p in range(nmo):
            Zm[ti, p] = sum(D_act[ti, ui] * Fi[p, u] for ui, u in enumerate(act))
    virt = list(range(ncore + nact, nmo))
    g = {}
    for a_ in virt:
        for i in core:
            g[(a_, i)] = 4.0 * (Fi[a_, i] + Fa[a_, i])
    for a_ in virt:
        for ti, t in enumerate(act):
            g[(a_, t)] = 2.0 * (Qm[ti, a_] + Zm[ti, a_])
    for ti, t in enumerate(act):
        for i in core:
            g[(t, i)] = 4.0 * (Fi[t, i] + Fa[t, i]) - 2.0 * (Qm[ti, i] + Zm[ti, i])
    if active_active:
        for ti, t in enumerate(act):
            for ui, u in enumerate(act[:ti]):
                g[(t, u)] = 2.0 * (Qm[ui, t] + Zm[ui, t] - Qm[ti, u] - Zm[ti, u])
    return g

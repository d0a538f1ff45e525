"""CPU restatements for the orbital-optimisation side of v2RDM-CASSCF (test
infrastructure: the checker for hilbert_b200.orbital and the packing kernel,
never the measured path).

* pack_spatial_density: hilbert's PackSpatialDensity
  (src/v2rdm_casscf/v2rdm_solver.cc:3110-3219) for C1 active spaces.
  Pinned bit-exactly to the reference's own compiled function
  (oracle/_ref, tests/test_orbital.py).
* focas_gradient: the orbital gradient of focas (src/focas/
  orbopt_gradient.cc:26-146 with Fi 852-1118, Fa 441-851, Q 218-440,
  Z 185-216) restated on dense matrices from the same definitions: inactive
  Fock Fi, active Fock Fa, Q and Z, gradient blocks
  ed = 4 (Fi + Fa), ea = 2 (Q + Z), ad = 4 (Fi + Fa) - 2 (Q + Z), aa
  (optional) = 2 (Q + Z - (Q + Z)^T).
* focas_diagonal_hessian: focas's exact diagonal Hessian
  (src/focas/orbopt_hessian.cc), literally, loops and half-triangle sums.
* focas_optimize: focas's orbital step loop (src/focas/orbopt_optimize.cc:
  25-264) on these, with scipy's expm.
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


def _focas_intermediates(h, B, D_act, G_act, ncore, nact):
    """eri, Fi, Fa, Q (nact x nmo) and Z (nact x nmo) as focas defines them
    (orbopt_gradient.cc: Fi 852-1118, Fa 441-851, Q 218-440, Z 185-216)."""
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
    return eri, Fi, Fa, Qm, Zm


def focas_diagonal_hessian(h, B, d2p, d1p, ncore, nact, active_active=False):
    """focas's exact diagonal orbital Hessian (ORBOPT_EXACT_DIAGONAL_HESSIAN,
    on by default, plugin.cc:162), restated on dense integrals from
    orbopt_hessian.cc.  d2p, d1p: PackSpatialDensity's output; focas's Sort
    (orbopt_sort.cc:40-117) rescales each packed element by 2 / m (m the size
    of its index orbit) on entry, so the d2(tu|vw) of the formulas below is
    the dense spin-summed 2-RDM G_tuvw:
      ed (a, i)  ComputeH_diag_ed, :426-463
                 4 [F_aa - F_ii + 3 (ia|ia) - (ii|aa)],   F = Fi + Fa
      ad (t, i)  ComputeH_diag_ad, :135-188, and tei_terms_H_ad, :190-424
                 2 [2 (F_tt - F_ii) + D_tt Fi_ii - Q_tt - Z_tt]
                 + sum_u [sum_{v<u} 4 d2(tt|uv) (uv|ii) + 2 d2(tt|uu) (uu|ii)]
                 + 4 [sum_u D_tu (tu|ii) - (tt|ii)]
                 + sum_uv 4 d2(tu|tv) (ui|vi) + 12 [(ti|ti) - sum_u D_tu (ui|ti)]
      ea (a, t)  ComputeH_diag_ea, :830-870, and tei_terms_H_ea, :872-1047
                 2 [D_tt Fi_aa - Q_tt - Z_tt]
                 + 4 sum_u [sum_{v<u} d2(tt|uv) (uv|aa) + 1/2 d2(tt|uu) (uu|aa)]
                 + 8 sum_u [sum_{v<u} (ua|va) d2(ut|vt) + 1/2 (ua|ua) d2(ut|ut)]
      aa (t, u), t > u, with active_active (ComputeH_diag_aa, :465-827)
                 2 [D_tt Fi_uu + D_uu Fi_tt - Q_tt - Z_tt - Q_uu - Z_uu - 2 D_tu Fi_tu]
                 + sum_rs [(tt|rs) d2(uu|rs) + (uu|rs) d2(tt|rs) - 2 (tu|rs) d2(tu|rs)]
                 + 2 sum_rs [(tr|ts) d2(ur|us) + (ur|us) d2(tr|ts) - 2 (ur|ts) d2(ur|ts)]
    Returns {(p, q): H} for the pairs of different classes (and the
    active-active pairs when asked), keyed like focas_gradient."""
    nmo = h.shape[0]
    core = list(range(ncore))
    act = list(range(ncore, ncore + nact))
    virt = list(range(ncore + nact, nmo))
    D_act, G_act = unpack_active(d2p, d1p, nact)
    eri, Fi, Fa, Qm, Zm = _focas_intermediates(h, B, D_act, G_act, ncore, nact)
    F = Fi + Fa

    def P(a, b, c, d):   # focas's d2(ab|cd) after its rescale (active local indices)
        return G_act[a, b, c, d]

    H = {}
    for a_ in virt:
        for i in core:
            H[(a_, i)] = 4.0 * (F[a_, a_] - F[i, i] + 3.0 * eri[i, a_, i, a_] - eri[i, i, a_, a_])
    for a_ in virt:
        for t in range(nact):
            T = act[t]
            v = 2.0 * (D_act[t, t] * Fi[a_, a_] - Qm[t, T] - Zm[t, T])
            c = 0.0
            for u in range(nact):
                for w in range(u):
                    c += P(t, t, u, w) * eri[act[u], act[w], a_, a_]
                c += 0.5 * P(t, t, u, u) * eri[act[u], act[u], a_, a_]
            x = 0.0
            for u in range(nact):
                for w in range(u):
                    x += eri[act[u], a_, act[w], a_] * P(u, t, w, t)
                x += 0.5 * eri[act[u], a_, act[u], a_] * P(u, t, u, t)
            H[(a_, T)] = v + 4.0 * c + 8.0 * x
    for t in range(nact):
        T = act[t]
        for i in core:
            v = 2.0 * (2.0 * (F[T, T] - F[i, i]) + D_act[t, t] * Fi[i, i] - Qm[t, T] - Zm[t, T])
            c = 0.0
            for u in range(nact):
                for w in range(u):
                    c += 4.0 * P(t, t, u, w) * eri[act[u], act[w], i, i]
                c += 2.0 * P(t, t, u, u) * eri[act[u], act[u], i, i]
            d = -eri[T, T, i, i] + sum(D_act[t, u] * eri[T, act[u], i, i] for u in range(nact))
            x = 0.0
            for u in range(nact):
                for w in range(nact):
                    x += 4.0 * P(t, u, t, w) * eri[act[u], i, act[w], i]
            e = eri[T, i, T, i] - sum(D_act[t, u] * eri[act[u], i, T, i] for u in range(nact))
            H[(T, i)] = v + c + 4.0 * d + x + 12.0 * e
    if active_active:
        # ComputeH_diag_aa's sums read the three-index array tei (Q-major
        # over the packed lower triangle of all orbitals) at the positions of
        # its four-index scratch array (orbopt_hessian.cc:640-642, 731-733,
        # 797-799): tei[y m + x] with x, y packed active-pair indices and
        # m = nact (nact + 1) / 2, restated as read
        m = nact * (nact + 1) // 2
        iu = np.tril_indices(B.shape[1])
        tei = np.ascontiguousarray(B[:, iu[0], iu[1]]).reshape(-1)

        def L(i, j):
            return i * (i + 1) // 2 + j if i >= j else j * (j + 1) // 2 + i

        def T3(x, y):
            return tei[y * m + x]

        A = act
        for t in range(nact):
            for u in range(t):
                T, Uo = A[t], A[u]
                v = 2.0 * (-(Qm[t, T] + Zm[t, T] + Qm[u, Uo] + Zm[u, Uo] + 2.0 * D_act[t, u] * Fi[T, Uo])
                           + D_act[t, t] * Fi[Uo, Uo] + D_act[u, u] * Fi[T, T])
                c = 0.0
                x = 0.0
                for r in range(nact):
                    for q in range(nact):
                        R, S = A[r], A[q]
                        c += (T3(L(r, q), L(t, t)) * P(u, u, r, q) + T3(L(r, q), L(u, u)) * P(t, t, r, q)
                              - 2.0 * T3(L(r, q), L(t, u)) * P(t, u, r, q))
                        x += (T3(L(t, r), L(t, q)) * P(u, r, u, q) + T3(L(u, r), L(u, q)) * P(t, r, t, q)
                              - 2.0 * T3(L(u, r), L(t, q)) * P(u, r, t, q))
                H[(T, Uo)] = v + c + 2.0 * x
    return H


def focas_gradient(h, B, D_act, G_act, ncore, nact, active_active=False):
    """focas's orbital gradient on dense matrices (see module docstring).

    h: (nmo, nmo) one-electron integrals; B: (naux, nmo, nmo) DF factors,
    (pq|rs) = sum_Q B[Q,p,q] B[Q,r,s]; D_act, G_act: dense spin-summed active
    densities.  Returns {(p, q): g} for the rotation pairs p > q of different
    classes (core 0, active 1, virtual 2), focas's sign convention."""
    nmo = h.shape[0]
    core = list(range(ncore))
    act = list(range(ncore, ncore + nact))
    eri, Fi, Fa, Qm, Zm = _focas_intermediates(h, B, D_act, G_act, ncore, nact)
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


def rotation_pairs(ncore, nact, nvirt, active_active=False):
    """focas's rotation order (Determine_GradIndMap, orbopt_gradient.cc:151-186):
    active-core, active-active (t > u, with active-active rotations),
    virtual-core, virtual-active; then p, then q."""
    core = range(ncore)
    act = range(ncore, ncore + nact)
    virt = range(ncore + nact, ncore + nact + nvirt)
    pairs = [(p, q) for p in act for q in core]
    if active_active:
        pairs += [(p, q) for p in act for q in act if q < p]
    pairs += [(p, q) for p in virt for q in core] + [(p, q) for p in virt for q in act]
    return pairs


def focas_optimize(h, B, d2p, d1p, ncore, nact, maxiter=10, g_conv=1e-4, e_conv=1e-8,
                   active_active=False):
    """focas's optimize_orbitals (src/focas/orbopt_optimize.cc:25-96) with
    Update_kappa (:98-115), Update_r (:117-146), Compute_Quadratic_dE
    (:162-176), Restore_last_step (:226-245) and Precondition_Step
    (:247-264), at fixed densities, on dense numpy integrals.  The rotation
    of a step k is expm(K), K[p, q] = k_pq, K[q, p] = -k_pq for the pairs
    p > q (ExponentiateKappa, orbopt_exponential.cc:151-182); the integrals
    accumulate the rotations.  Returns (h, B, U, history) with history the
    per-iteration (E_new, dE, |g|, r)."""
    from scipy.linalg import expm
    nmo = h.shape[0]
    nvirt = nmo - ncore - nact
    pairs = rotation_pairs(ncore, nact, nvirt, active_active)
    D_act, G_act = unpack_active(d2p, d1p, nact)
    D, G = full_densities(D_act, G_act, ncore)
    if nvirt:
        Dn = np.zeros((nmo, nmo)); Dn[:D.shape[0], :D.shape[0]] = D
        Gn = np.zeros((nmo,) * 4); m = D.shape[0]; Gn[:m, :m, :m, :m] = G
        D, G = Dn, Gn
    h, B = h.copy(), B.copy()
    U = np.eye(nmo)

    def rotate(k):
        nonlocal h, B, U
        K = np.zeros((nmo, nmo))
        for (p, q), v in zip(pairs, k):
            K[p, q], K[q, p] = v, -v
        R = expm(K)
        h = R.T @ h @ R
        B = np.einsum("mp,Qmn,nq->Qpq", R, B, R)
        U = U @ R

    def E():
        return energy(h, np.einsum("Qpq,Qrs->pqrs", B, B), D, G)

    r, eval_g = 1.0, True
    k_cur = np.zeros(len(pairs))
    k_ref, k_save = k_cur.copy(), k_cur.copy()
    E_init = gnorm = dE = 0.0
    conv_e = conv_g = False
    hist = []
    for it in range(maxiter):
        if eval_g:
            E_init = E()
            gd = focas_gradient(h, B, D_act, G_act, ncore, nact, active_active)
            g = np.array([gd[pq] for pq in pairs])
            gnorm = float(np.sqrt(g @ g))
            Hd_ = focas_diagonal_hessian(h, B, d2p, d1p, ncore, nact, active_active)
            Hd = np.array([Hd_[pq] for pq in pairs])
            dE_quad = 0.5 * (2.0 * (g @ k_cur) + float(np.sum(k_cur * Hd * k_cur)))
            Hc = np.abs(Hd)
            Hc[Hc < 1e-2] = 1e-2
            k_ref = -g / Hc
            k_cur = r * k_ref
            k_save = k_cur.copy()
        rotate(k_cur)
        E_new = E()
        dE = E_new - E_init
        hist.append((E_new, dE, gnorm, r))
        conv_g = gnorm < g_conv
        conv_e = abs(dE) < e_conv
        if conv_e or conv_g or it == maxiter - 1:
            break
        eval_g = not (dE > 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = np.float64(dE) / np.float64(dE_quad)
        if dE < 0.0:
            if ratio > 0.75:
                r *= 1.2
            if ratio < 0.25:
                r *= 0.7
        else:
            r *= 0.7
        if not eval_g:
            k_cur = r * k_ref - k_cur
            k_save = k_save + k_cur
    if dE > 0.0:
        if conv_e or conv_g:
            rotate(-k_cur)
        if not eval_g:
            rotate(-k_save)
    return h, B, U, hist

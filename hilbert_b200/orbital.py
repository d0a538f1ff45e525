"""Orbital side of v2RDM-CASSCF: the energy of rotated orbitals from the
v2RDM densities with density-fitted integrals, and its orbital gradient
through a hand-written adjoint of the integral transform.

With U = exp(kappa) (kappa antisymmetric), the transformed integrals are
h' = U^T h U and B'^Q = U^T B^Q U ((pq|rs) = sum_Q B^Q_pq B^Q_rs, focas's DF
transform, src/focas/orbopt_integraltransform_cpu.cc:25-329), and

    E(kappa) = sum_pq h'_pq D_pq + 1/2 sum_Q b'_Q^T Gm b'_Q,    b'_Q = vec(B'^Q),

with D and Gm (= G_{pq,rs}) the spin-summed core + active densities.
RotatedEnergy's backward does not replay the forward on a tape: it forms
M_Q = Gm b'_Q (= dE/dB'^Q), dE/dU = h U D^T + h^T U D + sum_Q (B^Q U M_Q^T +
B^Q^T U M_Q), and the adjoint of the matrix exponential, L_exp(kappa^T, dE/dU),
as the upper-right block of exp([[kappa^T, dE/dU], [0, kappa^T]]).  At
kappa = 0 the rotation-pair gradient dE/dkappa_pq - dE/dkappa_qp (p > q) is
focas's orbital gradient (orbopt_gradient.cc:26-147: ed = 4 (Fi + Fa),
ea = 2 (Q + Z), ad = 4 (Fi + Fa) - 2 (Q + Z)).

Orbital steps at fixed densities: optimize_orbitals (L-BFGS on the adjoint
gradient) or optimize_orbitals_focas, focas's own step (src/focas/
orbopt_optimize.cc:25-96): kappa = -r g / max(|H_diag|, 1e-2) with focas's
exact diagonal Hessian (diagonal_hessian, orbopt_hessian.cc) and its trust
factor r.

The densities come from the device solve through
V2RDMProblem.pack_spatial_density (hilbert's PackSpatialDensity) and
unpack_densities here.  All tensors are float64; the GEMMs are torch's.
"""
import numpy as np
import torch


def _tri(i, j):
    return torch.where(i >= j, i * (i + 1) // 2 + j, j * (j + 1) // 2 + i)


def unpack_densities(d2p, d1p, n):
    """Dense spin-summed active densities (D[t, u], G[t, u, v, w]) from
    PackSpatialDensity's packed arrays: a packed element holds half the sum of
    G over the orbit of its index under t <-> u, v <-> w and (tu) <-> (vw)
    (v2rdm_solver.cc:3152-3185), so G = 2 d2[id] / |orbit| and
    E_act = sum h_tu D_tu + 1/2 sum (tu|vw) G_tuvw."""
    dev = d2p.device
    r = torch.arange(n, device=dev)
    t, u = torch.meshgrid(r, r, indexing="ij")
    D = d1p[_tri(t, u)]
    t, u, v, w = torch.meshgrid(r, r, r, r, indexing="ij")
    tu, vw = _tri(t, u), _tri(v, w)
    mult = ((t != u).double() + 1.0) * ((v != w).double() + 1.0) * ((tu != vw).double() + 1.0)
    G = 2.0 * d2p[_tri(tu, vw)] / mult
    return D, G


def full_densities(D_act, G_act, ncore, nvirt=0):
    """Spin-summed densities over core (doubly occupied) + active + virtual
    orbitals, G[p, q, r, s] pairing (pq|rs)."""
    na = D_act.shape[0]
    n = ncore + na + nvirt
    dev, dt = D_act.device, D_act.dtype
    D = torch.zeros((n, n), dtype=dt, device=dev)
    G = torch.zeros((n, n, n, n), dtype=dt, device=dev)
    a = slice(ncore, ncore + na)
    D[a, a] = D_act
    G[a, a, a, a] = G_act
    for i in range(ncore):
        D[i, i] = 2.0
        for j in range(ncore):
            G[i, i, j, j] += 4.0
            G[i, j, j, i] -= 2.0
        G[i, i, a, a] += 2.0 * D_act
        G[a, a, i, i] += 2.0 * D_act
        G[i, a, a, i] -= D_act.T
        G[a, i, i, a] -= D_act
    return D, G


def _dptr(t):
    import ctypes
    return ctypes.c_void_p(t.data_ptr())


def df_transform(U, B):
    """B'_Q = U^T B_Q U for every Q of B (count x n x n): focas's DF integral
    transform (orbopt_integraltransform_cpu.cc:235-261).  CUDA tensors run
    the library's FP64 tensor-core kernel (v2b_df_transform); CPU tensors
    evaluate the same products in torch."""
    if not U.is_cuda:
        return U.T @ B @ U
    from . import _capi
    lib = _capi.load()
    n, count = U.shape[0], B.shape[0]
    U = U.contiguous()
    B = B.contiguous()
    out = torch.empty_like(B)
    _capi.check(lib.v2b_df_transform(_dptr(U), _dptr(B), _dptr(out), n, count,
                                     _dptr_stream(U.device)))
    return out


def df_transform_adjoint(U, B, M):
    """sum_Q (B_Q U M_Q^T + B_Q^T U M_Q): the U-gradient of
    sum_Q <M_Q, U^T B_Q U>.  CUDA tensors run v2b_df_transform_adjoint."""
    if not U.is_cuda:
        return (B @ U @ M.transpose(1, 2)).sum(0) + (B.transpose(1, 2) @ U @ M).sum(0)
    from . import _capi
    lib = _capi.load()
    n, count = U.shape[0], B.shape[0]
    U, B, M = U.contiguous(), B.contiguous(), M.contiguous()
    dU = torch.empty_like(U)
    work = torch.empty_like(B)
    _capi.check(lib.v2b_df_transform_adjoint(_dptr(U), _dptr(B), _dptr(M), _dptr(dU), _dptr(work), n,
                                             count, _dptr_stream(U.device)))
    return dU


def _dptr_stream(device):
    import ctypes
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class RotatedEnergy(torch.autograd.Function):
    """E(kappa) for U = exp(kappa); backward by the hand-written adjoint.
    The integral transforms h' = U^T h U, B'_Q = U^T B_Q U and their adjoint
    run in the library's kernels for CUDA tensors (df_transform,
    df_transform_adjoint); the 2-RDM contraction b' Gm is a plain GEMM."""

    @staticmethod
    def forward(ctx, kappa, h, B, D, Gm):
        n = h.shape[0]
        U = torch.linalg.matrix_exp(kappa)
        hp = df_transform(U, h.unsqueeze(0))[0]
        Bp = df_transform(U, B)               # (naux, n, n), one matrix per CTA
        b = Bp.reshape(B.shape[0], n * n)
        Gb = b @ Gm                           # rows: (Gm b'_Q)^T, Gm symmetric
        E = (hp * D).sum() + 0.5 * (Gb * b).sum()
        ctx.save_for_backward(kappa, h, B, D, U, Gb)
        return E

    @staticmethod
    def backward(ctx, gE):
        kappa, h, B, D, U, Gb = ctx.saved_tensors
        n = h.shape[0]
        M = Gb.reshape(B.shape[0], n, n)      # dE/dB'^Q
        dU = df_transform_adjoint(U, h.unsqueeze(0), D.unsqueeze(0))   # h U D^T + h^T U D
        dU = dU + df_transform_adjoint(U, B, M)
        Z = torch.zeros((2 * n, 2 * n), dtype=kappa.dtype, device=kappa.device)
        Z[:n, :n] = kappa.T
        Z[n:, n:] = kappa.T
        Z[:n, n:] = dU
        dK = torch.linalg.matrix_exp(Z)[:n, n:]
        return gE * dK, None, None, None, None


def rotated_energy(kappa, h, B, D, G):
    n = h.shape[0]
    return RotatedEnergy.apply(kappa, h, B, D, G.reshape(n * n, n * n))


def rotation_pairs(ncore, nact, nvirt, active_active=False):
    """Non-redundant rotation pairs (p, q), p > q, in focas's order
    (Determine_GradIndMap, src/focas/C_files/orbopt_gradient.cc:151-186): by
    the class of p (active, then virtual), then the class of q (core, then
    active; active-active pairs only with active_active), then p, then q."""
    core = range(ncore)
    act = range(ncore, ncore + nact)
    virt = range(ncore + nact, ncore + nact + nvirt)
    pairs = [(p, q) for p in act for q in core]
    if active_active:
        pairs += [(p, q) for p in act for q in act if q < p]
    pairs += [(p, q) for p in virt for q in core]
    pairs += [(p, q) for p in virt for q in act]
    return pairs


def orbital_gradient(h, B, D, G, pairs):
    """dE/dkappa_pq - dE/dkappa_qp at kappa = 0 for the given pairs (p > q)."""
    n = h.shape[0]
    kappa = torch.zeros((n, n), dtype=h.dtype, device=h.device, requires_grad=True)
    E = rotated_energy(kappa, h, B, D, G)
    (gK,) = torch.autograd.grad(E, kappa)
    p = torch.tensor([a for a, _ in pairs], device=h.device)
    q = torch.tensor([b for _, b in pairs], device=h.device)
    return E.detach(), gK[p, q] - gK[q, p]


def casscf_df_problem(nbf=40, naux=160, ncore=5, nact=10, seed_b=0, seed_h=1, seed_c=2):
    """Synthetic DF CASSCF integrals in a random orthonormal MO basis:
    B^Q_mn ~ N(0, 0.1) symmetrised per Q (seed_b), h = diag(linspace(-1, -10,
    nbf)) + 0.05 sym N(0, 1) (seed_h), C0 = Q of the QR of N(0, 1) (seed_c).
    Returns (h_mo, B_mo, active-space h, active-space g, frozen-core energy)."""
    rb = np.random.default_rng(seed_b)
    B = rb.normal(0.0, 0.1, size=(naux, nbf, nbf))
    B = 0.5 * (B + B.transpose(0, 2, 1))
    rh = np.random.default_rng(seed_h)
    m = rh.standard_normal((nbf, nbf))
    h = np.diag(np.linspace(-1.0, -10.0, nbf)) + 0.05 * 0.5 * (m + m.T)
    C0, _ = np.linalg.qr(np.random.default_rng(seed_c).standard_normal((nbf, nbf)))
    h_mo = C0.T @ h @ C0
    B_mo = np.einsum("mp,Qmn,nq->Qpq", C0, B, C0)
    core = list(range(ncore))
    act = list(range(ncore, ncore + nact))
    # inactive Fock: Fi_pq = h_pq + sum_i 2 (pq|ii) - (pi|iq)
    occ = B_mo[:, core][:, :, core].trace(axis1=1, axis2=2)           # sum_i B^Q_ii
    J = np.einsum("Qpq,Q->pq", B_mo, occ)
    K = np.einsum("Qpi,Qiq->pq", B_mo[:, :, core], B_mo[:, core, :])
    Fi = h_mo + 2.0 * J - K
    e_core = float(sum(h_mo[i, i] + Fi[i, i] for i in core))
    Ba = B_mo[:, act][:, :, act]
    g_act = np.einsum("Qtu,Qvw->tuvw", Ba, Ba)
    return h_mo, B_mo, Fi[np.ix_(act, act)], g_act, e_core


def optimize_orbitals(h, B, D, G, pairs, max_iter=100, gtol=1e-10):
    """Orbital optimisation at fixed densities (what focas iterates between SDP
    solves, orbopt_optimize.cc:25-98): minimise E(kappa) over the given
    rotation pairs by L-BFGS with the adjoint gradient.  Returns U = exp(kappa),
    the energy there, and the gradient norms (over the pairs) at the start and
    at the end."""
    n = h.shape[0]
    p = torch.tensor([a for a, _ in pairs], device=h.device)
    q = torch.tensor([b for _, b in pairs], device=h.device)
    theta = torch.zeros(len(pairs), dtype=h.dtype, device=h.device, requires_grad=True)

    def kappa(t):
        K = torch.zeros((n, n), dtype=h.dtype, device=h.device)
        K = K.index_put((p, q), t)
        return K.index_put((q, p), -t)

    Gm = G.reshape(n * n, n * n)
    E0 = RotatedEnergy.apply(kappa(theta), h, B, D, Gm)
    (g0,) = torch.autograd.grad(E0, theta)
    opt = torch.optim.LBFGS([theta], max_iter=max_iter, tolerance_grad=gtol, tolerance_change=1e-14,
                            history_size=20, line_search_fn="strong_wolfe")

    def closure():
        opt.zero_grad()
        E = RotatedEnergy.apply(kappa(theta), h, B, D, Gm)
        E.backward()
        return E

    opt.step(closure)   # returns the first evaluation; the final state is taken below
    K = kappa(theta)
    E = RotatedEnergy.apply(K, h, B, D, Gm)
    (g1,) = torch.autograd.grad(E, theta)
    with torch.no_grad():
        U = torch.linalg.matrix_exp(K)
    return U, float(E.detach()), float(g0.norm()), float(g1.norm())


def _fock_q_z(h, B, Da, Ga, ncore, nact):
    """focas's intermediates on the full orbital range (orbopt_gradient.cc:
    Fi 852-1118, Fa 441-851, Q 218-440, Z 185-216):
    Fi_pq = h_pq + sum_i 2 (pq|ii) - (pi|iq),
    Fa_pq = sum_tu D_tu [(pq|tu) - 1/2 (pt|uq)],
    Q_tp = sum_uvw G_tuvw (pu|vw),  Z_tp = sum_u D_tu Fi_pu."""
    c = slice(0, ncore)
    a = slice(ncore, ncore + nact)
    Bd = torch.diagonal(B, dim1=1, dim2=2)                        # B^Q_pp
    Fi = (h + 2.0 * torch.einsum("Qpq,Q->pq", B, Bd[:, c].sum(1))
          - torch.einsum("Qpi,Qiq->pq", B[:, :, c], B[:, c, :]))
    Ba = B[:, a, a]
    Fa = (torch.einsum("Qpq,Q->pq", B, torch.einsum("Qtu,tu->Q", Ba, Da))
          - 0.5 * torch.einsum("Qpt,tu,Quq->pq", B[:, :, a], Da, B[:, a, :]))
    Qm = torch.einsum("Qpu,Qtu->tp", B[:, :, a], torch.einsum("tuvw,Qvw->Qtu", Ga, Ba))
    Z = Da @ Fi[a, :]
    return Fi, Fa, Qm, Z


def diagonal_hessian(h, B, Da, Ga, ncore, nact, active_active=False):
    """focas's exact diagonal orbital Hessian (ORBOPT_EXACT_DIAGONAL_HESSIAN,
    on by default) for the rotation pairs of rotation_pairs(ncore, nact,
    nvirt, active_active), from src/focas/orbopt_hessian.cc:
      ed (a, i) :426-463   4 [F_aa - F_ii + 3 (ia|ia) - (ii|aa)],  F = Fi + Fa
      ea (a, t) :830-1047  2 [D_tt Fi_aa - Q_tt - Z_tt] + 2 sum_uv G_ttuv (uv|aa)
                           + 4 sum_uv G_utvt (ua|va)
      ad (t, i) :135-424   2 [2 (F_tt - F_ii) + D_tt Fi_ii - Q_tt - Z_tt]
                           + 2 sum_uv G_ttuv (uv|ii) + 4 [sum_u D_tu (tu|ii) - (tt|ii)]
                           + 4 sum_uv G_utvt (ui|vi) + 12 [(ti|ti) - sum_u D_tu (ui|ti)]
      aa (t, u) :465-827   2 [D_tt Fi_uu + D_uu Fi_tt - Q_tt - Z_tt - Q_uu - Z_uu - 2 D_tu Fi_tu]
           (t > u)         + sum_rs [(tt|rs) G_uurs + (uu|rs) G_ttrs - 2 (tu|rs) G_turs]
                           + 2 sum_rs [(tr|ts) G_urus + (ur|us) G_trts - 2 (ur|ts) G_urts]
    G is the dense spin-summed active 2-RDM, the d2 focas works with after
    its Sort (orbopt_sort.cc:40-117 rescales the packed elements by 2 / m);
    the half-triangle sums of the reference become full sums by the pair
    symmetries of G.  Every (pq|rs) is a contraction of the DF factors."""
    nmo = h.shape[0]
    c = slice(0, ncore)
    a = slice(ncore, ncore + nact)
    v = slice(ncore + nact, nmo)
    Fi, Fa, Qm, Z = _fock_q_z(h, B, Da, Ga, ncore, nact)
    Fd, Fid = torch.diagonal(Fi + Fa), torch.diagonal(Fi)
    Qtt = torch.diagonal(Qm[:, a])
    Ztt = torch.diagonal(Z[:, a])
    Dtt = torch.diagonal(Da)
    Bd = torch.diagonal(B, dim1=1, dim2=2)                        # (Q, nmo)
    Ba = B[:, a, a]
    Bap = B[:, a, :]                                              # B^Q_up
    # sum_uv G_ttuv (uv|pp) and sum_uv G_utvt (up|vp), for every p
    coul = torch.einsum("uvt,Quv->tQ", torch.diagonal(Ga, dim1=0, dim2=1), Ba) @ Bd
    exch = torch.einsum("Qup,uvt,Qvp->tp", Bap, torch.diagonal(Ga, dim1=1, dim2=3), Bap)
    # ed
    Bvc = B[:, v, c]
    H_ed = 4.0 * (Fd[v][:, None] - Fd[c][None, :] + 3.0 * (Bvc * Bvc).sum(0)
                  - torch.einsum("Qa,Qi->ai", Bd[:, v], Bd[:, c]))
    # ea, indexed (a, t)
    H_ea = (2.0 * (Dtt[None, :] * Fid[v][:, None] - (Qtt + Ztt)[None, :])
            + 2.0 * coul[:, v].T + 4.0 * exch[:, v].T)
    # ad, indexed (t, i)
    tupp = torch.einsum("tu,Qtu,Qp->tp", Da, Ba, Bd[:, c])        # sum_u D_tu (tu|ii)
    ttpp = torch.diagonal(Ba, dim1=1, dim2=2).T @ Bd[:, c]         # (tt|ii)
    tptp = (Bap[:, :, c] * Bap[:, :, c]).sum(0)                   # (ti|ti)
    uptp = torch.einsum("tu,Qup,Qtp->tp", Da, Bap[:, :, c], Bap[:, :, c])
    H_ad = (2.0 * (2.0 * (Fd[a][:, None] - Fd[c][None, :]) + Dtt[:, None] * Fid[c][None, :]
                   - (Qtt + Ztt)[:, None])
            + 2.0 * coul[:, c] + 4.0 * (tupp - ttpp) + 4.0 * exch[:, c] + 12.0 * (tptp - uptp))
    parts = [H_ad.reshape(-1)]
    if active_active:
        Fia = Fi[a, a]
        H_aa = 2.0 * (Dtt[:, None] * torch.diagonal(Fia)[None, :] + Dtt[None, :] * torch.diagonal(Fia)[:, None]
                      - (Qtt + Ztt)[:, None] - (Qtt + Ztt)[None, :] - 2.0 * Da * Fia)
        H_aa = H_aa + _focas_aa_two_electron(B, Ga, nact)
        t_idx, u_idx = torch.tril_indices(nact, nact, offset=-1, device=h.device)
        parts.append(H_aa[t_idx, u_idx])
    parts += [H_ed.reshape(-1), H_ea.reshape(-1)]   # focas's order (Determine_GradIndMap)
    return torch.cat(parts)


def _focas_aa_two_electron(B, Ga, nact):
    """The two-electron part of focas's active-active diagonal Hessian as the
    compiled ComputeH_diag_aa computes it (orbopt_hessian.cc:465-827).  Its
    comment names Shepard's Eq. B27 sums over four-index integrals (tu|rs),
    which the routine forms by DGEMM into a scratch array, but its sums read
    the three-index array tei at those scratch positions instead
    (tei[ttrs_int], tei[uurs_int], tei[turs_int] in the Coulomb part,
    tei[trts_int], tei[urus_int], tei[urts_int] in the exchange part).  With
    L(i, j) the packed index of an active pair (i, j) (i >= j: i (i + 1) / 2
    + j), m = nact (nact + 1) / 2 and T(x, y) = tei[y m + x], tei being the
    factors Q-major over the packed lower triangle of all orbitals
    (tei.cc:281-283) in the current orbitals, it adds for t > u
      sum_rs [T(L_rs, L_tt) G_uurs + T(L_rs, L_uu) G_ttrs - 2 T(L_rs, L_tu) G_turs]
      + 2 sum_rs [T(L_tr, L_ts) G_urus + T(L_ur, L_us) G_trts - 2 T(L_ur, L_ts) G_urts],
    which this function reproduces (the compiled values to 1e-15).  Raises
    when those positions would run past the array, where the reference reads
    out of bounds."""
    n = B.shape[1]
    m = nact * (nact + 1) // 2
    tri = torch.tril_indices(n, n, device=B.device)
    tei = B[:, tri[0], tri[1]].reshape(-1)
    if m * m > tei.numel():
        raise ValueError(f"focas's active-active Hessian reads {m * m} elements of a three-index array "
                         f"of {tei.numel()} (naux too small for {nact} active orbitals)")
    T = tei[:m * m].reshape(m, m)          # T[y, x] = tei[y m + x]
    i = torch.arange(nact, device=B.device)
    hi, lo = torch.maximum(i[:, None], i[None, :]), torch.minimum(i[:, None], i[None, :])
    L = hi * (hi + 1) // 2 + lo            # L[i, j], packed active pair index
    G = Ga
    d = torch.diagonal(L)                  # L_tt
    # Coulomb: C[t, r, s] = T(L_rs, L_tt); Tu[t, u, r, s] = T(L_rs, L_tu)
    C = T[d][:, L]
    Tu = T[L][:, :, L]
    Guu = torch.diagonal(G, dim1=0, dim2=1).permute(2, 0, 1)   # Guu[u, r, s] = G_uurs
    coul = (torch.einsum("trs,urs->tu", C, Guu) + torch.einsum("urs,trs->tu", C, Guu)
            - 2.0 * torch.einsum("turs,turs->tu", Tu, G))
    # exchange: T(L_tr, L_ts) = T[L_ts, L_tr]; T(L_ur, L_ts) = T[L_ts, L_ur]
    X = T[L[:, None, :], L[:, :, None]]    # X[t, r, s] = T[L_ts, L_tr]
    Y = T[L[:, None, None, :], L[None, :, :, None]]   # Y[t, u, r, s] = T[L_ts, L_ur]
    Gxr = torch.einsum("urus->urs", G)     # G_urus as [u, r, s]
    exch = (torch.einsum("trs,urs->tu", X, Gxr) + torch.einsum("urs,trs->tu", X, Gxr)
            - 2.0 * torch.einsum("turs,urts->tu", Y, G))
    return coul + 2.0 * exch


def _pair_kappa(theta, pairs, n):
    p = torch.tensor([x for x, _ in pairs], device=theta.device)
    q = torch.tensor([y for _, y in pairs], device=theta.device)
    K = torch.zeros((n, n), dtype=theta.dtype, device=theta.device)
    K = K.index_put((p, q), theta)
    return K.index_put((q, p), -theta)


def optimize_orbitals_focas(h, B, Da, Ga, ncore, nact, maxiter=10, g_conv=1e-4, e_conv=1e-8,
                            active_active=False):
    """focas's orbital optimisation at fixed densities (src/focas/
    orbopt_optimize.cc:25-96; ORBOPT_MAXITER 10, ORBOPT_GRADIENT_CONVERGENCE
    1e-4, ORBOPT_ENERGY_CONVERGENCE 1e-8 by default, plugin.cc:153-168):

    * with the gradient due: E, g, H at the current orbitals; the quadratic
      model dE_quad = g.k + 1/2 sum H k^2 of the step k held then (zero on
      the first iteration, afterwards the last accepted step:
      Compute_Quadratic_dE runs before Precondition_Step, :162-176); the
      preconditioned step k_ref = -g / max(|H|, 1e-2) (:247-264), k = r k_ref;
    * rotate by exp(k) and take dE = E_new - E (the integrals accumulate the
      rotations, as TransformIntegrals does);
    * stop on |g| < g_conv, |dE| < e_conv or the last iteration;
    * Update_r (:117-146): dE < 0: r *= 1.2 if dE / dE_quad > 0.75, r *= 0.7
      if < 0.25; dE > 0: r *= 0.7 and the gradient is not re-evaluated; the
      next step k' = r k_ref - k, and the saved step accumulates it
      (Update_kappa, :98-115);
    * after the loop, dE > 0 undoes the last step (when converged) and the
      steps since the last gradient (when it was not re-evaluated)
      (Restore_last_step, :226-245).
    Returns U (the product of the rotations), the final energy and a list of
    per-iteration records (E_new, dE, |g|, r)."""
    nmo = h.shape[0]
    nvirt = nmo - ncore - nact
    pairs = rotation_pairs(ncore, nact, nvirt, active_active)
    D, G = full_densities(Da, Ga, ncore, nvirt)
    Gm = G.reshape(nmo * nmo, nmo * nmo)
    zero = torch.zeros((nmo, nmo), dtype=h.dtype, device=h.device)
    Utot = torch.eye(nmo, dtype=h.dtype, device=h.device)

    def rotate(k):
        nonlocal h, B, Utot
        U = torch.linalg.matrix_exp(_pair_kappa(k, pairs, nmo))
        h = df_transform(U, h.unsqueeze(0))[0]
        B = df_transform(U, B)
        Utot = Utot @ U

    def energy():
        return float(RotatedEnergy.apply(zero, h, B, D, Gm))

    r = 1.0
    eval_g = True
    k_cur = torch.zeros(len(pairs), dtype=h.dtype, device=h.device)
    k_ref = k_save = k_cur
    E_init = gnorm = dE = 0.0
    conv_e = conv_g = False
    history = []
    for it in range(maxiter):
        if eval_g:
            E0, g = orbital_gradient(h, B, D, G, pairs)
            E_init = float(E0)
            gnorm = float(torch.sqrt(g @ g))
            Hd = diagonal_hessian(h, B, Da, Ga, ncore, nact, active_active)
            dE_quad = float(0.5 * (2.0 * (g @ k_cur) + (k_cur * Hd * k_cur).sum()))
            k_ref = -g / torch.clamp(Hd.abs(), min=1e-2)
            k_cur = r * k_ref
            k_save = k_cur.clone()
        rotate(k_cur)
        E_new = energy()
        dE = E_new - E_init
        history.append((E_new, dE, gnorm, r))
        conv_g = gnorm < g_conv
        conv_e = abs(dE) < e_conv
        if conv_e or conv_g or it == maxiter - 1:
            break
        eval_g = not (dE > 0.0)
        ratio = dE / dE_quad if dE_quad != 0.0 else (-np.inf if dE < 0 else np.inf)
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
    return Utot, energy(), history


def active_space(h, B, ncore, nact):
    """Frozen-core energy, active one-electron integrals (the inactive Fock
    block) and active (tu|vw) from MO-basis h and DF factors B (torch)."""
    core = slice(0, ncore)
    act = slice(ncore, ncore + nact)
    occ = torch.diagonal(B[:, core, core], dim1=1, dim2=2).sum(1)
    J = torch.einsum("Qpq,Q->pq", B, occ)
    K = torch.einsum("Qpi,Qiq->pq", B[:, :, core], B[:, core, :])
    Fi = h + 2.0 * J - K
    e_core = float((torch.diagonal(h)[core] + torch.diagonal(Fi)[core]).sum())
    Ba = B[:, act, act]
    g = torch.einsum("Qtu,Qvw->tuvw", Ba, Ba)
    return e_core, Fi[act, act], g


def casscf(h, B, ncore, nact, solve_active, macro_iterations=None, active_active=False,
           orbital_step="lbfgs", g_conv=None, e_conv=None, info=None, orbopt_maxiter=10):
    """v2RDM-CASSCF macro-iterations in hilbert's order (v2rdm_solver.cc:1330-1361,
    v2rdm_doci_solver.cc:1111-1137): an SDP solve in the current orbitals, an
    orbital step at its densities, the rotation of h and B, repeated until
    the SDP has converged and the orbital step has met its thresholds.

    solve_active(h_act, g_act) -> (E_active, packed d2, packed d1[, converged])
    on the same device as h: either a full solve (three values, or
    converged True) or, as hilbert runs it, one call of ORBOPT_FREQUENCY
    iterations that continues from the previous call's state (active_solver
    with a frequency).  A solve_active whose ``exhausted`` attribute turns
    true has spent its MAXITER budget and ends the loop.

    orbital_step: "lbfgs" (optimize_orbitals) or "focas"
    (optimize_orbitals_focas with focas's defaults).  The orbital step has
    converged (orbopt_converged_, v2rdm_doci_solver.cc:1753-1762) when its
    total energy change is below e_conv and its final gradient norm below
    g_conv (ORBOPT_ENERGY_CONVERGENCE, ORBOPT_GRADIENT_CONVERGENCE); without
    g_conv and e_conv it never counts as converged.  macro_iterations (None:
    no cap) bounds the rounds of solve and orbital step.  The focas step runs
    at most orbopt_maxiter iterations (ORBOPT_MAXITER) with g_conv and e_conv
    as its own thresholds (focas's defaults 1e-4 and 1e-8 when not given).

    Returns the energies after each SDP solve, the orbital-gradient norms at
    each orbital step (at the solved densities, before the step), and h, B in
    the final orbitals.  ``info`` (a dict, optional) receives sdp_converged,
    orbitals_converged, rounds and final_energy (the energy at the last
    densities in the final orbitals, where hilbert reports it)."""
    if orbital_step not in ("lbfgs", "focas"):
        raise ValueError(f"orbital_step: {orbital_step!r}")
    if macro_iterations is None and (g_conv is None or e_conv is None):
        raise ValueError("give macro_iterations, or g_conv and e_conv to stop on")
    nmo = h.shape[0]
    nvirt = nmo - ncore - nact
    pairs = rotation_pairs(ncore, nact, nvirt, active_active)
    energies, gnorms = [], []
    sdp_conv = orb_conv = False
    e_final = None
    rounds = 0
    while macro_iterations is None or rounds < macro_iterations:
        e_core, h_act, g_act = active_space(h, B, ncore, nact)
        res = solve_active(h_act, g_act)
        e_act, d2p, d1p = res[:3]
        sdp_conv = bool(res[3]) if len(res) > 3 else True
        energies.append(e_core + e_act)
        Da, Ga = unpack_densities(d2p, d1p, nact)
        if orbital_step == "focas":
            U, e_final, hist = optimize_orbitals_focas(
                h, B, Da, Ga, ncore, nact, maxiter=orbopt_maxiter,
                g_conv=1e-4 if g_conv is None else g_conv, e_conv=1e-8 if e_conv is None else e_conv,
                active_active=active_active)
            g_first, g_last = hist[0][2], hist[-1][2]
        else:
            D, G = full_densities(Da, Ga, ncore, nvirt)
            U, e_final, g_first, g_last = optimize_orbitals(h, B, D, G, pairs)
        gnorms.append(g_first)
        h = df_transform(U, h.unsqueeze(0))[0]
        B = df_transform(U, B)
        rounds += 1
        orb_conv = (g_conv is not None and e_conv is not None
                    and abs(e_final - energies[-1]) < e_conv and abs(g_last) < g_conv)
        if (sdp_conv and orb_conv) or getattr(solve_active, "exhausted", False):
            break
    if info is not None:
        info.update(sdp_converged=sdp_conv, orbitals_converged=orb_conv, rounds=rounds,
                    final_energy=e_final)
    return energies, gnorms, h, B


def active_solver(p, options, frequency=None):
    """The active-space SDP solve on the device for casscf, from a problem p
    (v2rdm.V2RDMProblem or DOCIProblem) and its Options.

    frequency None: every call solves from the reference's random guess to
    convergence within MAXITER outer iterations and raises if it does not
    converge.  frequency k (ORBOPT_FREQUENCY): hilbert's schedule.  The first
    call starts from the random guess; every later call continues from the
    x, y, z and mu the previous call left, as libsdp's solver keeps them
    between solve() calls, for at most k outer iterations with mu updated
    after them (sdp_->solve(..., ORBOPT_FREQUENCY, ...),
    v2rdm_doci_solver.cc:1113).  MAXITER bounds the outer iterations of all
    calls together (hilbert hands it to libsdp as SDPOptions.maxiter,
    v2rdm_solver.cc:430); once it is spent without convergence the closure's
    ``exhausted`` attribute turns true.  A call returns (c.x, packed d2,
    packed d1, converged); x is packed as hilbert's PackSpatialDensity."""
    from . import v2rdm
    state = {"x": None, "oiter": 0, "iiter": 0}
    maxiter = int(options.get("MAXITER"))

    def solve(h_act, g_act):
        dev = h_act.device
        b = torch.from_numpy(p.b()).to(dev)
        c = torch.from_numpy(p.c_external(h_act.cpu().numpy(), g_act.cpu().numpy())).to(dev)
        if frequency is None:
            x = torch.from_numpy(p.guess("RANDOM")).to(dev)
            st = p.solve_device(x, b, c, options)
            if not st["converged"]:
                raise RuntimeError(f"the SDP did not converge in MAXITER = {maxiter} iterations")
        else:
            if state["x"] is None:
                state["x"] = torch.from_numpy(p.guess("RANDOM")).to(dev)
            else:
                p.continue_state()
            x = state["x"]
            k = max(1, min(int(frequency), maxiter - state["oiter"]))
            o = v2rdm.Options(dict(options._v))
            o.set("MAXITER", k)
            o.set("MU_UPDATE_FREQUENCY", k)
            st = p.solve_device(x, b, c, o)
            solve.exhausted = (not st["converged"]) and state["oiter"] + st["oiter"] >= maxiter
        state["oiter"] += st["oiter"]
        state["iiter"] += st["iiter"]
        solve.oiter, solve.iiter = state["oiter"], state["iiter"]
        d2p, d1p = p.pack_spatial_density(x)
        return float(c @ x), d2p, d1p, st["converged"]

    solve.problem = p
    solve.exhausted = False
    solve.oiter = solve.iiter = 0
    return solve


def doci_solve_active(nmo, nalpha, nbeta, positivity="DQG", options=None, frequency=None):
    """The active solve of v2RDM-DOCI on the device for casscf: the DOCI
    problem built once (v2rdm_doci_solver.cc:427-700), solved by
    active_solver (each call to convergence, or hilbert's calls of
    ORBOPT_FREQUENCY iterations with the state carried over,
    :1111-1137), its densities packed as hilbert's DOCI
    PackSpatialDensity does (:1568-1703)."""
    from . import v2rdm
    p = v2rdm.DOCIProblem(nmo, nalpha, nbeta, positivity)
    opts = options or v2rdm.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6,
                                     "MAXITER": 100000, "MU_UPDATE_FREQUENCY": 500})
    return active_solver(p, opts, frequency)


def doci_casscf(h, B, nalpha, nbeta, solve_active=None, positivity="DQG", macro_iterations=None,
                g_conv=None, e_conv=None, info=None, orbopt_maxiter=10):
    """Orbital-optimised v2RDM-DOCI: every orbital is active (no core, no
    virtuals) and active-active rotations are on, as hilbert's DOCI
    RotateOrbitals sets focas up (v2rdm_doci_solver.cc:997-1019, 1705-1766).
    solve_active defaults to the device DOCI solve (doci_solve_active)."""
    nmo = h.shape[0]
    if solve_active is None:
        solve_active = doci_solve_active(nmo, nalpha, nbeta, positivity)
    return casscf(h, B, 0, nmo, solve_active, macro_iterations=macro_iterations, active_active=True,
                  orbital_step="focas", g_conv=g_conv, e_conv=e_conv, info=info,
                  orbopt_maxiter=orbopt_maxiter)


def eri_factors(g, rel_tol=1e-12):
    """Exact factors of 4-index integrals for the DF orbital code:
    g[p, q, r, s] = (pq|rs) = sum_Q B[Q, p, q] B[Q, r, s].  (pq|rs) over the
    pairs (pq) is a symmetric positive semidefinite matrix for real orbitals;
    its eigenvectors with eigenvalues above rel_tol * the largest give B.
    This lets the focas step of the density-fitted path run on the
    integrals of hilbert's non-DF path (SCF_TYPE PK, 4-index integrals)."""
    g = torch.as_tensor(g)
    n = g.shape[0]
    M = g.reshape(n * n, n * n)
    M = 0.5 * (M + M.T)
    w, V = torch.linalg.eigh(M)
    top = float(w.max()) if w.numel() else 0.0
    if float(w.min()) < -max(rel_tol * top, 1e-12) * 1e3:
        raise ValueError("the integrals are not positive semidefinite over orbital pairs")
    keep = w > rel_tol * top
    B = (V[:, keep] * torch.sqrt(w[keep])).T.reshape(-1, n, n)
    return B

"""Orbital side of v2RDM-CASSCF: the energy of rotated orbitals from the
v2RDM densities with density-fitted integrals, and its orbital gradient
through a hand-written adjoint of the integral transform.

With U = exp(kappa) (kappa antisymmetric), the transformed integrals are
h' = U^T h U and B'^Q = U^T B^Q U ((pq|rs) = sum_Q B^Q_pq B^Q_rs, focas's DF
transform, src/focas/C_files/orbopt_integraltransform_cpu.cc:25-329), and

    E(kappa) = sum_pq h'_pq D_pq + 1/2 sum_Q b'_Q^T Gm b'_Q,    b'_Q = vec(B'^Q),

with D and Gm (= G_{pq,rs}) the spin-summed core + active densities.
RotatedEnergy's backward does not replay the forward on a tape: it forms
M_Q = Gm b'_Q (= dE/dB'^Q), dE/dU = h U D^T + h^T U D + sum_Q (B^Q U M_Q^T +
B^Q^T U M_Q), and the adjoint of the matrix exponential, L_exp(kappa^T, dE/dU),
as the upper-right block of exp([[kappa^T, dE/dU], [0, kappa^T]]).  At
kappa = 0 the rotation-pair gradient dE/dkappa_pq - dE/dkappa_qp (p > q) is
focas's orbital gradient (orbopt_gradient.cc:26-147: ed = 4 (Fi + Fa),
ea = 2 (Q + Z), ad = 4 (Fi + Fa) - 2 (Q + Z)).

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


class RotatedEnergy(torch.autograd.Function):
    """E(kappa) for U = exp(kappa); backward by the hand-written adjoint."""

    @staticmethod
    def forward(ctx, kappa, h, B, D, Gm):
        n = h.shape[0]
        U = torch.linalg.matrix_exp(kappa)
        hp = U.T @ h @ U
        Bp = U.T @ B @ U                      # (naux, n, n), one GEMM pair per Q
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
        dU = h @ U @ D.T + h.T @ U @ D
        dU = dU + (B @ U @ M.transpose(1, 2)).sum(0) + (B.transpose(1, 2) @ U @ M).sum(0)
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
    """Non-redundant rotation pairs (p, q), p > q, in focas's order: by the
    classes of (p, q) (virtual-core, virtual-active, active-core, then optional
    active-active), then p, then q."""
    core = range(ncore)
    act = range(ncore, ncore + nact)
    virt = range(ncore + nact, ncore + nact + nvirt)
    pairs = [(p, q) for p in virt for q in core]
    pairs += [(p, q) for p in virt for q in act]
    pairs += [(p, q) for p in act for q in core]
    if active_active:
        pairs += [(p, q) for p in act for q in act if q < p]
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


def casscf(h, B, ncore, nact, solve_active, macro_iterations=8, active_active=False):
    """v2RDM-CASSCF macro-iterations: solve the active-space v2RDM in the
    current orbitals (solve_active(h_act, g_act) -> (E_active, packed d2,
    packed d1) on the same device as h), optimise the orbitals at those
    densities, rotate h and B, repeat.  Returns the energies after each SDP
    solve and the orbital-gradient norms at each orbital step."""
    nmo = h.shape[0]
    nvirt = nmo - ncore - nact
    pairs = rotation_pairs(ncore, nact, nvirt, active_active)
    energies, gnorms = [], []
    for _ in range(macro_iterations):
        e_core, h_act, g_act = active_space(h, B, ncore, nact)
        e_act, d2p, d1p = solve_active(h_act, g_act)
        energies.append(e_core + e_act)
        Da, Ga = unpack_densities(d2p, d1p, nact)
        D, G = full_densities(Da, Ga, ncore, nvirt)
        U, _, gn, _ = optimize_orbitals(h, B, D, G, pairs)
        gnorms.append(gn)
        h = U.T @ h @ U
        B = U.T @ B @ U
    return energies, gnorms, h, B

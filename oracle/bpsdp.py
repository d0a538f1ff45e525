"""ORACLE -- test infrastructure only.

numpy restatement of the boundary-point SDP iteration that hilbert drives
through libsdp (``external/libsdp`` is FetchContent-only and absent from the
reference tree, pinned at edeprince3/libsdp@5c17c758ef99a128a54e92c60c1404ebb063e809).
The algorithm is the published one: Povh, Rendl & Wiegele, Computing 78, 277
(2006); Malick, Povh, Rendl & Wiegele, SIAM J. Optim. 20, 336 (2009); as
applied to v2RDM by Mazziotti, PRL 106, 083001 (2011).

Primal  min c.x  s.t. A x = b, x in (+)_k S+^{n_k};  dual  max b.y  s.t. A^T y + z = c, z >= 0.
One outer iteration, penalty mu:
  1. rhs = A(c - z) + mu (b - A x)
  2. solve (A A^T) y = rhs by conjugate gradients, warm-started from the last y,
     stopping when ||r||_2 < cg_convergence or after cg_maxiter iterations
  3. U = mu x + A^T y - c; per PSD block, U_b = V diag(l) V^T of its symmetric part;
     x_b = V diag(max(l,0)) V^T / mu, z_b = -V diag(min(l,0)) V^T
  4. eps_p = ||A x - b||_2, eps_d = ||A^T y + z - c||_2, E_p = c.x, E_d = b.y;
     converged when eps_p, eps_d < r_convergence and |E_p - E_d| < e_convergence.

Outer protocol (v2rdm_solver.cc:1296-1361 and the reference trace
tests/mcpdft/output.ref:495-506, 1021-1024): mu starts at 0.1, stays fixed
inside one ``solve(maxiter)`` call, and afterwards becomes mu * eps_p / eps_d
(e.g. 0.100 * 6.58093e-3 / 4.47092e-5 = 14.719 at oiter 499).
The norms (absolute 2-norms) and the CG stopping rule are this
restatement's choices: libsdp's own are not available to pin them.
"""
import numpy as np


class SDPOptions:
    """Field names follow libsdp::SDPOptions as set at v2rdm_solver.cc:426-431."""

    def __init__(self, sdp_objective_convergence=1e-6, sdp_error_convergence=1e-5,
                 cg_convergence=1e-9, cg_maxiter=10000, maxiter=50):
        self.sdp_objective_convergence = sdp_objective_convergence
        self.sdp_error_convergence = sdp_error_convergence
        self.cg_convergence = cg_convergence
        self.cg_maxiter = cg_maxiter
        self.maxiter = maxiter


def cg_solve(apply, rhs, y, tol, maxiter, split=None):
    """Plain conjugate gradients on the SPD-on-range operator A A^T (warm start y).

    split = (ATu, Au): the step length's denominator p.(A A^T p) is taken as
    ||A^T p||^2, equal in exact arithmetic (the form CG takes on normal
    equations, which the device kernel uses)."""
    r = rhs - apply(y)
    p = r.copy()
    rs = float(r @ r)
    it = 0
    if np.sqrt(rs) < tol:
        return y, 0
    while it < maxiter:
        if split is None:
            Ap = apply(p)
            pAp = float(p @ Ap)
        else:
            t = split[0](p)
            Ap = split[1](t)
            pAp = float(t @ t)
        if pAp <= 0.0:
            break
        alpha = rs / pAp
        y = y + alpha * p
        r = r - alpha * Ap
        rs_new = float(r @ r)
        it += 1
        if np.sqrt(rs_new) < tol:
            break
        p = r + (rs_new / rs) * p
        rs = rs_new
    return y, it


def project_blocks(U, dims, mu, precision="fp64"):
    """Split U into U+ / mu (new x) and -U- (new z), block by block.

    precision "fp64": LAPACK eigh in FP64.  "fp32rr": the eigenvectors from
    an FP32 eigh, then one FP64 Rayleigh-Ritz step: V re-orthonormalised by
    one Newton-Schulz step, T = V^T sym(U) V in FP64, and U+ = V (G o T) V^T
    with G_pq = (f(t_pp) - f(t_qq)) / (t_pp - t_qq), f(t) = max(t, 0) (the
    first-order Daleckii-Krein form, exact on the diagonal and for pairs of
    the same sign).  The precision study of the mixed-precision projection
    runs the whole iteration with it."""
    if precision not in ("fp64", "fp32rr"):
        raise ValueError(f"precision: {precision!r}")
    x = np.empty_like(U)
    z = np.empty_like(U)
    off = 0
    for d in dims:
        d = int(d)
        m = U[off:off + d * d].reshape(d, d)
        m = 0.5 * (m + m.T)
        if precision == "fp64":
            w, v = np.linalg.eigh(m)
            x[off:off + d * d] = ((v * np.maximum(w, 0.0)) @ v.T).ravel() / mu
            z[off:off + d * d] = -((v * np.minimum(w, 0.0)) @ v.T).ravel()
            off += d * d
            continue
        else:
            _, v32 = np.linalg.eigh(m.astype(np.float32))
            v = v32.astype(np.float64)
            v = v @ (1.5 * np.eye(d) - 0.5 * (v.T @ v))
            t = v.T @ m @ v
            dg = np.diag(t).copy()
            fp = np.maximum(dg, 0.0)
            num = fp[:, None] - fp[None, :]
            den = dg[:, None] - dg[None, :]
            g = np.where(den != 0.0, num / np.where(den == 0.0, 1.0, den), (dg[:, None] > 0.0) * 1.0)
            up = v @ (g * t) @ v.T
        x[off:off + d * d] = up.ravel() / mu
        z[off:off + d * d] = (up - m).ravel()
        off += d * d
    return x, z


class BPSDPSolver:
    """libsdp::BPSDPSolver-shaped driver: state (mu, y, z) persists across solve() calls.

    cg_start: "last" starts each CG from the last y; "extrapolate" from the
    polynomial extrapolation through the last solutions of the same solve()
    call (2y - y1 after one, 3y - 3y1 + y2 after two), as the device solve
    does.  Either start reaches the same CG tolerance: only the number of CG
    iterations changes.  precision: the projection's (project_blocks).
    cg_step: "pq" takes the CG step length as r.r / p.(A A^T p), "normal" as
    r.r / ||A^T p||^2 (the device's form; cg_solve)."""

    def __init__(self, n_primal, n_dual, options=None, cg_start="last", precision="fp64", cg_step="pq"):
        if cg_start not in ("last", "extrapolate"):
            raise ValueError(f"cg_start: {cg_start!r}")
        if cg_step not in ("pq", "normal"):
            raise ValueError(f"cg_step: {cg_step!r}")
        self.cg_start = cg_start
        self.cg_step = cg_step
        self.precision = precision
        self.n_primal = int(n_primal)
        self.n_dual = int(n_dual)
        self.options = options or SDPOptions()
        self.mu = 0.1
        self.y = np.zeros(self.n_dual)
        self.z = np.zeros(self.n_primal)
        self._iiter_total = 0
        self._oiter_total = 0
        self._converged = False
        self.primal_error = np.inf
        self.dual_error = np.inf

    def is_converged(self):
        return self._converged

    def iiter_total(self):
        return self._iiter_total

    def oiter_total(self):
        return self._oiter_total

    def solve(self, x, b, c, dims, maxiter, Au, ATu, monitor=None):
        o = self.options
        AAT = lambda v: Au(ATu(v))
        hist = []
        for k in range(int(maxiter)):
            rhs = Au(c - self.z) + self.mu * (b - Au(x))
            y0 = self.y
            if self.cg_start == "extrapolate" and k >= 2:
                y0 = 3.0 * (self.y - hist[-1]) + hist[-2]
            elif self.cg_start == "extrapolate" and k == 1:
                y0 = 2.0 * self.y - hist[-1]
            hist = (hist + [self.y])[-2:]
            self.y, iiter = cg_solve(AAT, rhs, y0, o.cg_convergence, o.cg_maxiter,
                                     split=(ATu, Au) if self.cg_step == "normal" else None)
            ATy = ATu(self.y)
            U = self.mu * x + ATy - c
            xn, self.z = project_blocks(U, dims, self.mu, self.precision)
            x[:] = xn
            self.primal_error = float(np.linalg.norm(Au(x) - b))
            self.dual_error = float(np.linalg.norm(ATy + self.z - c))
            ep = float(c @ x)
            ed = float(b @ self.y)
            self._iiter_total += iiter
            if monitor is not None:
                monitor(self._oiter_total, iiter, ep, ed, self.mu, self.primal_error, self.dual_error)
            self._oiter_total += 1
            self._converged = (self.primal_error < o.sdp_error_convergence
                               and self.dual_error < o.sdp_error_convergence
                               and abs(ep - ed) < o.sdp_objective_convergence)
            if self._converged:
                break
        if not self._converged and self.dual_error > 0.0:
            self.mu = self.mu * self.primal_error / self.dual_error
        return x


def run_v2rdm(problem, x0, options, mu_update_frequency=1000, max_outer=None, monitor=None):
    """hilbert's outer loop for Hubbard / external Hamiltonians (v2rdm_solver.cc:1296-1361):
    call solve(maxiter = MU_UPDATE_FREQUENCY) until converged (bounded by options.maxiter)."""
    solver = BPSDPSolver(problem.n_primal, problem.n_dual, options)
    x = np.array(x0, dtype=np.float64, copy=True)
    total = options.maxiter if max_outer is None else max_outer
    while not solver.is_converged() and solver.oiter_total() < total:
        budget = min(mu_update_frequency, total - solver.oiter_total())
        solver.solve(x, problem.b, problem.c, problem.dims, budget, problem.Au, problem.ATu, monitor)
    return x, solver

"""Warm eigen-refinement of the PSD projection on the B200 against numpy's
LAPACK eigendecomposition, over sequences of slowly changing blocks whose
spectra hold the hard cases: degenerate same-sign clusters, eigenvalues near
zero of both signs, exact zeros."""
import numpy as np
import pytest

import hilbert_b200 as hb
from oracle.bpsdp import project_blocks

pytestmark = pytest.mark.gpu

TOL = 1e-11   # |x - x_ref|_max <= TOL * max(1, |U|_F)


def hard_spectrum(d, rng, zero_frac=0.0):
    lam = rng.uniform(-3.0, 3.0, d)
    if d < 24:   # blocks this small always take the Jacobi kernels
        return lam
    if zero_frac:
        # a large group near zero of both signs: its eigenvectors turn freely
        # from one step to the next, so the whole group forms one cluster
        m = int(zero_frac * d)
        lam[:m] = 1e-8 * rng.standard_normal(m)
        return lam
    k = d // 8
    lam[:k] = 1.0 + 1e-9 * rng.standard_normal(k)                 # degenerate, positive
    lam[k:2 * k] = -0.5 + 1e-10 * rng.standard_normal(k)          # degenerate, negative
    lam[2 * k:3 * k] = 1e-10 * rng.standard_normal(k)             # near zero, both signs
    lam[3 * k] = 0.0
    return lam


def drift(q, rng, step):
    a = rng.standard_normal(q.shape) * step
    a = a - a.T
    r, _ = np.linalg.qr(np.eye(len(q)) + a)
    return q @ (r * np.sign(np.diag(r)))


@pytest.mark.parametrize("n,steps,step,zero_frac", [(6, 12, 1e-4, 0.0), (10, 8, 1e-4, 0.0),
                                                    (10, 6, 3e-3, 0.0), (10, 5, 1e-4, 0.85)])
def test_warm_projection_sequence(cuda_device, n, steps, step, zero_frac):
    import torch
    p = hb.V2RDMProblem(n, n // 2, n // 2)
    rng = np.random.default_rng(100 + n)
    qs = [np.linalg.qr(rng.standard_normal((d, d)))[0] for d in p.dims]
    ls = [hard_spectrum(d, rng, zero_frac) for d in p.dims]
    mu = 0.7
    for it in range(steps):
        U = np.concatenate([((q * l) @ q.T).ravel() for q, l in zip(qs, ls)])
        x, z = p.project(torch.from_numpy(U).to(cuda_device), mu, warm=True)
        xr, zr = project_blocks(U, p.dims, mu)
        scale = max(1.0, np.linalg.norm(U))
        ex = np.max(np.abs(x.cpu().numpy() - xr))
        ez = np.max(np.abs(z.cpu().numpy() - zr))
        assert ex <= TOL * scale and ez <= TOL * scale, (it, ex, ez, scale)
        qs = [drift(q, rng, step) for q in qs]
        ls = [l + 1e-6 * rng.standard_normal(len(l)) for l in ls]
    rc = p.refine_counts()
    # blocks of at least 24 rows are refined after the first (cold) call
    assert rc["accepted"] > 0, rc
    assert rc["passes"] > 0, rc
    if zero_frac:
        # the near-zero groups (85 and 170 rows) went to the Jacobi kernels as clusters
        assert rc["large_clusters"] > 0, rc


def test_cold_projection_resets_warm_basis(cuda_device):
    """A stand-alone projection between warm ones leaves the next warm call cold
    (identity basis) and both stay exact."""
    import torch
    p = hb.V2RDMProblem(6, 3, 3)
    rng = np.random.default_rng(7)
    U = rng.standard_normal(p.n_primal)
    for warm in (True, True, False, True):
        x, z = p.project(torch.from_numpy(U).to(cuda_device), 0.4, warm=warm)
        xr, zr = project_blocks(U, p.dims, 0.4)
        scale = max(1.0, np.linalg.norm(U))
        assert np.max(np.abs(x.cpu().numpy() - xr)) <= TOL * scale
        assert np.max(np.abs(z.cpu().numpy() - zr)) <= TOL * scale
        U = U + 1e-5 * rng.standard_normal(p.n_primal)


def test_mixed_precision_projection_mode_matches_fp64(cuda_device):
    """Projection mode "mixed": blocks above 160 rows that would take
    block-Jacobi sweeps get an FP32 eigensolve, then the FP64 Rayleigh-Ritz
    step and Newton passes.  On a (10e, 10o) DF problem (G2aa block of 200
    rows) the solve converges to the FP64 (mode "refine") energy within
    1e-6 Eh, and the FP32 eigensolve did run."""
    import torch
    from hilbert_b200.synthetic import df_hamiltonian
    p = hb.V2RDMProblem(10, 5, 5, "DQG")
    assert max(p.dims) > 160
    b = torch.from_numpy(p.b()).to(cuda_device)
    c = torch.from_numpy(p.c_external(*df_hamiltonian(10, 400, 4, 5))).to(cuda_device)
    x0 = p.guess("RANDOM")
    opts = hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": 200000,
                       "MU_UPDATE_FREQUENCY": 500})
    e = {}
    for mode in ("refine", "mixed"):
        p.set_projection_mode(mode)
        x = torch.from_numpy(x0).to(cuda_device)
        st = p.solve_device(x, b, c, opts)
        assert st["converged"], mode
        e[mode] = float(c @ x)
    assert abs(e["mixed"] - e["refine"]) <= 1e-6
    assert p.refine_counts()["fp32_eigensolves"] > 0
    p.set_projection_mode("refine")

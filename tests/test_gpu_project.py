"""Per-block PSD projection on the B200 against numpy's LAPACK eigendecomposition."""
import numpy as np
import pytest

import hilbert_b200 as hb
from oracle.bpsdp import project_blocks

pytestmark = pytest.mark.gpu

# eigen-projection tolerance: |x - x_ref|_max <= 1e-11 * max(1, |U|_F)
TOL = 1e-11


@pytest.mark.parametrize("n,na,nb", [(2, 1, 1), (4, 2, 2), (3, 2, 1), (8, 4, 4), (10, 5, 5),
                                     (20, 10, 10)])
def test_projection_matches_lapack(cuda_device, n, na, nb):
    import torch
    p = hb.V2RDMProblem(n, na, nb)
    rng = np.random.default_rng(n)
    U = rng.standard_normal(p.n_primal)          # non-symmetric on purpose
    mu = 0.37
    x, z = p.project(torch.from_numpy(U).to(cuda_device), mu)
    x, z = x.cpu().numpy(), z.cpu().numpy()
    xr, zr = project_blocks(U, p.dims, mu)
    scale = max(1.0, np.linalg.norm(U))
    assert np.max(np.abs(x - xr)) <= TOL * scale
    assert np.max(np.abs(z - zr)) <= TOL * scale


def test_projection_degenerate_and_definite_blocks(cuda_device):
    import torch
    p = hb.V2RDMProblem(4, 2, 2)
    U = np.zeros(p.n_primal)
    off = 0
    rng = np.random.default_rng(5)
    for k, d in enumerate(p.dims):
        if k % 3 == 0:
            m = np.eye(d) * 2.0                       # PSD, degenerate
        elif k % 3 == 1:
            m = -np.eye(d)                            # negative definite
        else:
            q, _ = np.linalg.qr(rng.standard_normal((d, d)))
            m = q @ np.diag(np.repeat([1.0, -1.0], (d + 1) // 2)[:d]) @ q.T   # +-1 clusters
        U[off:off + d * d] = m.ravel()
        off += d * d
    x, z = p.project(torch.from_numpy(U).to(cuda_device), 1.0)
    xr, zr = project_blocks(U, p.dims, 1.0)
    assert np.max(np.abs(x.cpu().numpy() - xr)) <= TOL * 10
    assert np.max(np.abs(z.cpu().numpy() - zr)) <= TOL * 10


def test_large_block_repeated_projection(cuda_device):
    """Repeated cold projections of slowly changing U with a 200-row block (cluster
    Jacobi) match LAPACK each time (the work arrays are reused between calls)."""
    import torch
    p = hb.V2RDMProblem(10, 5, 5)
    rng = np.random.default_rng(3)
    U = rng.standard_normal(p.n_primal)
    for k in range(3):
        U2 = U + 1e-4 * k * rng.standard_normal(p.n_primal)
        x, z = p.project(torch.from_numpy(U2).to(cuda_device), 0.5)
        xr, zr = project_blocks(U2, p.dims, 0.5)
        scale = max(1.0, np.linalg.norm(U2))
        assert np.max(np.abs(x.cpu().numpy() - xr)) <= TOL * scale
        assert np.max(np.abs(z.cpu().numpy() - zr)) <= TOL * scale


def test_split_k_gemm_matches_lapack_and_repeats(cuda_device):
    """The GEMM tiles of blocks of 256 rows or more cut along K (the 288-row
    block of n = 12; the part count is the autotuner's) and in one piece both
    match LAPACK; the split sums its parts in a fixed order, so two
    projections give the same bits."""
    import torch
    p = hb.V2RDMProblem(12, 6, 6)
    assert max(p.dims) >= 256
    rng = np.random.default_rng(12)
    U = rng.standard_normal(p.n_primal)
    xr, zr = project_blocks(U, p.dims, 0.61)
    scale = max(1.0, np.linalg.norm(U))
    out = {}
    for on in (True, False, True):
        p.set_gemm_split(on)
        x, z = p.project(torch.from_numpy(U).to(cuda_device), 0.61)
        x, z = x.cpu().numpy(), z.cpu().numpy()
        assert np.max(np.abs(x - xr)) <= TOL * scale, on
        assert np.max(np.abs(z - zr)) <= TOL * scale, on
        if on in out:
            assert np.array_equal(out[on][0], x) and np.array_equal(out[on][1], z)
        out[on] = (x, z)
    full, upper = p.gemm_split_choice()   # the autotuner's part counts
    assert full in (1, 2, 4) and upper in (1, 2, 4)

"""The allocation-free projection entry point, for callers that cannot call
cudaMalloc (their host owns all device memory, or an allocation's device
synchronisation is not acceptable where they project).

It must give the same x = U+/mu and z = U+ - sym(U) as the library's own
projection entry point (which allocates its working buffers), on two calls in
a row through the same static scratch array.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

import hilbert_b200 as hb
from hilbert_b200 import _capi

pytestmark = pytest.mark.gpu

# same tolerance as the projection tests: |dx|max <= 1e-11 * max(1, |U|_F)
TOL = 1e-11


def _noalloc(lib, dU, off, n, mu, x, z, stream):
    return lib.v2b_project_block_noalloc(ctypes.c_void_p(dU.data_ptr() + 8 * off), n, mu,
                                         ctypes.c_void_p(x.data_ptr() + 8 * off),
                                         ctypes.c_void_p(z.data_ptr() + 8 * off),
                                         ctypes.c_void_p(stream))


def test_noalloc_projection_matches_library_projection(cuda_device):
    import torch
    lib = _capi.load()
    p = hb.V2RDMProblem(8, 4, 4)          # PSD blocks of 8, 28, 64 and 128 rows
    rng = np.random.default_rng(21)
    U = rng.standard_normal(p.n_primal)   # not symmetric on purpose
    mu = 0.37
    dU = torch.from_numpy(U).to(cuda_device)
    xr, zr = p.project(dU, mu)
    xr, zr = xr.cpu().numpy(), zr.cpu().numpy()
    scale = max(1.0, np.linalg.norm(U))
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        x = torch.full_like(dU, float("nan"))
        z = torch.full_like(dU, float("nan"))
        off = 0
        for n in p.dims:
            n = int(n)
            rc = _noalloc(lib, dU, off, n, mu, x, z, stream)
            assert rc == _capi.V2B_OK, lib.v2b_last_error()
            off += n * n
        torch.cuda.synchronize()
        xn, zn = x.cpu().numpy(), z.cpu().numpy()
        assert np.all(np.isfinite(xn)) and np.all(np.isfinite(zn))
        assert np.max(np.abs(xn - xr)) <= TOL * scale, f"call {call}"
        assert np.max(np.abs(zn - zr)) <= TOL * scale, f"call {call}"


def test_noalloc_rejects_sizes_beyond_its_array(cuda_device):
    import torch
    lib = _capi.load()
    d = torch.zeros(130 * 130, dtype=torch.float64, device=cuda_device)
    stream = torch.cuda.current_stream().cuda_stream
    for n in (0, 129):
        rc = _noalloc(lib, d, 0, n, 1.0, d, d, stream)
        assert rc == _capi.V2B_BAD_ARG
        assert "outside 1..128" in lib.v2b_last_error().decode()

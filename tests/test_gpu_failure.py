"""Failure detection on the device without a fault: a grid-barrier wait that
runs out returns V2B_DEVICE_TIMEOUT and leaves the context usable; a NaN in
the device inputs returns V2B_NAN before the first iteration."""
import numpy as np
import pytest

import hilbert_b200 as hb
from hilbert_b200 import _capi

pytestmark = pytest.mark.gpu


def ring(L=6):
    p = hb.V2RDMProblem(L, L // 2, L // 2, "DQG", hubbard_multiplicity=True)
    return p, p.b(), p.c_hubbard(1.0, 4.0)


def test_barrier_wait_that_runs_out_returns_timeout(cuda_device):
    """With a wait limit of one poll, the first CTA that waits at a CG grid
    barrier gives up: the solve returns DEVICE_TIMEOUT.  With the default
    limit the same problem then solves to convergence in the same context."""
    import torch
    p, b, c = ring(6)
    opts = hb.Options({"R_CONVERGENCE": 1e-5, "E_CONVERGENCE": 1e-5, "MAXITER": 200000,
                       "MU_UPDATE_FREQUENCY": 500})
    dev = cuda_device
    db, dc = torch.from_numpy(b).to(dev), torch.from_numpy(c).to(dev)
    x = torch.from_numpy(p.guess("RANDOM")).to(dev)
    p.set_wait_limit(1)
    with pytest.raises(_capi.V2BError) as e:
        p.solve_device(x, db, dc, opts)
    assert e.value.code == _capi.V2B_DEVICE_TIMEOUT
    assert "grid barrier" in str(e.value)
    p.set_wait_limit(0)
    x = torch.from_numpy(p.guess("RANDOM")).to(dev)
    st = p.solve_device(x, db, dc, opts)
    assert st["converged"]
    torch.cuda.synchronize()
    p.close()


@pytest.mark.parametrize("which", ["x", "b", "c"])
def test_nonfinite_device_input_returns_nan(cuda_device, which):
    import torch
    p, b, c = ring(4)
    x = p.guess("RANDOM")
    vec = {"x": x, "b": b, "c": c}[which]
    vec[11] = np.nan
    dev = cuda_device
    launches = p.kernel_launches()
    with pytest.raises(_capi.V2BError) as e:
        p.solve_device(torch.from_numpy(x).to(dev), torch.from_numpy(b).to(dev),
                       torch.from_numpy(c).to(dev), hb.Options({"MAXITER": 5}))
    assert e.value.code == _capi.V2B_NAN
    assert f"non-finite value in {which} at index 11" in str(e.value)
    assert p.kernel_launches() - launches <= 2   # the check itself; no iteration ran
    p.close()

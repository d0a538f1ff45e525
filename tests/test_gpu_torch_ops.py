"""torch.ops.v2rdm on the B200: the operators equal the problem's own device
calls bit for bit, their autograd rules are each other's adjoint, and the
solve operator equals solve_device."""
import pytest

torch = pytest.importorskip("torch")

import hilbert_b200 as hb  # noqa: E402
import hilbert_b200.torch_ops  # noqa: E402,F401

pytestmark = pytest.mark.gpu

SPEC = (4, 2, 2, "DQG", True, True, True)


def _problem():
    return hb.V2RDMProblem(4, 2, 2, "DQG", True, True, hubbard_multiplicity=True)


def test_map_operators_and_their_adjoints(cuda_device):
    p = _problem()
    g = torch.Generator().manual_seed(0)
    x = torch.randn(p.n_primal, dtype=torch.float64, generator=g).to(cuda_device)
    y = torch.randn(p.n_dual, dtype=torch.float64, generator=g).to(cuda_device)
    assert torch.equal(torch.ops.v2rdm.Au(x, *SPEC), p.Au(x))
    assert torch.equal(torch.ops.v2rdm.ATu(y, *SPEC), p.ATu(y))
    xr = x.clone().requires_grad_(True)
    (torch.ops.v2rdm.Au(xr, *SPEC) @ y).backward()
    assert torch.equal(xr.grad, p.ATu(y))
    yr = y.clone().requires_grad_(True)
    (torch.ops.v2rdm.ATu(yr, *SPEC) @ x).backward()
    assert torch.equal(yr.grad, p.Au(x))


def test_solve_operator_matches_solve_device(cuda_device):
    p = _problem()
    x0 = torch.from_numpy(p.guess("RANDOM")).to(cuda_device)
    b = torch.from_numpy(p.b()).to(cuda_device)
    c = torch.from_numpy(p.c_hubbard(1.0, 4.0)).to(cuda_device)
    out = torch.ops.v2rdm.solve(x0, b, c, *SPEC, 1e-6, 1e-6, 100000, 500, 1e-9, 10000)
    x = x0.clone()
    st = p.solve_device(x, b, c, hb.Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6,
                                             "MAXITER": 100000, "MU_UPDATE_FREQUENCY": 500,
                                             "CG_CONVERGENCE": 1e-9, "CG_MAXITER": 10000}))
    assert st["converged"]
    assert torch.equal(out, x)
    assert not torch.equal(out, x0)

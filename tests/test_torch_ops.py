"""torch.ops.v2rdm.{Au, ATu, solve} without a GPU: registration, shape
inference on meta tensors, and no CPU fallback."""
import pytest

torch = pytest.importorskip("torch")

import hilbert_b200 as hb  # noqa: E402
import hilbert_b200.torch_ops  # noqa: E402,F401  (registers the operators)

SPEC = (4, 2, 2, "DQG", True, True, True)


def test_operators_are_registered():
    for name in ("Au", "ATu", "solve"):
        assert hasattr(torch.ops.v2rdm, name)


def test_shapes_from_meta_tensors():
    p = hb.V2RDMProblem(4, 2, 2, "DQG", True, True, hubbard_multiplicity=True)
    x = torch.empty(p.n_primal, dtype=torch.float64, device="meta")
    y = torch.empty(p.n_dual, dtype=torch.float64, device="meta")
    assert torch.ops.v2rdm.Au(x, *SPEC).shape == (p.n_dual,)
    assert torch.ops.v2rdm.ATu(y, *SPEC).shape == (p.n_primal,)
    c = torch.empty(p.n_primal, dtype=torch.float64, device="meta")
    out = torch.ops.v2rdm.solve(x, y, c, *SPEC, 1e-6, 1e-6, 100, 50, 1e-9, 1000)
    assert out.shape == (p.n_primal,)


def test_cpu_tensors_are_refused():
    p = hb.V2RDMProblem(4, 2, 2, "DQG", True, True, hubbard_multiplicity=True)
    x = torch.zeros(p.n_primal, dtype=torch.float64)
    with pytest.raises((NotImplementedError, RuntimeError)):
        torch.ops.v2rdm.Au(x, *SPEC)


def test_clear_releases_cached_problems():
    from hilbert_b200 import torch_ops
    p = hb.V2RDMProblem(2, 1, 1, "DQG", True, True, hubbard_multiplicity=True)
    torch_ops._problems[("test",)] = p
    torch_ops.clear()
    assert not torch_ops._problems and p._h is None


def test_doci_operators_shapes_and_no_cpu_fallback():
    p = hb.DOCIProblem(4, 2, 2, "DQG+D3")
    x = torch.empty(p.n_primal, dtype=torch.float64, device="meta")
    y = torch.empty(p.n_dual, dtype=torch.float64, device="meta")
    assert torch.ops.v2rdm.doci_Au(x, 4, 2, 2, "DQG+D3").shape == (p.n_dual,)
    assert torch.ops.v2rdm.doci_ATu(y, 4, 2, 2, "DQG+D3").shape == (p.n_primal,)
    with pytest.raises((NotImplementedError, RuntimeError)):
        torch.ops.v2rdm.doci_Au(torch.zeros(p.n_primal, dtype=torch.float64), 4, 2, 2, "DQG+D3")

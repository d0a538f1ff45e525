"""A.x and A^T.y on the B200 through the C ABI: bit-exact to hilbert's maps."""
import numpy as np
import pytest

from conftest import case_kwargs
import hilbert_b200 as hb
from oracle.maps import OracleProblem

pytestmark = pytest.mark.gpu


def gpu_problem(kw):
    return hb.V2RDMProblem(kw["n"], kw["na"], kw["nb"], kw["positivity"], kw["constrain_spin"],
                           kw["constrain_sz"], hubbard_multiplicity="hubbard" in kw)


@pytest.mark.parametrize("name", ["hub2_dqg", "hub4_dqg", "hub4_d_nospin", "ext3_dqg_triplet",
                                  "ext4_dq_nosz", "ext4_dg_doublet", "ext5_dqg", "ext1_dqg",
                                  "hub3_dqgt2", "ext3_dqgt2_doublet", "hub4_dqgt1",
                                  "ext4_dqgt1t2_doublet", "hub4_dqg_d3", "ext3_d_d3_nosz_doublet",
                                  "ext3_dqg_q3_doublet", "hub3_d_e3", "ext3_d_f3_doublet",
                                  "ext4_d_d4_quartet"])
def test_maps_bit_exact_golden(golden, cuda_device, name):
    import torch
    case = golden[name]
    p = gpu_problem(case_kwargs(case))
    x = torch.from_numpy(case["x"]).to(cuda_device)
    y = torch.from_numpy(case["y"]).to(cuda_device)
    ax = p.Au(x).cpu().numpy()
    aty = p.ATu(y).cpu().numpy()
    torch.cuda.synchronize()
    assert np.array_equal(ax, case["Ax"])
    assert np.array_equal(aty, case["ATy"])


@pytest.mark.parametrize("n,na,nb,pos,spin,sz", [(8, 4, 4, "DQG", 1, 1), (7, 4, 3, "DQG", 1, 1),
                                                 (6, 3, 3, "DQG", 0, 0), (9, 5, 4, "DG", 1, 0),
                                                 (20, 10, 10, "DQG", 1, 1)])
def test_maps_bit_exact_vs_oracle(cuda_device, n, na, nb, pos, spin, sz):
    import torch
    rng = np.random.default_rng(n * 100 + na)
    h = rng.standard_normal((n, n))
    g = rng.standard_normal((n,) * 4)
    o = OracleProblem(n, na, nb, pos, spin, sz, h=h, g=g)
    p = hb.V2RDMProblem(n, na, nb, pos, bool(spin), bool(sz))
    assert (p.n_primal, p.n_dual) == (o.n_primal, o.n_dual)
    x = rng.standard_normal(o.n_primal)
    y = rng.standard_normal(o.n_dual)
    ax = p.Au(torch.from_numpy(x).to(cuda_device)).cpu().numpy()
    aty = p.ATu(torch.from_numpy(y).to(cuda_device)).cpu().numpy()
    assert np.array_equal(ax, o.Au(x))
    assert np.array_equal(aty, o.ATu(y))
    # adjoint identity as a size-independent property
    assert abs(float(ax @ y) - float(x @ aty)) <= 1e-10 * max(1.0, abs(float(ax @ y)))


def test_maps_on_torch_stream(cuda_device):
    import torch
    p = hb.V2RDMProblem(6, 3, 3)
    s = torch.cuda.Stream()
    x = torch.randn(p.n_primal, dtype=torch.float64, device=cuda_device)
    with torch.cuda.stream(s):
        a1 = p.Au(x)
    s.synchronize()
    a2 = p.Au(x)
    torch.cuda.synchronize()
    assert torch.equal(a1, a2)

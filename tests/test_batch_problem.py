"""Independent problems as one block-diagonal problem (v2b_batch_problem_create),
on the CPU: the joint operator is the parts' operators along the diagonal, bit
for bit, and the joint SDP's optimum is the parts' optima."""
import ctypes
import types

import numpy as np
import pytest

import hilbert_b200 as hb
from hilbert_b200 import _capi
from oracle.bpsdp import SDPOptions, run_v2rdm
from oracle.maps import OracleProblem
from test_host_problem import operator, packed_apply


def parts():
    return [hb.V2RDMProblem(4, 2, 2, "DQG", True, True, hubbard_multiplicity=True),
            hb.V2RDMProblem(3, 2, 1, "DQG"),
            hb.DOCIProblem(4, 2, 2, "DQG"),
            hb.V2RDMProblem(3, 1, 1, "DQGT2")]


def test_batch_operator_is_block_diagonal():
    ps = parts()
    batch = hb.BatchProblem(ps)
    assert batch.n_primal == sum(p.n_primal for p in ps) and batch.n_dual == sum(p.n_dual for p in ps)
    assert list(batch.dims) == [int(d) for p in ps for d in p.dims]
    rng = np.random.default_rng(4)
    x, y = rng.standard_normal(batch.n_primal), rng.standard_normal(batch.n_dual)
    rp, ent, pal = operator(batch, False)
    got = batch.split(packed_apply(rp, ent, pal, x), dual=True)
    for p, xp, g in zip(ps, batch.split(x), got):
        assert np.array_equal(g, packed_apply(*operator(p, False), xp))
    rp, ent, pal = operator(batch, True)
    got = batch.split(packed_apply(rp, ent, pal, y))
    for p, yp, g in zip(ps, batch.split(y, dual=True), got):
        assert np.array_equal(g, packed_apply(*operator(p, True), yp))
    batch.close()
    for p in ps:
        p.close()


def test_batch_refuses_what_belongs_to_the_parts():
    ps = parts()
    batch = hb.BatchProblem(ps)
    for call in (batch.b, lambda: batch.guess("RANDOM"), lambda: batch.c_hubbard(1.0, 4.0),
                 lambda: batch.rdm_records(np.zeros(batch.n_primal))):
        with pytest.raises(hb.V2BError):
            call()
    d2, d1 = ctypes.c_long(), ctypes.c_long()
    assert batch._lib.v2b_problem_pack_dims(batch._h, ctypes.byref(d2), ctypes.byref(d1)) == _capi.V2B_BAD_ARG
    with pytest.raises(hb.V2BError):
        hb.BatchProblem([batch])   # a batch is not a part
    batch.close()


def test_batch_palette_overflow_is_an_error():
    """Each electron count adds its own contraction coefficients; enough of
    them overflow one 16-entry palette."""
    ps = [hb.V2RDMProblem(12, k, k, "DQG") for k in range(1, 13)]
    with pytest.raises(hb.V2BError, match="palette"):
        hb.BatchProblem(ps)


def test_joint_solve_reaches_the_parts_optima():
    """The numpy oracle on the joint problem of two rings against each ring
    alone (|dE| <= 1e-6 per part)."""
    probs = [OracleProblem(2, 1, 1, "DQG", True, True, hubbard=(1.0, 4.0)),
             OracleProblem(3, 1, 1, "DQG", True, True, hubbard=(1.0, 2.0))]
    opts = SDPOptions(1e-7, 1e-7, 1e-10, 10000, 100000)
    alone = []
    for p in probs:
        x, s = run_v2rdm(p, p.guess("random"), opts, 500)
        assert s.is_converged()
        alone.append(float(p.c @ x))
    po = np.cumsum([0] + [p.n_primal for p in probs])
    do = np.cumsum([0] + [p.n_dual for p in probs])
    joint = types.SimpleNamespace(
        n_primal=int(po[-1]), n_dual=int(do[-1]), b=np.concatenate([p.b for p in probs]),
        c=np.concatenate([p.c for p in probs]), dims=[d for p in probs for d in p.dims],
        Au=lambda x: np.concatenate([p.Au(x[po[k]:po[k + 1]]) for k, p in enumerate(probs)]),
        ATu=lambda y: np.concatenate([p.ATu(y[do[k]:do[k + 1]]) for k, p in enumerate(probs)]))
    x, s = run_v2rdm(joint, np.concatenate([p.guess("random") for p in probs]), opts, 500)
    assert s.is_converged()
    for k, p in enumerate(probs):
        assert abs(float(p.c @ x[po[k]:po[k + 1]]) - alone[k]) <= 1e-6


def test_launch_groups_keep_palettes_within_sixteen():
    from hilbert_b200.batch import hubbard_batch, launch_groups
    insts = hubbard_batch(count=64)
    probs = [inst.problem()[0] for inst in insts]
    groups = launch_groups(probs)
    assert [k for g in groups for k in g] == list(range(64))
    assert len(groups) == 1   # the 64 rings share 14 coefficients
    over = [hb.V2RDMProblem(12, k, k, "DQG") for k in range(1, 13)]
    groups = launch_groups(over)
    assert len(groups) > 1 and [k for g in groups for k in g] == list(range(12))
    for g in groups:
        assert len(set().union(*[over[k].palette() for k in g])) <= 16
        hb.BatchProblem([over[k] for k in g]).close()
    for p in probs + over:
        p.close()

"""Batches of independent ring instances: the seeded workload, the shard
across ranks, the Hamiltonian each instance builds (against the oracle), and
the host gather over two gloo ranks on the CPU (a stand-in solve; the device
solve is the one the GPU tests cover)."""
import os
import socket

import numpy as np
import pytest

from hilbert_b200.batch import RingInstance, hubbard_batch, shard, solve_batch
from oracle.maps import OracleProblem


def test_batch_is_seeded_and_in_range():
    a, b = hubbard_batch(), hubbard_batch()
    assert a == b and len(a) == 64
    assert [i.index for i in a] == list(range(64))
    for i in a:
        assert 6 <= i.sites <= 14 and i.electrons - i.sites in (-2, 0, 2) and 1.0 <= i.U <= 8.0
        assert i.nalpha + i.nbeta == i.electrons and i.nalpha - i.nbeta == i.electrons % 2
    assert any(i.hubbard_path for i in a) and any(not i.hubbard_path for i in a)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_covers_every_instance_once_and_balances(world):
    batch = hubbard_batch()
    parts = shard(batch, world)
    assert sorted(k for p in parts for k in p) == list(range(len(batch)))
    cost = {i.index: i.cost() for i in batch}
    loads = [sum(cost[k] for k in p) for p in parts]
    assert max(loads) - min(loads) <= max(cost.values())   # longest-first bound


@pytest.mark.parametrize("inst", [RingInstance(0, 6, 6, 3.5), RingInstance(1, 7, 5, 2.25),
                                  RingInstance(2, 7, 9, 6.0)])
def test_instance_hamiltonian_matches_the_oracle(inst):
    p, b, c = inst.problem()
    if inst.hubbard_path:
        o = OracleProblem(inst.sites, inst.nalpha, inst.nbeta, "DQG", True, True, hubbard=(1.0, inst.U))
    else:
        h, g = inst.integrals()
        o = OracleProblem(inst.sites, inst.nalpha, inst.nbeta, "DQG", True, True, h=h, g=g)
    assert (p.n_primal, p.n_dual) == (o.n_primal, o.n_dual)
    assert np.array_equal(b, o.b) and np.array_equal(c, o.c)


def _fake_solve(inst, options):
    return {"energy": -float(inst.index) - inst.U, "converged": True, "oiter": inst.sites,
            "iiter": inst.electrons}


def _rank_main(rank, world, port, out_dir, one_launch=False):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = solve_batch(hubbard_batch(), rank=rank, world=world, solve=_fake_solve,
                          one_launch=one_launch, solve_slice=_fake_slice)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"),
                np.array([(r["index"], r["rank"], r["energy"], r["oiter"]) for r in res]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("one_launch", [False, True])
def test_two_gloo_ranks_gather_every_result(tmp_path, one_launch):
    torch = pytest.importorskip("torch")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    torch.multiprocessing.spawn(_rank_main, args=(2, port, str(tmp_path), one_launch), nprocs=2, join=True)
    r0, r1 = (np.load(tmp_path / f"rank{k}.npy") for k in (0, 1))
    assert np.array_equal(r0, r1)
    batch = hubbard_batch()
    parts = shard(batch, 2)
    assert list(r0[:, 0].astype(int)) == list(range(64))
    for k, rank in zip(r0[:, 0].astype(int), r0[:, 1].astype(int)):
        assert k in parts[rank]
    assert np.array_equal(r0[:, 2], [-float(i.index) - i.U for i in batch])


def test_concurrent_slice_gives_the_same_results():
    """concurrency > 1 runs a rank's instances from host threads; the results
    and their order do not change."""
    import threading
    seen = set()

    def solve(inst, options):
        seen.add(threading.get_ident())
        return _fake_solve(inst, options)

    batch = hubbard_batch(count=12)
    a = solve_batch(batch, solve=_fake_solve)
    b = solve_batch(batch, solve=solve, concurrency=4)
    assert a == b and [r["index"] for r in b] == list(range(12))



def _fake_slice(insts, options):
    return [_fake_solve(i, options) for i in insts]


def test_one_launch_slice_gives_the_same_results():
    """one_launch=True hands the rank's whole slice to one slice solver and
    keeps the per-instance results and their order."""
    calls = []

    def solve_slice(insts, options):
        calls.append(len(insts))
        return _fake_slice(insts, options)

    batch = hubbard_batch(count=12)
    assert solve_batch(batch, one_launch=True, solve_slice=solve_slice) == solve_batch(batch, solve=_fake_solve)
    assert calls == [12]

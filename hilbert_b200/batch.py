"""Batches of independent v2RDM instances, sharded across GPUs.

The instances of a batch share no data, so a batch runs as replicas: each
rank solves a disjoint slice on its own device, and the host gathers the
per-instance scalars (energy, convergence, iteration counts).  No device
collective takes part.

hubbard_batch() draws the 64-ring workload: L ~ U{6..14} sites, N in
{L-2, L, L+2} electrons, U/t ~ U[1, 8], periodic, seed 3.  Even N runs
through hilbert's Hubbard path (nalpha = nbeta = N/2,
v2rdm_solver.cc:841-863).  Odd N runs through the external-Hamiltonian
constructor with the ring's integrals and nalpha = ceil(N/2), nbeta =
floor(N/2) (v2rdm_solver.cc:147-195), because the Hubbard path requires
even N.
"""
from dataclasses import dataclass

import numpy as np

from .v2rdm import BatchProblem, Options, V2RDMProblem, block_layout


@dataclass(frozen=True)
class RingInstance:
    index: int
    sites: int        # L, one orbital per site
    electrons: int    # N
    U: float          # on-site repulsion, in units of t = 1
    positivity: str = "DQG"

    @property
    def nalpha(self):
        return (self.electrons + 1) // 2

    @property
    def nbeta(self):
        return self.electrons // 2

    @property
    def hubbard_path(self):
        return self.electrons % 2 == 0

    def cost(self):
        """Relative work of a solve: the projection's sum (16/3) n_b^3."""
        dims = [d for _, d in block_layout(self.sites, self.nalpha, self.nbeta, self.positivity, True)]
        return float(sum((16.0 / 3.0) * float(d) ** 3 for d in dims))

    def integrals(self):
        """(h, g) of the periodic ring: h_{i,i+-1} = -1 (once for L = 2,
        oei.cc:76-95), (ii|ii) = U (tei.cc:285-292); g in (pq|rs) order."""
        L = self.sites
        h = np.zeros((L, L))
        for i in range(L):
            j = (i + 1) % L
            if j != i:
                h[i, j] = h[j, i] = -1.0
        g = np.zeros((L, L, L, L))
        for i in range(L):
            g[i, i, i, i] = self.U
        return h, g

    def problem(self):
        """The device problem and its b and c (host arrays)."""
        p = V2RDMProblem(self.sites, self.nalpha, self.nbeta, self.positivity, True, True,
                         hubbard_multiplicity=self.hubbard_path)
        c = p.c_hubbard(1.0, self.U) if self.hubbard_path else p.c_external(*self.integrals())
        return p, p.b(), c


def hubbard_batch(count=64, seed=3, positivity="DQG"):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        L = int(rng.integers(6, 15))
        N = L + int(rng.choice([-2, 0, 2]))
        U = float(rng.uniform(1.0, 8.0))
        out.append(RingInstance(k, L, N, U, positivity))
    return out


def shard(instances, world):
    """Instance indices per rank: longest first, each to the least-loaded
    rank (ties to the lower rank); every instance exactly once."""
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for inst in sorted(instances, key=lambda i: (-i.cost(), i.index)):
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(inst.index)
        loads[r] += inst.cost()
    return [sorted(p) for p in parts]


def solve_on_device(inst, options, device=None):
    """One instance through the device path from the RANDOM guess."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    with torch.cuda.device(dev):
        p, b, c = inst.problem()
        try:
            x = torch.from_numpy(p.guess("RANDOM")).to(dev)
            st = p.solve_device(x, torch.from_numpy(b).to(dev), torch.from_numpy(c).to(dev), options)
            energy = float(np.dot(c, x.cpu().numpy()))
        finally:
            p.close()
    return {"energy": energy, "converged": bool(st["converged"]), "oiter": int(st["oiter"]),
            "iiter": int(st["iiter"])}


def launch_groups(problems, capacity=16):
    """Indices of problems grouped for BatchProblem, in order: a group grows
    while the union of its parts' A and A^T palettes each stays within
    `capacity` coefficients."""
    groups, pal_a, pal_at = [], set(), set()
    for k, p in enumerate(problems):
        a, at = p.palette(False), p.palette(True)
        if groups and len(pal_a | a) <= capacity and len(pal_at | at) <= capacity:
            groups[-1].append(k)
            pal_a |= a
            pal_at |= at
        else:
            groups.append([k])
            pal_a, pal_at = set(a), set(at)
    return groups


def solve_in_one_launch(instances, options=None, device=None):
    """This rank's instances solved together, one BatchProblem per palette
    group: every device launch of the iteration covers all of a group's
    instances.  Each instance starts from its own random guess; the results
    are those of solve_on_device, per instance, in input order, plus the
    group's shared outer and CG iteration counts."""
    import torch
    if options is None:
        options = Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": 400000,
                           "MU_UPDATE_FREQUENCY": 500})
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    built = [inst.problem() for inst in instances]
    results = [None] * len(instances)
    with torch.cuda.device(dev):
        for group in launch_groups([p for p, _, _ in built]):
            parts = [built[k] for k in group]
            batch = BatchProblem([p for p, _, _ in parts])
            try:
                x = torch.from_numpy(np.concatenate([p.guess("RANDOM") for p, _, _ in parts])).to(dev)
                b = torch.from_numpy(np.concatenate([b for _, b, _ in parts])).to(dev)
                c = np.concatenate([c for _, _, c in parts])
                st = batch.solve_device(x, b, torch.from_numpy(c).to(dev), options)
                for k, xk, (_, _, ck) in zip(group, batch.split(x), parts):
                    results[k] = {"energy": float(np.dot(ck, xk)), "converged": bool(st["converged"]),
                                  "oiter": int(st["oiter"]), "iiter": int(st["iiter"]),
                                  "group": len(group)}
            finally:
                batch.close()
    for p, _, _ in built:
        p.close()
    return results


def solve_batch(instances, options=None, rank=0, world=1, group=None, solve=solve_on_device,
                concurrency=1, one_launch=False, solve_slice=solve_in_one_launch):
    """Solve this rank's slice, then gather every rank's results on the host
    (torch.distributed.all_gather_object over `group`, which should be a
    gloo group when the default one is NCCL).  Returns the results of all
    instances, ordered by index, each {"index", "rank", ...solve's dict}.

    concurrency > 1 solves that many of the slice's instances at a time from
    host threads: every problem runs on its own CUDA stream and the library
    calls release the GIL, so small instances can share the GPU.  A new
    thread starts on CUDA device 0, so each worker first takes the caller's
    current device.

    one_launch=True solves the whole slice together instead, with
    solve_slice(instances, options) (default solve_in_one_launch: one
    block-diagonal problem per palette group, every launch covering them)."""
    if options is None:
        options = Options({"R_CONVERGENCE": 1e-6, "E_CONVERGENCE": 1e-6, "MAXITER": 400000,
                           "MU_UPDATE_FREQUENCY": 500})
    by_index = {i.index: i for i in instances}
    if len(by_index) != len(instances):
        raise ValueError("instance indices must be unique")
    mine = shard(instances, world)[rank]

    def one(k):
        r = dict(solve(by_index[k], options))
        r.update(index=k, rank=rank)
        return r

    if one_launch:
        results = []
        if mine:
            for k, r in zip(mine, solve_slice([by_index[k] for k in mine], options)):
                r = dict(r)
                r.update(index=k, rank=rank)
                results.append(r)
    elif concurrency > 1 and len(mine) > 1:
        from concurrent.futures import ThreadPoolExecutor
        init = None
        import torch
        if torch.cuda.is_available():
            dev = torch.cuda.current_device()
            init = lambda: torch.cuda.set_device(dev)   # noqa: E731
        with ThreadPoolExecutor(max_workers=int(concurrency), initializer=init) as pool:
            results = list(pool.map(one, mine))
    else:
        results = [one(k) for k in mine]
    if world > 1:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, results, group=group)
        results = [r for part in gathered for r in part]
    return sorted(results, key=lambda r: r["index"])


def main(argv=None):
    """python -m hilbert_b200.batch [--count 64] [--mode one-launch|sequential|both] [--maxiter N]
    Solves the seeded ring batch on this process's GPU and prints one JSON
    line: wall time per mode (CUDA-synchronised, problem set-up included),
    instances converged, outer iterations, and the largest energy difference
    between the modes.  --maxiter caps the outer iterations of every solve
    (hilbert's MAXITER) for a bounded run."""
    import argparse
    import json
    import time

    import torch

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--mode", choices=("one-launch", "sequential", "both"), default="both")
    ap.add_argument("--r-convergence", type=float, default=1e-6)
    ap.add_argument("--maxiter", type=int, default=400000)
    args = ap.parse_args(argv)
    if not torch.cuda.is_available():
        raise SystemExit("hilbert_b200.batch: needs a CUDA device")
    insts = hubbard_batch(count=args.count)
    opts = Options({"R_CONVERGENCE": args.r_convergence, "E_CONVERGENCE": args.r_convergence,
                    "MAXITER": args.maxiter, "MU_UPDATE_FREQUENCY": 500})
    out = {"workload": f"{args.count} Hubbard rings (L 6-14, seed 3), DQG", "r_convergence": args.r_convergence,
           "maxiter": args.maxiter}
    energies = {}
    for mode in (("one-launch", "sequential") if args.mode == "both" else (args.mode,)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if mode == "one-launch":
            res = solve_in_one_launch(insts, opts)
        else:
            res = [solve_on_device(inst, opts) for inst in insts]
        torch.cuda.synchronize()
        out[f"{mode}_s"] = round(time.perf_counter() - t0, 3)
        out[f"{mode}_converged"] = sum(r["converged"] for r in res)
        out[f"{mode}_outer_iterations_max"] = max(int(r["oiter"]) for r in res)
        energies[mode] = np.array([r["energy"] for r in res])
    if len(energies) == 2:
        out["max_abs_dE"] = float(np.max(np.abs(energies["one-launch"] - energies["sequential"])))
    print(json.dumps(out))


if __name__ == "__main__":
    main()

"""Benchmark: time to 1e-6 boundary-point SDP convergence of a v2RDM problem on B200.

Workloads (plain v2RDM, POSITIVITY DQG, fixed orbitals, FP64, C1, converged to
primal and dual error < 1e-6 and |E_p - E_d| < 1e-6 from the reference's
random guess (srand(0)), MU_UPDATE_FREQUENCY 500, CG_CONVERGENCE 1e-9):

  df20 (default)  the (20e, 20o) active space on synthetic density-fitted
                  integrals: naux = 400, B^Q_pq ~ N(0, 0.05) symmetrised (seed 4),
                  h = diag(linspace(-2, -0.1, 20)) + N(0, 0.02) symmetrised
                  off-diagonal (seed 5), g_pqrs = sum_Q B^Q_pq B^Q_rs through
                  the external-Hamiltonian path.  PSD blocks 20, 190, 210, 400, 800.
  hubbard8        the 1D periodic Hubbard ring with 8 sites, 8 electrons,
                  t = 1, U = 4 (hilbert's own Hubbard path).

Data are synthetic by construction (no molecular integrals exist offline).

One step = one full solve to convergence.  ``value`` is the device solve
time with b, c, x already in HBM (CUDA events on the library's stream);
``e2e`` is the same solve through the public API with host arrays (pinned
H2D of x0, b, c and D2H of x inside the timed region).  L2 is flushed between
steps (a 256 MiB write).

Multi-GPU: replicas only.  Each rank solves its own copy of the workload;
the reported time is the max over ranks; nothing crosses NVLink in the data
path.

``roofline`` is the CG kernel's: algorithmic bytes 8 (2 n_p + 7 n_d) per CG
iteration over its CUDA-event launch time, against the measured HBM copy
bandwidth; ``traffic`` is the kernel's DRAM bytes per iteration from one ncu
capture on the same problem (CG_DRAM_BYTES_PER_ITERATION) times the launch's
iterations.

``--impl reference`` times the reference's own CPU implementation of the path
(hilbert's compiled constraint maps from oracle/_ref, else the C restatement,
driven by the numpy boundary-point restatement), each step a bounded sample
of CG iterations and outer-iteration bodies extrapolated to the workload's
iteration counts.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "df20": dict(nmo=20, nalpha=10, nbeta=10, positivity="DQG", hamiltonian="df",
                 df=dict(n=20, naux=400, seed_b=4, seed_h=5), hubbard_multiplicity=False,
                 r_conv=1e-6, e_conv=1e-6, cg_conv=1e-9, muf=500, maxiter=400000),
    "hubbard8": dict(nmo=8, nalpha=4, nbeta=4, positivity="DQG", hamiltonian="hubbard",
                     hubbard=(1.0, 4.0), hubbard_multiplicity=True,
                     r_conv=1e-6, e_conv=1e-6, cg_conv=1e-9, muf=500, maxiter=400000),
    # config 5: the 4 x 4 periodic Hubbard lattice, 16 electrons, U/t = 8, DQG+T2
    # (80.4 M primal variables, T2 blocks of 1,920 and 6,016 rows)
    "hubbard4x4": dict(nmo=16, nalpha=8, nbeta=8, positivity="DQGT2", hamiltonian="hubbard2d",
                       hubbard2d=dict(lx=4, ly=4, t=1.0, U=8.0), hubbard_multiplicity=False,
                       r_conv=1e-6, e_conv=1e-6, cg_conv=1e-9, muf=500, maxiter=400000),
    # config 3: 64 independent DQG rings (L 6..14, N in {L-2, L, L+2}, U/t ~ U[1, 8], seed 3)
    "batch64": dict(kind="batch", count=64, seed=3, positivity="DQG", r_conv=1e-6, e_conv=1e-6,
                    cg_conv=1e-9, muf=500, maxiter=400000, concurrency=16),
}
# FP64 reference of each workload: the CPU oracle's converged solve, hilbert's
# compiled maps (oracle/_ref) driven by the numpy boundary-point restatement
# (oracle/bpsdp.py), generated by tests/golden/make_fp64_energies.py into
# tests/golden/fp64_<workload>.json.  Its outer / CG iteration counts scale
# the reference arm's per-iteration sample; its energy is what |dE| is taken
# against.
GOLDEN = os.path.join(ROOT, "tests", "golden")


def fp64_reference(workload):
    """{"energy", "outer_iterations", "cg_iterations", "wall_s", ...} of the
    CPU oracle's FP64 solve, or None when its fixture is absent."""
    path = os.path.join(GOLDEN, f"fp64_{workload}.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


# Outer and CG iteration counts of the device's own FP64 solve of each
# workload to convergence (default path, B200): what the CPU arm's sampled
# per-iteration costs are scaled by when the CPU oracle's full solve is not
# available as a fixture.
DEVICE_COUNTS = {"df20": {"outer_iterations": 4101, "cg_iterations": 127159}}
# DRAM bytes the CG kernel moves per CG iteration (dram__bytes_read.sum +
# dram__bytes_write.sum from one ncu capture of a whole launch: 9.56 + 4.70 GB
# over 142 iterations and the initial residual, on the same df20 problem;
# `python -m hilbert_b200.synthetic --n 20 --naux 400 --max-outer 1`).  The
# bench's launches run the same passes over the same vectors, so their traffic
# is this figure times their iterations.
CG_DRAM_BYTES_PER_ITERATION = {"df20": 14.26e9 / 143}


def iteration_counts(workload):
    """(counts, source): the CPU oracle's FP64 solve when its fixture exists,
    else the device solve's counts, else (None, None)."""
    ref = fp64_reference(workload)
    if ref is not None:
        return ref, "the CPU oracle's FP64 solve to convergence"
    if workload in DEVICE_COUNTS:
        return dict(DEVICE_COUNTS[workload]), "the device's FP64 solve to convergence (B200, default path)"
    return None, None


def hamiltonian(w):
    """('hubbard', (t, U)) or ('external', (h, g)) for a workload"""
    if w["hamiltonian"] == "hubbard":
        return "hubbard", w["hubbard"]
    if w["hamiltonian"] == "hubbard2d":
        from hilbert_b200.synthetic import hubbard_2d
        return "external", hubbard_2d(**w["hubbard2d"])
    from hilbert_b200.synthetic import df_hamiltonian
    return "external", df_hamiltonian(**w["df"])


METRIC = "time to 1e-6 SDP convergence, mixed/batched vs plain FP64 on B200; |dE| vs FP64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="df20", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-sample-seconds", type=float, default=60.0,
                    help="seconds of CPU work sampled for the CPU baseline (the reference arm "
                         "divides a few minutes among its steps)")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the solve on the plain FP64 path (selective Jacobi on every block "
                         "every iteration) that a 1-GPU run times for comparison")
    ap.add_argument("--max-outer", type=int, default=0,
                    help="cap the outer iterations of each solve (profiling runs; the line then "
                         "reports a capped, not a converged, solve)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region.

    One ``nvidia-smi -lms 200`` process runs for the whole sampling window and
    writes to a temporary file: the benchmark process forks once, before the
    work it measures (a fork per sample from a process holding a CUDA context
    stalls that context for tens of milliseconds each time)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self._proc = None
        self._file = None

    def start(self):
        import tempfile
        self._file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self._file, stderr=subprocess.DEVNULL)
        except OSError:
            self._proc = None
        return self

    def stop(self):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=10)
            except subprocess.TimeoutExpired:
                self._proc.kill()
                self._proc.wait()
        if self._file is not None:
            self._file.flush()
            self._file.seek(0)
            for line in self._file.read().splitlines():
                if line.strip():
                    self.rows.append([v.strip() for v in line.split(",")])
            self._file.close()
            os.unlink(self._file.name)
            self._file = None

    def __enter__(self):
        return self.start()

    def __exit__(self, *a):
        self.stop()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 1 and r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(self.rows)}


def dist_setup():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_threads():
    """(OpenMP threads of the compiled maps, BLAS threads of numpy's LAPACK)"""
    omp = int(os.environ.get("OMP_NUM_THREADS", "0") or 0) or (os.cpu_count() or 1)
    blas = 1
    try:
        import numpy  # noqa: F401  (loads the BLAS the query below looks for)
        from threadpoolctl import threadpool_info
        n = [i.get("num_threads", 1) for i in threadpool_info() if i.get("user_api") == "blas"]
        blas = max(n) if n else 1
    except Exception:
        pass
    return omp, blas


_CPU_PROBLEMS = {}


def cpu_sample(w, seconds):
    """Time the CPU path on a bounded sample.

    The boundary-point iteration's cost is (cost of one CG iteration: A^T.p,
    A.t, two dots, three axpys) x CG iterations + (fixed cost of one outer
    iteration: A.x, A.(c-z), A^T.y, the block eigendecompositions, norms) x
    outer iterations.  Both unit costs are timed here on the host, each for
    about seconds/2, from the reference's random guess.
    Returns (seconds per CG iteration, seconds per outer iteration, kind, repeats).
    """
    import numpy as np
    from oracle import maps
    from oracle.bpsdp import project_blocks
    kind = "reference" if maps.ref_available() else "port"
    key = (id(w), kind)
    if key not in _CPU_PROBLEMS:   # built once per workload: the steps time the iteration only
        P = maps.RefProblem if kind == "reference" else maps.OracleProblem
        kind_h, ham = hamiltonian(w)
        kw = dict(hubbard=ham) if kind_h == "hubbard" else dict(h=ham[0], g=ham[1])
        prob = P(w["nmo"], w["nalpha"], w["nbeta"], w["positivity"], True, True, **kw)
        o = maps.OracleProblem(w["nmo"], w["nalpha"], w["nbeta"], w["positivity"], True, True, **kw)
        _CPU_PROBLEMS[key] = (prob, o.guess("random"))
    prob, x = _CPU_PROBLEMS[key]
    x = x.copy()
    z = np.zeros(prob.n_primal)
    y = np.random.default_rng(0).standard_normal(prob.n_dual)
    r = y.copy()
    pv = y.copy()
    mu = 0.1
    reps = [0, 0]
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds / 2 or reps[0] < 3:
        q = prob.Au(prob.ATu(pv))
        a = float(r @ r) / float(pv @ q)
        y += a * pv
        r -= a * q
        pv = r + 0.5 * pv
        reps[0] += 1
    t_cg = (time.perf_counter() - t0) / reps[0]
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds / 2 or reps[1] < 3:
        ax = prob.Au(x)
        acz = prob.Au(prob.c - z)
        rhs = acz + mu * (prob.b - ax)
        aty = prob.ATu(y)
        U = mu * x + aty - prob.c
        xn, z = project_blocks(U, prob.dims, mu)
        ep = np.linalg.norm(prob.Au(xn) - prob.b)
        ed = np.linalg.norm(aty + z - prob.c)
        _ = float(prob.c @ xn) + float(prob.b @ y) + ep + ed + float(rhs[0])
        reps[1] += 1
    t_outer = (time.perf_counter() - t0) / reps[1]
    return t_cg, t_outer, kind, reps


def config_of(args, w):
    """The workload description both arms print (the same keys and values)."""
    kind_h = "hubbard" if w["hamiltonian"] == "hubbard" else "external"
    return {"workload": args.workload, "nmo": w["nmo"], "nalpha": w["nalpha"], "nbeta": w["nbeta"],
            "positivity": w["positivity"],
            "hamiltonian": ({"hubbard_t_U": list(w["hubbard"])} if kind_h == "hubbard"
                            else {"hubbard_2d": w["hubbard2d"]} if "hubbard2d" in w
                            else {"synthetic_df": w["df"]}),
            "r_convergence": w["r_conv"], "e_convergence": w["e_conv"], "cg_convergence": w["cg_conv"],
            "mu_update_frequency": w["muf"], "tpdm_guess": "RANDOM",
            "parallelism": "replicas" if args.gpus > 1 else "single",
            "l2": "flushed between steps (256 MiB write)"}


def cpu_baseline(w, ref, seconds, steps=1, source="the CPU oracle's FP64 solve to convergence"):
    """The CPU path timed on a bounded sample, scaled to the iteration counts
    of an FP64 solve to convergence (ref; source says whose)."""
    omp, blas = cpu_threads()
    vals = []
    for _ in range(steps):
        t_cg, t_out, kind, reps = cpu_sample(w, seconds)
        vals.append(t_cg * ref["cg_iterations"] + t_out * ref["outer_iterations"])
    return {"value": statistics.mean(vals), "unit": "s", "cores": omp, "kind": kind,
            "openmp_threads_maps": omp, "blas_threads": blas,
            "sample": f"{reps[0]} CG iterations ({t_cg * 1e3:.2f} ms each) and {reps[1]} outer-iteration "
                      f"bodies ({t_out * 1e3:.2f} ms each) timed on the host per step, scaled to the "
                      f"{ref['cg_iterations']} CG + {ref['outer_iterations']} outer iterations of {source}",
            "measured_full_solve": {"wall_s": ref.get("wall_s"), "omp_threads": ref.get("omp_threads"),
                                    "where": "the build container's host cores (generator run)"}}


def run_reference(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    ref, source = iteration_counts(args.workload)
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": f"no converged FP64 solve of {args.workload} "
                                                             "to scale the CPU sample by"}))
        return
    # each step a bounded sample; the whole run stays within a few minutes
    per_step = max(2.0, min(args.cpu_sample_seconds, 180.0 / max(1, args.warmup + args.steps)))
    vals = []
    cb = None
    for k in range(args.warmup + args.steps):
        b = cpu_baseline(w, ref, per_step, source=source)
        if k >= args.warmup:
            vals.append(b["value"])
            cb = b
    total = max(vals)
    cb["value"] = total
    line = {"impl": "reference", "metric": METRIC, "value": total, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(args, w),
            "cpu_baseline": cb,
            "e2e": {"value": total, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cusolver_projection_ms(p, dev, reps=5):
    """Reference point for the plain FP64 path: one projection of the
    problem's blocks by cuSOLVER's syevd (torch.linalg.eigh, the blocks of
    each size batched) and U+ = V max(L, 0) V^T, ms per call."""
    import torch
    dims = [int(d) for d in p.dims]
    by = {}
    for d in dims:
        by[d] = by.get(d, 0) + 1
    mats = {d: torch.randn(k, d, d, dtype=torch.float64, device=dev) for d, k in by.items()}
    mats = {d: 0.5 * (m + m.transpose(1, 2)) for d, m in mats.items()}

    def once():
        for m in mats.values():
            lam, V = torch.linalg.eigh(m)
            _ = (V * lam.clamp(min=0.0).unsqueeze(1)) @ V.transpose(1, 2)

    once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        once()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_b200(args, w):
    import numpy as np
    import torch

    import hilbert_b200 as hb
    world, rank, local = dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    opts = hb.Options({"R_CONVERGENCE": w["r_conv"], "E_CONVERGENCE": w["e_conv"],
                       "CG_CONVERGENCE": w["cg_conv"],
                       "MAXITER": args.max_outer if args.max_outer else w["maxiter"],
                       "MU_UPDATE_FREQUENCY": w["muf"]})
    p = hb.V2RDMProblem(w["nmo"], w["nalpha"], w["nbeta"], w["positivity"], True, True,
                        hubbard_multiplicity=w["hubbard_multiplicity"])
    b = p.b()
    kind_h, ham = hamiltonian(w)
    c = p.c_hubbard(*ham) if kind_h == "hubbard" else p.c_external(*ham)
    x0 = p.guess("RANDOM")
    db = torch.from_numpy(b).to(dev)
    dc = torch.from_numpy(c).to(dev)
    dx0 = torch.from_numpy(x0).to(dev)
    dx = torch.empty_like(dx0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ref = fp64_reference(args.workload)

    def one():
        dx.copy_(dx0)
        flush.fill_(1.0)
        torch.cuda.synchronize()
        barrier(world)
        return p.solve_device(dx, db, dc, opts)

    clk = ClockSampler(local).start()   # started before the warm-up: no fork in the timed region
    for _ in range(args.warmup):
        one()
    times, stats = [], None
    launches0 = p.kernel_launches()
    # kernel-class CUDA events only (level 1) in the timed steps: they give
    # the CG kernel's launch time for the roofline at negligible cost
    p.set_profiling(1)
    with clk:
        for _ in range(args.steps):
            dx.copy_(dx0)
            flush.fill_(1.0)
            torch.cuda.synchronize()
            barrier(world)
            s = torch.cuda.Stream(device=dev)
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(s)
            stats = p.solve_device(dx, db, dc, opts)
            ev1.record(s)
            torch.cuda.synchronize()
            times.append(ev0.elapsed_time(ev1) / 1e3)
    prof = p.profile()
    split_choice = p.gemm_split_choice()
    launches = p.kernel_launches() - launches0
    p.set_profiling(0)
    t = max_over_ranks(max(times), world)
    energy = float(c @ dx.cpu().numpy())

    # end to end through the public API (host arrays in and out)
    e2e_times = []
    for _ in range(max(1, args.steps // 2)):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        xh, st2 = p.solve(x0, b, c, opts)
        e2e_times.append(time.perf_counter() - t0)
    te2e = max_over_ranks(max(e2e_times), world)

    # one more solve with the phase timers on (level 2), outside the timed steps
    phases = None
    if world == 1:
        p.set_profiling(2)
        one()
        phases = {"cg_kernel": {k: round(v, 1) for k, v in p.cg_profile().items()},
                  "projection": {k: [round(v[0], 1), v[1]] for k, v in p.projection_profile().items()},
                  "kernel_classes_ms": {k: round(v[0], 1) for k, v in p.profile().items()}}
        p.set_profiling(0)

    # the plain FP64 path on the same problem (1 GPU only): every block fully
    # diagonalised by selective Jacobi every iteration, as libsdp does with LAPACK
    plain = None
    if world == 1 and not args.no_plain:
        p.set_projection_mode("jacobi")
        p.set_profiling(1)
        dx.copy_(dx0)
        flush.fill_(1.0)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        st_plain = p.solve_device(dx, db, dc, opts)
        ev1.record()
        torch.cuda.synchronize()
        pprof = p.profile()
        p.set_profiling(0)
        e_plain = float(c @ dx.cpu().numpy())
        p.set_projection_mode("refine")
        sec = ev0.elapsed_time(ev1) / 1e3
        cus = cusolver_projection_ms(p, dev)
        proj_ms, proj_n = pprof["projection"]
        plain = {"seconds": sec, "energy": e_plain,
                 "outer_iterations": st_plain["oiter"], "cg_iterations": st_plain["iiter"],
                 "converged": st_plain["converged"],
                 "projection_ms_per_call": proj_ms / max(proj_n, 1),
                 "cusolver_syevd_projection_ms_per_call": cus,
                 "seconds_with_cusolver_projection_estimate":
                     sec - proj_ms / 1e3 + st_plain["oiter"] * cus / 1e3}

    # the mixed-precision arm (1 GPU only): FP32 eigensolves of the large
    # blocks where the warm refinement would take block-Jacobi sweeps, each
    # followed by an FP64 Rayleigh-Ritz step and FP64 Newton passes
    mixed = None
    if world == 1 and not args.no_plain:
        p.set_projection_mode("mixed")
        dx.copy_(dx0)
        flush.fill_(1.0)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        c0 = p.refine_counts()
        ev0.record()
        st_mx = p.solve_device(dx, db, dc, opts)
        ev1.record()
        torch.cuda.synchronize()
        c1 = p.refine_counts()
        e_mx = float(c @ dx.cpu().numpy())
        p.set_projection_mode("refine")
        mixed = {"seconds": ev0.elapsed_time(ev1) / 1e3, "energy": e_mx,
                 "outer_iterations": st_mx["oiter"], "cg_iterations": st_mx["iiter"],
                 "converged": st_mx["converged"],
                 "fp32_eigensolves": c1["fp32_eigensolves"] - c0["fp32_eigensolves"],
                 "block_jacobi_sweeps": c1["block_jacobi_sweeps"] - c0["block_jacobi_sweeps"],
                 "abs_dE_vs_fp64": abs(e_mx - ref["energy"]) if ref else None,
                 "speedup_vs_plain_fp64": (plain["seconds"] / (ev0.elapsed_time(ev1) / 1e3)) if plain else None}

    # roofline: cg_kernel, the largest single kernel (the projection is a
    # sequence of GEMM-tile, test and Jacobi kernels; its FLOP rate is reported
    # beside it).  Its launch time comes from the timed steps' CUDA events.
    oiter, iiter = stats["oiter"], stats["iiter"]
    npr, ndu = p.n_primal, p.n_dual
    nnz_a, nnz_t = p.operator_nnz()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    ms_cg, n_cg = prof["cg_kernel"]
    m = iiter / max(oiter, 1)   # CG iterations per launch (one launch per outer iteration)
    # algorithmic bytes: vectors only (index tables excluded), per CG iteration
    # one A and one A^T (read / write x and y once each) and ~5 CG vector streams
    per_iter = 8.0 * (2 * npr + 7 * ndu)
    bytes_launch = (m + 1) * per_iter   # + the initial residual's A^T and A pass
    ach = bytes_launch / (ms_cg / n_cg / 1e3) / 1e9
    roof = {"kernel": "cg_kernel", "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
            "frac": ach / hbm,
            "traffic": (CG_DRAM_BYTES_PER_ITERATION[args.workload] * (m + 1)
                        if args.workload in CG_DRAM_BYTES_PER_ITERATION else None),
            "traffic_source": ("ncu DRAM bytes per CG iteration of one captured launch on the same "
                               "problem, times (m + 1)" if args.workload in CG_DRAM_BYTES_PER_ITERATION
                               else None),
            "algorithmic_bytes": "per CG iteration 8 (2 n_p + 7 n_d) vector bytes (index tables "
                                 f"excluded); (m + 1) iterations per launch, m = {m:.1f}",
            "peak_source": ("MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks
                            else "fallback 6650 GB/s (of fallback)"),
            "launch_ms": ms_cg / max(n_cg, 1)}
    ms_pj, n_pj = prof["projection"]
    flops = sum((16.0 / 3.0) * float(d) ** 3 for d in p.dims)
    roof["projection"] = {"ms_per_call": ms_pj / max(n_pj, 1),
                          "fp64_tflops": flops / (ms_pj / max(n_pj, 1) / 1e3) / 1e12,
                          "flops_per_call": flops,
                          "note": "sum (16/3) n_b^3 per call (eigendecomposition + back-transform "
                                  "counted as for LAPACK), FP64; no FP64 peak is measured"}
    tot = sum(x[0] for x in prof.values())
    roof["kernel_ms_share"] = {k: round(v[0] / tot, 4) for k, v in prof.items()}
    roof["phases_ms"] = phases

    cpu = None
    counts, source = iteration_counts(args.workload)
    if counts is None and stats is not None and stats["converged"]:
        counts = {"outer_iterations": int(stats["oiter"]), "cg_iterations": int(stats["iiter"])}
        source = "this run's device solve to convergence"
    if rank == 0 and world == 1 and args.cpu_sample_seconds > 0 and counts is not None:
        cpu = cpu_baseline(w, counts, args.cpu_sample_seconds, source=source)
    clocks = clk.summary()
    if rank == 0:
        cfg = config_of(args, w)
        fp64_e = ref["energy"] if ref else None
        cfg.update({"n_primal": npr, "n_dual": ndu, "block_dims": sorted(set(int(d) for d in p.dims)),
                    "outer_iterations": oiter, "cg_iterations": iiter,
                    "energy": energy, "converged": stats["converged"],
                    "fp64_energy": fp64_e,
                    "fp64_energy_source": ("CPU oracle FP64 solve (hilbert's compiled maps + numpy "
                                           "boundary-point restatement), tests/golden/fp64_"
                                           f"{args.workload}.json") if ref else None,
                    "fp64_outer_iterations": ref["outer_iterations"] if ref else None,
                    "abs_dE_vs_fp64": abs(energy - fp64_e) if ref else None,
                    "plain_fp64_path": plain,
                    "mixed_precision_path": mixed,
                    "speedup_vs_plain_fp64": (plain["seconds"] / t) if plain else None,
                    "abs_dE_vs_plain_fp64": abs(energy - plain["energy"]) if plain else None,
                    "projection_refine_counts": p.refine_counts(),
                    "gemm_split_autotuned": {"full_list": split_choice[0], "upper_list": split_choice[1]},
                    "max_outer_cap": args.max_outer or None})
        line = {"metric": METRIC, "value": t, "unit": "s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": cfg,
                "e2e": {"value": te2e, "unit": "s", "h2d_bytes_per_step": 8 * (2 * npr + ndu),
                        "d2h_bytes_per_step": 8 * npr},
                "gpu_launches": int(launches),
                "roofline": roof, "cpu_baseline": cpu, "clocks": clocks}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_batch(args, w):
    """Config 3: the 64-ring batch on one GPU.  Every instance keeps its own
    problem, stream, penalty and convergence test (its result is the one it
    gets alone); `concurrency` host threads drive the instances at once, so
    the GPU runs many small solves side by side.  ``value``: inputs already
    in device memory; ``e2e``: host arrays through the public solve().  Both
    are device-synchronised wall clocks around the whole batch (the work
    spans many streams).  The four smallest instances are also timed one at a
    time and four at once, beside it."""
    import numpy as np
    import torch
    from concurrent.futures import ThreadPoolExecutor

    import hilbert_b200 as hb
    from hilbert_b200.batch import hubbard_batch
    world, rank, local = dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    opts = hb.Options({"R_CONVERGENCE": w["r_conv"], "E_CONVERGENCE": w["e_conv"],
                       "CG_CONVERGENCE": w["cg_conv"], "MAXITER": args.max_outer or w["maxiter"],
                       "MU_UPDATE_FREQUENCY": w["muf"]})
    insts = hubbard_batch(count=w["count"], seed=w["seed"], positivity=w["positivity"])
    built = [i.problem() for i in insts]
    x0 = [p.guess("RANDOM") for p, _, _ in built]
    dev_in = [(torch.from_numpy(b).to(dev), torch.from_numpy(c).to(dev)) for _, b, c in built]

    def init():
        torch.cuda.set_device(dev)

    def device_one(k):
        p = built[k][0]
        x = torch.from_numpy(x0[k]).to(dev)
        st = p.solve_device(x, dev_in[k][0], dev_in[k][1], opts)
        return float(built[k][2] @ x.cpu().numpy()), st

    def host_one(k):
        p, b, c = built[k]
        xh, st = p.solve(x0[k], b, c, opts)
        return float(c @ xh), st

    def timed(fn, idx, workers):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=workers, initializer=init) as pool:
            out = list(pool.map(fn, idx))
        torch.cuda.synchronize()
        return time.perf_counter() - t0, out

    order = sorted(range(len(insts)), key=lambda k: -insts[k].cost())   # longest first
    k_conc = int(w["concurrency"])
    small = order[-4:]
    for _ in range(args.warmup):   # warm-up: the four smallest instances at once
        timed(device_one, small, 4)
    launches0 = sum(p.kernel_launches() for p, _, _ in built)
    times, res = [], None
    for _ in range(args.steps):
        t, res = timed(device_one, order, k_conc)
        times.append(t)
    launches = sum(p.kernel_launches() for p, _, _ in built) - launches0
    t = max(times)
    te2e, res_h = timed(host_one, order, k_conc)
    # the same four instances one at a time and at once (the smallest four,
    # to keep the sequential leg short)
    t_seq4, _ = timed(device_one, small, 1)
    t_conc4, _ = timed(device_one, small, 4)
    energies = {k: e for k, (e, _) in zip(order, res)}
    energies_h = {k: e for k, (e, _) in zip(order, res_h)}
    conv = sum(bool(st["converged"]) for _, st in res)
    if rank == 0:
        cfg = {"workload": args.workload, "instances": len(insts), "seed": w["seed"],
               "positivity": w["positivity"], "sites": [i.sites for i in insts],
               "electrons": [i.electrons for i in insts], "U_over_t": [round(i.U, 4) for i in insts],
               "r_convergence": w["r_conv"], "e_convergence": w["e_conv"], "cg_convergence": w["cg_conv"],
               "mu_update_frequency": w["muf"], "concurrency": k_conc, "converged": conv,
               "outer_iterations_max": max(int(st["oiter"]) for _, st in res),
               "max_abs_dE_device_vs_host_arrays": max(abs(energies[k] - energies_h[k]) for k in energies),
               "smallest4_sequential_s": t_seq4, "smallest4_concurrent_s": t_conc4,
               "smallest4_speedup": t_seq4 / t_conc4,
               "parallelism": "single", "timing": "device-synchronised wall clock (many streams)"}
        line = {"metric": METRIC, "value": t, "unit": "s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": cfg,
                "e2e": {"value": te2e, "unit": "s",
                        "h2d_bytes_per_step": int(sum(8 * (2 * p.n_primal + p.n_dual) for p, _, _ in built)),
                        "d2h_bytes_per_step": int(sum(8 * p.n_primal for p, _, _ in built))},
                "gpu_launches": int(launches), "roofline": None, "cpu_baseline": None}
        print(json.dumps(line), flush=True)
    for p, _, _ in built:
        p.close()


def main():
    args = parse()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        if w.get("kind") == "batch":
            print(json.dumps({"impl": "reference", "unavailable": "the batch workload has no CPU arm; "
                                                                 "time its instances as hubbard rings"}))
            return
        run_reference(args, w)
    elif w.get("kind") == "batch":
        run_batch(args, w)
    else:
        run_b200(args, w)


if __name__ == "__main__":
    main()

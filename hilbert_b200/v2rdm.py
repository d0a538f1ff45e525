"""Host-side mirror of hilbert's v2RDM-CASSCF interface for the B200 path.

* ``Options``        -- the HILBERT option names and defaults that the v2RDM
                         path reads (src/plugin.cc:80-463).
* ``v2RDMHelper``    -- the pybind class of src/python_api/python_helpers.cc:104-113
                         (external-Hamiltonian constructor and the Hubbard path).
* ``V2RDMProblem``   -- the device-map problem: A.x, A^T.y, projection and the
                         full solve on CUDA tensors through the C ABI.
* ``BPSDPSolver``    -- libsdp::BPSDPSolver-shaped solver with host callbacks
                         (src/v2rdm_casscf/v2rdm_solver.cc:424-447, 1340).
"""
import ctypes

import numpy as np

from . import _capi
from ._capi import SDP_CALLBACK, SDP_MONITOR, SDPOptions, check

# option name -> default (src/plugin.cc line of the add_* call in comments)
DEFAULTS = {
    "E_CONVERGENCE": 1e-6,          # :94
    "R_CONVERGENCE": 1e-5,          # :97
    "MAXITER": 50,                  # :100
    "CG_CONVERGENCE": 1e-9,         # :238
    "CG_MAXITER": 10000,            # :241
    "MU_UPDATE_FREQUENCY": 1000,    # :217
    "POSITIVITY": "DQG",            # :220
    "CONSTRAIN_SPIN": True,         # :306
    "CONSTRAIN_SZ": True,           # :309
    "CONSTRAIN_D3": False,          # :226
    "CONSTRAIN_Q3": False,          # :235
    "CONSTRAIN_E3": False,          # :229
    "CONSTRAIN_F3": False,          # :232
    "CONSTRAIN_D4": False,          # :303
    "TPDM_GUESS": "RANDOM",         # :205
    "SDP_SOLVER": "BPSDP",          # :246
    "HUBBARD_HAMILTONIAN": False,   # :249
    "HUBBARD_T": 1.0,               # :252
    "HUBBARD_U": 1.0,               # :255
    "N_HUBBARD_SITES": 4,           # :258
    "N_HUBBARD_SPINS": 4,           # :261
    "OPTIMIZE_ORBITALS": True,      # :138
    "ORBOPT_FREQUENCY": 500,        # :150
    "ORBOPT_MAXITER": 10,           # :168
    "ORBOPT_GRADIENT_CONVERGENCE": 1e-4,   # :153
    "ORBOPT_ENERGY_CONVERGENCE": 1e-8,     # :156
    "TPDM_WRITE_FULL": False,       # :103
    "WRITE_CHECKPOINT_FILE": False,  # :208
    "OPDM_WRITE_FULL": False,       # :286
    "TPDM_WRITE_SPIN_FREE": False,  # :289
    "TPDM_WRITE": False,            # :292
    "3PDM_WRITE": False,            # :295
    "RESTART_FROM_CHECKPOINT_FILE": "",   # :185
    "GPC_CONSTRAINTS": "NONE",      # :223
    "DERTYPE": "NONE",              # Psi4's global derivative option
}


class Options:
    """Case-insensitive option store with Psi4-style accessors."""

    def __init__(self, values=None, **kw):
        self._v = dict(DEFAULTS)
        for src in (values or {}), kw:
            for k, v in src.items():
                self.set(k, v)

    def set(self, key, value):
        key = key.upper()
        if isinstance(value, str):
            value = value.upper()
        self._v[key] = value

    def get(self, key):
        return self._v[key.upper()]

    get_str = get_double = get_int = get_bool = get

    def __getitem__(self, key):
        return self.get(key)

    def sdp_options(self):
        return SDPOptions(float(self.get("E_CONVERGENCE")), float(self.get("R_CONVERGENCE")),
                          float(self.get("CG_CONVERGENCE")), int(self.get("CG_MAXITER")),
                          int(self.get("MAXITER")))


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _tptr(t):
    return ctypes.c_void_p(t.data_ptr())


class V2RDMProblem:
    """One C1 v2RDM problem whose constraint maps live on the GPU."""

    def __init__(self, nmo, nalpha, nbeta, positivity="DQG", constrain_spin=True,
                 constrain_sz=True, hubbard_multiplicity=False):
        lib = _capi.load()
        self._lib = lib
        h = ctypes.c_void_p()
        pos, *extras = positivity.upper().split("+")
        if pos not in _capi.POSITIVITY or not set(extras) <= {"D3", "Q3", "E3", "F3", "D4"}:
            raise ValueError(f"POSITIVITY {positivity} is not on the device path "
                             f"(supported: {sorted(_capi.POSITIVITY)}, each optionally "
                             f"+D3 / +Q3 / +E3 / +F3 / +D4)")
        code = (_capi.POSITIVITY[pos] | (_capi.V2B_CONSTRAIN_D3 if "D3" in extras else 0)
                | (_capi.V2B_CONSTRAIN_Q3 if "Q3" in extras else 0)
                | (_capi.V2B_CONSTRAIN_E3 if "E3" in extras else 0)
                | (_capi.V2B_CONSTRAIN_F3 if "F3" in extras else 0)
                | (_capi.V2B_CONSTRAIN_D4 if "D4" in extras else 0))
        check(lib.v2b_problem_create(int(nmo), int(nalpha), int(nbeta), code,
                                     int(bool(constrain_spin)), int(bool(constrain_sz)),
                                     int(bool(hubbard_multiplicity)), ctypes.byref(h)))
        self._sizes(h, nmo, nalpha, nbeta)

    def _sizes(self, h, nmo, nalpha, nbeta):
        lib = self._lib
        self._h = h
        self.nmo, self.nalpha, self.nbeta = nmo, nalpha, nbeta
        self.n_primal = lib.v2b_problem_n_primal(h)
        self.n_dual = lib.v2b_problem_n_dual(h)
        nb = lib.v2b_problem_n_blocks(h)
        dims = (ctypes.c_int * nb)()
        check(lib.v2b_problem_block_dims(h, dims))
        self.dims = np.array(dims[:], dtype=np.int32)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.v2b_problem_destroy(self._h)
            self._h = None

    def palette(self, transposed=False):
        """The distinct coefficients of A (or A^T), as bit patterns: parts
        whose palettes together hold at most 16 can share one BatchProblem."""
        count = ctypes.c_int()
        check(self._lib.v2b_problem_palette(self._h, int(transposed), None, ctypes.byref(count)))
        out = np.zeros(count.value)
        check(self._lib.v2b_problem_palette(self._h, int(transposed), out.ctypes.data, ctypes.byref(count)))
        return set(out.view(np.uint64).tolist())

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # host-side problem data
    def b(self):
        out = np.zeros(self.n_dual)
        check(self._lib.v2b_problem_build_b(self._h, _dptr(out)))
        return out

    def c_hubbard(self, t, U):
        out = np.zeros(self.n_primal)
        check(self._lib.v2b_problem_build_c_hubbard(self._h, float(t), float(U), _dptr(out)))
        return out

    def c_external(self, h, g):
        h = np.ascontiguousarray(h, dtype=np.float64).ravel()
        g = np.ascontiguousarray(g, dtype=np.float64).ravel()
        if h.size != self.nmo ** 2 or g.size != self.nmo ** 4:
            raise ValueError("h must hold nmo^2 and g nmo^4 elements")
        out = np.zeros(self.n_primal)
        check(self._lib.v2b_problem_build_c_external(self._h, _dptr(h), _dptr(g), _dptr(out)))
        return out

    def guess(self, kind="RANDOM"):
        out = np.zeros(self.n_primal)
        check(self._lib.v2b_problem_guess(self._h, int(kind.upper() == "HF"), _dptr(out)))
        return out

    # device maps on torch CUDA tensors (float64, contiguous)
    def _stream(self):
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _check_tensor(t, n):
        if not (t.is_cuda and t.dtype.__repr__() == "torch.float64" and t.is_contiguous()
                and t.numel() == n):
            raise ValueError(f"expected a contiguous float64 CUDA tensor of {n} elements")

    def Au(self, x, out=None):
        import torch
        self._check_tensor(x, self.n_primal)
        out = torch.empty(self.n_dual, dtype=torch.float64, device=x.device) if out is None else out
        self._check_tensor(out, self.n_dual)
        check(self._lib.v2b_problem_Au(self._h, _tptr(x), _tptr(out), self._stream()))
        return out

    def ATu(self, y, out=None):
        import torch
        self._check_tensor(y, self.n_dual)
        out = torch.empty(self.n_primal, dtype=torch.float64, device=y.device) if out is None else out
        self._check_tensor(out, self.n_primal)
        check(self._lib.v2b_problem_ATu(self._h, _tptr(y), _tptr(out), self._stream()))
        return out

    def project(self, U, mu, warm=False):
        """x = U+ / mu, z = U+ - sym(U) per PSD block.  warm=True starts each block
        from the eigenvector basis the previous warm projection (or device solve)
        left, as the solver's iterations do; the default solves every block afresh."""
        import torch
        self._check_tensor(U, self.n_primal)
        x = torch.empty_like(U)
        z = torch.empty_like(U)
        fn = self._lib.v2b_problem_project_warm if warm else self._lib.v2b_problem_project
        check(fn(self._h, _tptr(U), float(mu), _tptr(x), _tptr(z), self._stream()))
        return x, z

    def solve(self, x0, b, c, options, monitor=None):
        """Host arrays in, converged x out (hilbert's compute_energy outer loop)."""
        x = np.array(x0, dtype=np.float64, copy=True)
        b = np.ascontiguousarray(b, dtype=np.float64)
        c = np.ascontiguousarray(c, dtype=np.float64)
        o = options.sdp_options() if isinstance(options, Options) else options
        muf = int(options.get("MU_UPDATE_FREQUENCY")) if isinstance(options, Options) else 1000
        cb = SDP_MONITOR(monitor) if monitor is not None else SDP_MONITOR()
        oi, ii, e = ctypes.c_long(), ctypes.c_long(), ctypes.c_double()
        rc = check(self._lib.v2b_problem_solve(self._h, _dptr(x), _dptr(b), _dptr(c), ctypes.byref(o),
                                               muf, cb, 1, None, ctypes.byref(oi), ctypes.byref(ii),
                                               ctypes.byref(e)),
                   allow=(_capi.V2B_OK, _capi.V2B_NOT_CONVERGED))
        return x, {"converged": rc == _capi.V2B_OK, "oiter": oi.value, "iiter": ii.value,
                   "energy": e.value, "mu": self._lib.v2b_problem_get_mu(self._h)}

    def solve_device(self, x, b, c, options, monitor=None):
        """x, b, c are CUDA float64 tensors; x is updated in place."""
        self._check_tensor(x, self.n_primal)
        self._check_tensor(b, self.n_dual)
        self._check_tensor(c, self.n_primal)
        o = options.sdp_options() if isinstance(options, Options) else options
        muf = int(options.get("MU_UPDATE_FREQUENCY")) if isinstance(options, Options) else 1000
        cb = SDP_MONITOR(monitor) if monitor is not None else SDP_MONITOR()
        oi, ii, e = ctypes.c_long(), ctypes.c_long(), ctypes.c_double()
        import torch
        torch.cuda.current_stream().synchronize()
        rc = check(self._lib.v2b_problem_solve_device(self._h, _tptr(x), _tptr(b), _tptr(c),
                                                      ctypes.byref(o), muf, cb, 1, None,
                                                      ctypes.byref(oi), ctypes.byref(ii),
                                                      ctypes.byref(e)),
                   allow=(_capi.V2B_OK, _capi.V2B_NOT_CONVERGED))
        return {"converged": rc == _capi.V2B_OK, "oiter": oi.value, "iiter": ii.value,
                "energy": e.value, "mu": self._lib.v2b_problem_get_mu(self._h)}

    def get_y(self):
        out = np.zeros(self.n_dual)
        check(self._lib.v2b_problem_get_y(self._h, _dptr(out)))
        return out

    def get_mu(self):
        return self._lib.v2b_problem_get_mu(self._h)

    def set_state(self, mu, y, z):
        """The next solve starts from mu, y and z (a restart from a checkpoint)."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        z = np.ascontiguousarray(z, dtype=np.float64)
        if y.shape != (self.n_dual,) or z.shape != (self.n_primal,):
            raise ValueError(f"y must hold {self.n_dual} values and z {self.n_primal}")
        check(self._lib.v2b_problem_set_state(self._h, float(mu), _dptr(y), _dptr(z)))

    def set_wait_limit(self, polls=0):
        """Polls of a CG grid-barrier wait before the solve gives up with
        V2B_DEVICE_TIMEOUT (0: the default, seconds)."""
        check(self._lib.v2b_problem_set_wait_limit(self._h, int(polls)))

    def continue_state(self):
        """The next solve continues from the penalty, dual variables and
        eigenvector bases the last device solve left, as libsdp's solver
        keeps them between solve() calls (v2rdm_solver.cc:1330-1361)."""
        check(self._lib.v2b_problem_continue(self._h))

    def get_z(self):
        out = np.zeros(self.n_primal)
        check(self._lib.v2b_problem_get_z(self._h, _dptr(out)))
        return out

    def kernel_launches(self):
        return self._lib.v2b_problem_kernel_launches(self._h)

    KERNEL_CLASSES = ("cg_kernel", "spmv_AT_U_kernel", "projection", "spmv_A2_kernel",
                      "stats_kernel")

    def set_profiling(self, on=True):
        """on: False/0 off, True/1 CUDA events per kernel class, 2 also the
        CG and projection phases."""
        check(self._lib.v2b_problem_set_profiling(self._h, int(on)))

    def profile(self):
        """{kernel: (total_ms, launches)} from CUDA events on the library's stream"""
        ms = (ctypes.c_double * 5)()
        n = (ctypes.c_long * 5)()
        check(self._lib.v2b_problem_profile(self._h, ms, n))
        return {k: (ms[i], n[i]) for i, k in enumerate(self.KERNEL_CLASSES)}

    PROJECTION_PHASES = ("gemm", "acceptance", "clusters_newton", "block_jacobi", "jacobi")

    def projection_profile(self):
        """{phase: (total_ms, count)} of the projection, with profiling on"""
        k = len(self.PROJECTION_PHASES)
        ms, n = (ctypes.c_double * k)(), (ctypes.c_long * k)()
        check(self._lib.v2b_problem_projection_profile(self._h, ms, n, k))
        return {name: (ms[i], n[i]) for i, name in enumerate(self.PROJECTION_PHASES)}

    # pass 1: t = A^T (r + beta p) and ||t||^2; pass 2: A t with the y, r
    # update and r.r
    CG_PHASES = ("initial_residual", "transpose_gather", "gather_update")

    def cg_profile(self):
        """{phase: total_ms} of the CG kernel, barrier to barrier, with profiling on"""
        k = len(self.CG_PHASES)
        ms = (ctypes.c_double * k)()
        check(self._lib.v2b_problem_cg_profile(self._h, ms, k))
        return {name: ms[i] for i, name in enumerate(self.CG_PHASES)}

    def projection_counts(self):
        """{"calls", "rotations", "sweep_overruns"} of the warm-started projection"""
        w, r, c = ctypes.c_long(), ctypes.c_long(), ctypes.c_long()
        check(self._lib.v2b_problem_projection_counts(self._h, ctypes.byref(w), ctypes.byref(r),
                                                      ctypes.byref(c)))
        return {"calls": w.value, "rotations": r.value, "sweep_overruns": c.value}

    def operator_nnz(self):
        """(nnz(A), nnz(A^T)) of the packed constraint operator"""
        out = []
        for t in (0, 1):
            nr, nnz, npal = ctypes.c_long(), ctypes.c_long(), ctypes.c_int()
            check(self._lib.v2b_problem_operator_size(self._h, t, ctypes.byref(nr), ctypes.byref(nnz),
                                                      ctypes.byref(npal)))
            out.append(nnz.value)
        return tuple(out)

    # the records of hilbert's density-matrix writers (struct tpdm / struct opdm)
    TPDM_RECORD = np.dtype([("i", np.int32), ("j", np.int32), ("k", np.int32), ("l", np.int32),
                            ("value", np.float64)])
    OPDM_RECORD = np.dtype([("i", np.int32), ("j", np.int32), ("value", np.float64)])
    RDM_FILES = ("D2aa", "D2bb", "D2ab", "D2", "D1a", "D1b")

    @staticmethod
    def read_rdm_files(path):
        """{file: {entry: bytes}} from write_rdm_files."""
        out = {}
        with np.load(path) as z:
            for k in z.files:
                name, key = k.split("/", 1)
                out.setdefault(name, {})[key] = z[k].tobytes()
        return out

    def rdm_records(self, x, ncore=0):
        """{file: records} as WriteTPDM, WriteTPDMSpinFree and WriteOPDM emit
        them (write_tpdm.cc:40-519, write_opdm.cc:40-114) for the host or
        device primal vector x: D2aa, D2bb, D2ab, the spin-free D2, D1a, D1b
        (for DOCI, what its WriteTPDM writes: D2aa, D2bb, D2ab).  ncore
        doubly occupied orbitals are numbered first, with their core-core and
        core-active records."""
        xh = np.ascontiguousarray(x.detach().cpu().numpy() if hasattr(x, "detach") else x,
                                  dtype=np.float64)
        if xh.shape != (self.n_primal,):
            raise ValueError(f"x must hold {self.n_primal} values")
        counts = np.zeros(6, np.int64)
        check(self._lib.v2b_problem_rdm_counts(self._h, int(ncore), counts.ctypes.data))
        out = {name: np.zeros(int(cnt), self.TPDM_RECORD if name.startswith("D2") else self.OPDM_RECORD)
               for name, cnt in zip(self.RDM_FILES, counts) if cnt >= 0}   # -1: not written
        check(self._lib.v2b_problem_rdm_records(
            self._h, int(ncore), xh.ctypes.data, *[out[name].ctypes.data if name in out else None
                                       for name in self.RDM_FILES]))
        return out

    def tpdm_iwl_records(self, x, ncore=0):
        """{"D2aa", "D2ab", "D2bb"}: the IWL::write_value calls of WriteTPDM_IWL
        (write_tpdm_iwl.cc:45-205) as records, fields i, j, k, l holding the
        labels (i, k, j, l) of D2(ij, kl); ncore as in rdm_records."""
        xh = np.ascontiguousarray(x.detach().cpu().numpy() if hasattr(x, "detach") else x,
                                  dtype=np.float64)
        if xh.shape != (self.n_primal,):
            raise ValueError(f"x must hold {self.n_primal} values")
        counts = np.zeros(6, np.int64)
        check(self._lib.v2b_problem_rdm_counts(self._h, int(ncore), counts.ctypes.data))
        out = {"D2aa": np.zeros(int(counts[0]), self.TPDM_RECORD),
               "D2ab": np.zeros(int(counts[2]), self.TPDM_RECORD),
               "D2bb": np.zeros(int(counts[0]), self.TPDM_RECORD)}
        check(self._lib.v2b_problem_tpdm_iwl_records(self._h, int(ncore), xh.ctypes.data, out["D2aa"].ctypes.data,
                                                     out["D2ab"].ctypes.data, out["D2bb"].ctypes.data))
        return out

    DM3_RECORD = np.dtype([("i", np.int32), ("j", np.int32), ("k", np.int32), ("l", np.int32),
                           ("m", np.int32), ("n", np.int32), ("value", np.float64)])

    def d3_entries(self, x, ncore=0):
        """{"D3aaa", "D3aab", "D3bba", "D3bbb"}: {entry: bytes} as
        WriteActive3PDM writes them (write_3pdm.cc:50-206): the records when
        there are any, then "length"."""
        xh = np.ascontiguousarray(x.detach().cpu().numpy() if hasattr(x, "detach") else x,
                                  dtype=np.float64)
        if xh.shape != (self.n_primal,):
            raise ValueError(f"x must hold {self.n_primal} values")
        counts = np.zeros(2, np.int64)
        check(self._lib.v2b_problem_d3_counts(self._h, counts.ctypes.data))
        rec = {name: np.zeros(int(counts[0 if name in ("D3aaa", "D3bbb") else 1]), self.DM3_RECORD)
               for name in ("D3aaa", "D3aab", "D3bba", "D3bbb")}
        check(self._lib.v2b_problem_d3_records(self._h, int(ncore), xh.ctypes.data,
                                               *[rec[k].ctypes.data for k in ("D3aaa", "D3aab", "D3bba", "D3bbb")]))
        return {name: ({name: r.tobytes()} if len(r) else {}) | {"length": np.int64(len(r)).tobytes()}
                for name, r in rec.items()}

    def rdm_entries(self, x, ncore=0):
        """{file: {entry: bytes}}: every entry hilbert's writers put in their
        PSIO files, byte for byte (the records when there are any, "length",
        and for the D2 files "NUMBER ACTIVE ORBITALS", "ACTIVE ORBITALS",
        "NUMBER INACTIVE ORBITALS" and, with core orbitals, "INACTIVE
        ORBITALS"; write_tpdm.cc:226-262, write_opdm.cc:108-113)."""
        recs = self.rdm_records(x, ncore)
        n, c = int(self.nmo), int(ncore)
        out = {}
        for name, r in recs.items():
            # an entry exists once something is written to it
            e = {name: r.tobytes()} if len(r) else {}
            e["length"] = np.int64(len(r)).tobytes()
            if name.startswith("D2"):
                e["NUMBER ACTIVE ORBITALS"] = np.int32(n).tobytes()
                e["ACTIVE ORBITALS"] = np.arange(c, c + n, dtype=np.int32).tobytes()
                e["NUMBER INACTIVE ORBITALS"] = np.int32(c).tobytes()
                if c:
                    e["INACTIVE ORBITALS"] = np.arange(c, dtype=np.int32).tobytes()
            out[name] = e
        return out

    def write_rdm_files(self, path, x, ncore=0):
        """Writes rdm_entries(x, ncore) to one .npz archive, one array per
        entry, named "<file>/<entry>" (the PSIO container itself is Psi4's)."""
        arrays = {f"{name}/{key}": np.frombuffer(val, np.uint8)
                  for name, ent in self.rdm_entries(x, ncore).items() for key, val in ent.items()}
        np.savez(path, **arrays)

    def pack_spatial_density(self, x):
        """hilbert's PackSpatialDensity of a device primal vector x (float64 CUDA
        tensor): (packed spin-summed active D2, packed D1), on the current stream"""
        import torch
        self._check_tensor(x, self.n_primal)
        n2, n1 = ctypes.c_long(), ctypes.c_long()
        check(self._lib.v2b_problem_pack_dims(self._h, ctypes.byref(n2), ctypes.byref(n1)))
        d2 = torch.empty(n2.value, dtype=torch.float64, device=x.device)
        d1 = torch.empty(n1.value, dtype=torch.float64, device=x.device)
        check(self._lib.v2b_problem_pack_spatial_density(self._h, _tptr(x), _tptr(d2), _tptr(d1),
                                                         self._stream()))
        return d2, d1

    def set_projection_mode(self, mode):
        """"refine" (default: warm refinement), "jacobi" (selective Jacobi on
        every block every iteration: the plain FP64 path) or "mixed" (warm
        refinement whose large blocks take an FP32 eigensolve, an FP64
        Rayleigh-Ritz step and FP64 Newton passes where refine would take
        block-Jacobi sweeps)"""
        check(self._lib.v2b_problem_set_projection_mode(self._h, {"refine": 0, "jacobi": 1, "mixed": 2}[mode]))

    def set_gemm_split(self, on=True):
        """the projection's GEMM tiles of large blocks cut along K when a
        launch has fewer tiles than CTA slots (default), or each in one piece"""
        check(self._lib.v2b_problem_set_gemm_split(self._h, int(bool(on))))

    def gemm_split_choice(self):
        """(S for the full tile list, S for the upper-tile list) chosen by the
        split autotuner when the projection plan was built; (0, 0) before"""
        full, upper = ctypes.c_int(), ctypes.c_int()
        check(self._lib.v2b_problem_gemm_split_choice(self._h, ctypes.byref(full), ctypes.byref(upper)))
        return full.value, upper.value

    REFINE_COUNTS = ("accepted", "jacobi", "passes", "clusters", "large_clusters",
                     "fallback_edges", "fallback_passes", "block_jacobi_sweeps", "fp32_eigensolves")

    def refine_counts(self):
        """counts of the warm eigen-refinement, keyed by REFINE_COUNTS"""
        v = (ctypes.c_long * len(self.REFINE_COUNTS))()
        check(self._lib.v2b_problem_refine_counts(self._h, v, len(v)))
        return dict(zip(self.REFINE_COUNTS, v))

    def stream_handle(self):
        return self._lib.v2b_problem_stream(self._h)


class DOCIProblem(V2RDMProblem):
    """One v2RDM-DOCI problem (hilbert's src/v2rdm_doci) on the same device
    path: b, c from h and (ij|kl), the random guess, A.x, A^T.y and the
    solves.  positivity is hilbert's POSITIVITY (D ... DQGT1T2; DQGT2 is D,
    Q, G and T2), optionally "+D3" for CONSTRAIN_D3."""

    def __init__(self, nmo, nalpha, nbeta, positivity="DQG"):
        lib = _capi.load()
        self._lib = lib
        h = ctypes.c_void_p()
        pos, *extras = positivity.upper().split("+")
        if pos not in _capi.POSITIVITY or not set(extras) <= {"D3"}:
            raise ValueError(f"DOCI POSITIVITY {positivity} is not one of "
                             f"{sorted(_capi.POSITIVITY)}, optionally +D3")
        code = _capi.POSITIVITY[pos] | (_capi.V2B_CONSTRAIN_D3 if extras else 0)
        check(lib.v2b_doci_problem_create(int(nmo), int(nalpha), int(nbeta), code, ctypes.byref(h)))
        self._sizes(h, nmo, nalpha, nbeta)

    def v2rdm_layout(self, x):
        """{"d2ab", "d2aa", "d2bb", "d1a", "d1b"}: the spin blocks of a DOCI
        solution as hilbert's DOCI PackSpatialDensity builds them
        (v2rdm_doci_solver.cc:1570-1597), flat, geminals numbered as in
        V2RDMProblem."""
        xh = np.ascontiguousarray(x.detach().cpu().numpy() if hasattr(x, "detach") else x,
                                  dtype=np.float64)
        if xh.shape != (self.n_primal,):
            raise ValueError(f"x must hold {self.n_primal} values")
        size = ctypes.c_long()
        check(self._lib.v2b_doci_v2rdm_layout(self._h, None, None, ctypes.byref(size)))
        out = np.zeros(size.value)
        check(self._lib.v2b_doci_v2rdm_layout(self._h, xh.ctypes.data, out.ctypes.data, ctypes.byref(size)))
        n = int(self.nmo)
        gab, gaa = n * n, n * (n - 1) // 2
        cuts = np.cumsum([gab * gab, gaa * gaa, gaa * gaa, n * n])
        return dict(zip(("d2ab", "d2aa", "d2bb", "d1a", "d1b"), np.split(out, cuts)))


class BatchProblem(V2RDMProblem):
    """Independent problems (V2RDMProblem / DOCIProblem parts) solved as one
    block-diagonal problem, every device launch covering all of them.  x, b,
    c and y are the parts' vectors concatenated in order (``split`` cuts a
    vector back into parts).  The parts may be closed afterwards."""

    def __init__(self, parts):
        lib = _capi.load()
        self._lib = lib
        parts = list(parts)
        handles = (ctypes.c_void_p * len(parts))(*[p._h.value if hasattr(p._h, "value") else p._h
                                                   for p in parts])
        h = ctypes.c_void_p()
        check(lib.v2b_batch_problem_create(handles, len(parts), ctypes.byref(h)))
        self._sizes(h, None, None, None)
        self.primal_cuts = np.cumsum([p.n_primal for p in parts])[:-1]
        self.dual_cuts = np.cumsum([p.n_dual for p in parts])[:-1]

    def split(self, v, dual=False):
        """The parts' pieces of a batch vector (host array or tensor)."""
        v = v.detach().cpu().numpy() if hasattr(v, "detach") else np.asarray(v)
        return np.split(v, self.dual_cuts if dual else self.primal_cuts)


class BPSDPSolver:
    """libsdp::BPSDPSolver with host callbacks (evaluate_Au / evaluate_ATu)."""

    def __init__(self, n_primal, n_dual, options):
        self._lib = _capi.load()
        self.n_primal, self.n_dual = int(n_primal), int(n_dual)
        o = options.sdp_options() if isinstance(options, Options) else options
        h = ctypes.c_void_p()
        check(self._lib.v2b_bpsdp_create(self.n_primal, self.n_dual, ctypes.byref(o), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        try:
            if self._h:
                self._lib.v2b_bpsdp_destroy(self._h)
        except Exception:
            pass

    def solve(self, x, b, c, primal_block_dims, maxiter, Au, ATu, monitor=None, print_level=1):
        """x (float64 numpy, updated in place); Au(in) / ATu(in) return numpy arrays."""
        nd, np_ = self.n_dual, self.n_primal

        def wrap(fn, n_in, n_out):
            def cb(out, inp, _data):
                vin = np.ctypeslib.as_array(inp, shape=(n_in,))
                vout = np.ctypeslib.as_array(out, shape=(n_out,))
                vout[:] = fn(vin)
            return SDP_CALLBACK(cb)

        cau = wrap(Au, np_, nd)
        catu = wrap(ATu, nd, np_)
        cmon = SDP_MONITOR(monitor) if monitor is not None else SDP_MONITOR()
        dims = np.ascontiguousarray(primal_block_dims, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.float64)
        c = np.ascontiguousarray(c, dtype=np.float64)
        rc = check(self._lib.v2b_bpsdp_solve(self._h, _dptr(x), _dptr(b), _dptr(c),
                                             dims.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                             len(dims), int(maxiter), cau, catu, cmon,
                                             int(print_level), None),
                   allow=(_capi.V2B_OK, _capi.V2B_NOT_CONVERGED))
        return rc == _capi.V2B_OK

    def is_converged(self):
        return bool(self._lib.v2b_bpsdp_is_converged(self._h))

    def get_mu(self):
        return self._lib.v2b_bpsdp_get_mu(self._h)

    def set_mu(self, mu):
        check(self._lib.v2b_bpsdp_set_mu(self._h, float(mu)))

    def get_y(self):
        out = np.zeros(self.n_dual)
        check(self._lib.v2b_bpsdp_get_y(self._h, _dptr(out)))
        return out

    def get_z(self):
        out = np.zeros(self.n_primal)
        check(self._lib.v2b_bpsdp_get_z(self._h, _dptr(out)))
        return out

    def set_y(self, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        check(self._lib.v2b_bpsdp_set_y(self._h, _dptr(y)))

    def set_z(self, z):
        z = np.ascontiguousarray(z, dtype=np.float64)
        check(self._lib.v2b_bpsdp_set_z(self._h, _dptr(z)))

    def iiter_total(self):
        return self._lib.v2b_bpsdp_iiter_total(self._h)

    def oiter_total(self):
        return self._lib.v2b_bpsdp_oiter_total(self._h)


def _check_unbuilt_options(options):
    # SDP_SOLVER (plugin.cc:246): hilbert offers libsdp's BPSDP and RRSDP
    # (v2rdm_solver.cc:424-447); only the boundary-point method is built here
    if str(options.get("SDP_SOLVER")).upper() != "BPSDP":
        raise NotImplementedError(f"SDP_SOLVER {options.get('SDP_SOLVER')}: only BPSDP is on the device path")
    # the generalized Pauli constraints (generalized_pauli*.cc) are not built
    if str(options.get("GPC_CONSTRAINTS")).upper() != "NONE":
        raise NotImplementedError(f"GPC_CONSTRAINTS {options.get('GPC_CONSTRAINTS')}: not on the device path")


class v2RDMHelper:
    """hilbert.v2RDMHelper (src/python_api/python_helpers.cc:104-113, 357-371).

    ``v2RDMHelper(nalpha, nbeta, nmo, h, g, options)`` builds the
    external-Hamiltonian problem (v2rdm_solver.cc:147-195);
    ``v2RDMHelper(None, options)`` with HUBBARD_HAMILTONIAN builds the 1D
    Hubbard ring (v2rdm_solver.cc:839-962).  Molecular wavefunctions need Psi4
    and are outside this package.
    """

    def __init__(self, *args):
        if len(args) == 6:
            nalpha, nbeta, nmo, h, g, options = args
            self.options = options if isinstance(options, Options) else Options(options)
            self._hubbard = False
        elif len(args) == 2:
            _ref_wfn, options = args
            self.options = options if isinstance(options, Options) else Options(options)
            if not self.options.get("HUBBARD_HAMILTONIAN"):
                raise NotImplementedError("molecular Hamiltonians need Psi4; use the external-"
                                          "Hamiltonian constructor or HUBBARD_HAMILTONIAN")
            nspins = int(self.options.get("N_HUBBARD_SPINS"))
            if nspins % 2:
                raise ValueError("Hubbard model only works for even numbers of electrons currently.")
            nmo = int(self.options.get("N_HUBBARD_SITES"))
            nalpha = nbeta = nspins // 2
            self._hubbard = True
        else:
            raise TypeError("v2RDMHelper(nalpha, nbeta, nmo, h, g, options) or v2RDMHelper(ref_wfn, options)")
        o = self.options
        _check_unbuilt_options(o)
        if o.get("RESTART_FROM_CHECKPOINT_FILE"):
            # v2rdm_solver.cc:958-959, 1081-1082
            kind = "Hubbard" if self._hubbard else "external"
            raise ValueError(f"RESTART_FROM_CHECKPOINT_FILE is incompatible with {kind} Hamiltonian "
                             "(restart a problem with hilbert_b200.checkpoint.restart)")
        pos = (o.get("POSITIVITY") + ("+D3" if o.get("CONSTRAIN_D3") else "")
               + ("+Q3" if o.get("CONSTRAIN_Q3") else "") + ("+E3" if o.get("CONSTRAIN_E3") else "")
               + ("+F3" if o.get("CONSTRAIN_F3") else "") + ("+D4" if o.get("CONSTRAIN_D4") else ""))
        self.problem = V2RDMProblem(nmo, nalpha, nbeta, pos, o.get("CONSTRAIN_SPIN"),
                                    o.get("CONSTRAIN_SZ"), hubbard_multiplicity=self._hubbard)
        p = self.problem
        if self._hubbard:
            self.c = p.c_hubbard(o.get("HUBBARD_T"), o.get("HUBBARD_U"))
        else:
            self.c = p.c_external(h, g)
        self.b = p.b()
        self.x = None
        self.stats = None
        self.variables = {}

    def _sdp_options(self):
        # hilbert solves in calls of MU_UPDATE_FREQUENCY iterations for the
        # Hubbard and external Hamiltonians, whatever OPTIMIZE_ORBITALS says
        # (v2rdm_solver.cc:1298-1301)
        return self.options

    def compute_energy(self, monitor=None):
        p = self.problem
        x0 = p.guess(self.options.get("TPDM_GUESS"))
        self.x, self.stats = p.solve(x0, self.b, self.c, self._sdp_options(), monitor)
        e = float(self.c @ self.x)
        # enuc = efzc = 0 for Hubbard / external Hamiltonians (v2rdm_solver.cc:851-853, 972-974)
        self.variables["CURRENT ENERGY"] = e
        self.variables["v2RDM TOTAL ENERGY"] = e
        self.files = self.written_files()
        return e

    def written_files(self):
        """The files hilbert's compute_energy writes after the solve under the
        write options (v2rdm_solver.cc:1474-1516), {file: {entry: bytes}}:
        TPDM_WRITE (WriteActiveTPDM, write_tpdm.cc:521-602: the active records
        and "length"), TPDM_WRITE_FULL (WriteTPDM), TPDM_WRITE_SPIN_FREE,
        OPDM_WRITE_FULL, 3PDM_WRITE with CONSTRAIN_D3 (WriteActive3PDM,
        write_3pdm.cc:50-206); with DERTYPE FIRST or WRITE_CHECKPOINT_FILE the
        checkpoint ("CHECKPOINT", entries as in hilbert_b200.checkpoint), and
        with DERTYPE FIRST the IWL 2-RDM records ("IWL"; the orbital
        Lagrangian that hilbert also builds then is not)."""
        o, p, x = self.options, self.problem, self.x
        out = {}
        first = str(o.get("DERTYPE")).upper() == "FIRST"
        if not (first or any(o.get(k) for k in ("TPDM_WRITE", "TPDM_WRITE_FULL", "TPDM_WRITE_SPIN_FREE",
                                                "OPDM_WRITE_FULL", "WRITE_CHECKPOINT_FILE", "3PDM_WRITE"))):
            return out
        entries = p.rdm_entries(x)
        if o.get("TPDM_WRITE"):
            n = int(p.nmo)
            counts = {"D2aa": n * (n - 1) * n * (n - 1), "D2bb": n * (n - 1) * n * (n - 1), "D2ab": n ** 4}
            for name, cnt in counts.items():   # the leading active-active records
                rec = np.frombuffer(entries[name].get(name, b""), self.problem.TPDM_RECORD)[:cnt]
                out[name] = ({name: rec.tobytes()} if cnt else {}) | {"length": np.int64(cnt).tobytes()}
        if o.get("TPDM_WRITE_FULL"):
            out.update({k: entries[k] for k in ("D2aa", "D2bb", "D2ab")})
        if o.get("TPDM_WRITE_SPIN_FREE"):
            out["D2"] = entries["D2"]
        if o.get("OPDM_WRITE_FULL"):
            out.update({k: entries[k] for k in ("D1a", "D1b")})
        if o.get("3PDM_WRITE") and o.get("CONSTRAIN_D3"):
            out.update(p.d3_entries(x))
        if first or o.get("WRITE_CHECKPOINT_FILE"):
            out["CHECKPOINT"] = {"MU": np.float64(p.get_mu()).tobytes(), "PRIMAL": x.tobytes(),
                                 "DUAL 1": p.get_y().tobytes(), "DUAL 2": p.get_z().tobytes()}
        if first:
            out["IWL"] = p.tpdm_iwl_records(x)
        return out

    def get_opdm(self):
        """Spin-summed active 1-RDM D1a + D1b (python_api.cc:374-394, C1 active block)."""
        n = self.problem.nmo
        o = self.options
        off = block_offsets(n, self.problem.nalpha, self.problem.nbeta, o.get("POSITIVITY"),
                            o.get("CONSTRAIN_SPIN"))
        d1a = self.x[off["d1a"]:off["d1a"] + n * n].reshape(n, n)
        d1b = self.x[off["d1b"]:off["d1b"] + n * n].reshape(n, n)
        return d1a + d1b


class v2RDM_DOCIHelper:
    """hilbert.v2RDM_DOCIHelper (src/python_api/python_helpers.cc:99-101, 339-352).

    hilbert builds it from a Psi4 wavefunction; here
    ``v2RDM_DOCIHelper(nalpha, nbeta, nmo, h, g, options)`` takes what the
    solver reads from one: the electron counts and the integrals h and
    g = (ij|kl) of the nmo orbitals.  POSITIVITY and CONSTRAIN_D3 choose the
    conditions (v2rdm_doci_solver.cc:427-494).  With OPTIMIZE_ORBITALS and the
    density-fitting factors ``B`` (naux x nmo x nmo, g = sum_Q B^Q B^Q) the
    orbitals are optimised as well (orbital.doci_casscf); given g alone, its
    exact factors (orbital.eri_factors) serve as B."""

    def __init__(self, nalpha, nbeta, nmo, h, g, options, B=None):
        self.options = options if isinstance(options, Options) else Options(options)
        o = self.options
        _check_unbuilt_options(o)
        pos = o.get("POSITIVITY") + ("+D3" if o.get("CONSTRAIN_D3") else "")
        self.problem = DOCIProblem(nmo, nalpha, nbeta, pos)
        self.h = np.ascontiguousarray(h, dtype=np.float64).reshape(nmo, nmo)
        self.B = None if B is None else np.ascontiguousarray(B, dtype=np.float64)
        if g is None:
            if self.B is None:
                raise ValueError("give g = (ij|kl) or the density-fitting factors B")
            g = np.einsum("Qij,Qkl->ijkl", self.B, self.B)
        self._g = np.ascontiguousarray(g, dtype=np.float64)
        self.c = self.problem.c_external(self.h, self._g)
        self.b = self.problem.b()
        self.x = None
        self.stats = None
        self.variables = {}

    def _sdp_options(self):
        # DOCI calls solve(ORBOPT_FREQUENCY) until converged, updating mu
        # after each call (v2rdm_doci_solver.cc:1113-1137)
        o = Options({k: v for k, v in self.options._v.items()})
        o.set("MU_UPDATE_FREQUENCY", int(self.options.get("ORBOPT_FREQUENCY")))
        return o

    def compute_energy(self, monitor=None, macro_iterations=None):
        """The DOCI energy.  With OPTIMIZE_ORBITALS it runs hilbert's loop
        (v2rdm_doci_solver.cc:1111-1137): solve() calls of ORBOPT_FREQUENCY
        SDP iterations that carry x, y, z and mu over, each followed by a
        focas orbital step (ORBOPT_MAXITER iterations at most), until the SDP
        has converged and the orbital step met ORBOPT_GRADIENT_CONVERGENCE and
        ORBOPT_ENERGY_CONVERGENCE.  MAXITER bounds the SDP iterations of all
        calls together; macro_iterations (None: no cap) the rounds.  The
        energy is c.x in the final orbitals, where hilbert takes it (:1142).
        stats["converged"] is False when a cap ended the loop first."""
        p = self.problem
        o = self.options
        if o.get("OPTIMIZE_ORBITALS"):
            import torch
            if not torch.cuda.is_available():
                raise _capi.V2BError(_capi.V2B_NO_DEVICE, "v2RDM-DOCI orbital optimisation needs a CUDA device")
        if o.get("OPTIMIZE_ORBITALS") and self.B is None and self._g is not None:
            from . import orbital
            self.B = orbital.eri_factors(self._g).numpy()
        if o.get("OPTIMIZE_ORBITALS") and self.B is not None:
            import torch
            from . import orbital
            dev = torch.device("cuda", torch.cuda.current_device())
            solve = orbital.active_solver(p, o, frequency=int(o.get("ORBOPT_FREQUENCY")))
            info = {}
            energies, gnorms, _, _ = orbital.doci_casscf(
                torch.from_numpy(self.h).to(dev), torch.from_numpy(self.B).to(dev), p.nalpha, p.nbeta,
                solve_active=solve, macro_iterations=macro_iterations,
                g_conv=float(o.get("ORBOPT_GRADIENT_CONVERGENCE")),
                e_conv=float(o.get("ORBOPT_ENERGY_CONVERGENCE")), info=info,
                orbopt_maxiter=int(o.get("ORBOPT_MAXITER")))
            converged = info["sdp_converged"] and info["orbitals_converged"]
            self.stats = {"energies": energies, "orbital_gradients": gnorms, "converged": converged,
                          "sdp_converged": info["sdp_converged"],
                          "orbitals_converged": info["orbitals_converged"], "rounds": info["rounds"],
                          "oiter": solve.oiter, "iiter": solve.iiter}
            e = info["final_energy"]
        else:
            self.x, self.stats = p.solve(p.guess("RANDOM"), self.b, self.c, self._sdp_options(), monitor)
            e = float(self.c @ self.x)
            n = p.nmo
            # natural-orbital occupations 2 D1(i) (v2rdm_doci_solver.cc:1148-1153)
            self.occupations = 2.0 * self.x[2 * n * n:2 * n * n + n]
        # enuc = efzc = 0 for given integrals (v2rdm_doci_solver.cc:1157-1158)
        self.variables["CURRENT ENERGY"] = e
        self.variables["v2RDM-DOCI TOTAL ENERGY"] = e
        return e


def block_layout(nmo, nalpha, nbeta, positivity="DQG", constrain_spin=True):
    """[(name, dim)] in the primal order of set_primal_offsets (v2rdm_solver.cc:3729-4079)."""
    n = int(nmo)
    gab, gaa = n * n, n * (n - 1) // 2
    pos, *extras = positivity.upper().split("+")
    blocks = [("d2ab", gab), ("d2aa", gaa), ("d2bb", gaa)]
    if constrain_spin:
        blocks.append(("d200", gab if nalpha == nbeta else 2 * gab))
    blocks += [("d1a", n), ("d1b", n), ("q1a", n), ("q1b", n)]
    t_opts = ("DQGT1", "DQGT2", "DQGT1T2", "DQGT")
    if pos in ("DQ", "DQG") + t_opts:
        blocks += [("q2ab", gab), ("q2aa", gaa), ("q2bb", gaa)]
    if pos in ("DG", "DQG") + t_opts:
        blocks += [("g2ab", gab), ("g2ba", gab), ("g2aa", 2 * gab)]
    aaa, aab, aba = n * (n - 1) * (n - 2) // 6, n * (n - 1) // 2 * n, n ** 3
    if pos in ("DQGT1", "DQGT1T2", "DQGT"):
        blocks += [("t1aaa", aaa), ("t1bbb", aaa), ("t1aab", aab), ("t1bba", aab)]
    if pos in ("DQGT2", "DQGT1T2", "DQGT"):
        blocks += [("t2aaa", aab + aba), ("t2bbb", aab + aba), ("t2aab", aab), ("t2bba", aab)]
    if "E3" in extras:
        blocks += [("e3aaa", aab + aba), ("e3bbb", aab + aba), ("e3aab", aab), ("e3bba", aab)]
    if "F3" in extras:
        blocks += [("f3aaa", aab + aba), ("f3bbb", aab + aba), ("f3aab", aab), ("f3bba", aab)]
    if "Q3" in extras:
        blocks += [("q3aaa", aaa), ("q3bbb", aaa), ("q3aab", aab), ("q3bba", aab)]
    if set(extras) & {"D3", "Q3", "E3", "F3", "D4"}:
        blocks += [("d3aaa", aaa), ("d3bbb", aaa), ("d3aab", aab), ("d3bba", aab)]
    if "D4" in extras:
        q4, q31, q22 = n * (n - 1) * (n - 2) * (n - 3) // 24, aaa * n, gaa * gaa
        blocks += [("d4aaaa", q4), ("d4aaab", q31), ("d4aabb", q22), ("d4bbba", q31), ("d4bbbb", q4)]
    return blocks


def block_offsets(nmo, nalpha, nbeta, positivity="DQG", constrain_spin=True):
    off, o = {}, 0
    for name, d in block_layout(nmo, nalpha, nbeta, positivity, constrain_spin):
        off[name] = o
        o += d * d
    return off

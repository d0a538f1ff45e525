"""ORACLE -- test infrastructure only.

ctypes bindings for the v2RDM-DOCI restatement (``doci_oracle.c``) and for
hilbert's own compiled DOCI code (``_ref/libdoci_ref.so``, built by
``build_ref.sh``), both behind one problem interface: sizes, block
dimensions, b, c, the random guess, A.x and A^T.y.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libdoci_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdoci_ref.so")
POSITIVITY = {"D": 0, "DQ": 1, "DG": 2, "DQG": 3, "DQGT2": 4, "DQGT1": 5, "DQGT1T2": 6}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_libs = {}


def build_oracle(force=False):
    """Compile doci_oracle.c with gcc (no FMA contraction, like the reference build)."""
    src = os.path.join(HERE, "doci_oracle.c")
    if not force and os.path.exists(ORACLE_SO) and os.path.getmtime(ORACLE_SO) >= os.path.getmtime(src):
        return ORACLE_SO
    os.makedirs(os.path.dirname(ORACLE_SO), exist_ok=True)
    subprocess.check_call(["gcc", "-std=c99", "-O2", "-fPIC", "-ffp-contract=off", "-shared",
                           src, "-o", ORACLE_SO])
    return ORACLE_SO


def ref_available():
    return os.path.exists(REF_SO)


def _bind(lib, prefix):
    for f in ("n_primal", "n_dual"):
        getattr(lib, prefix + f).restype = ctypes.c_long
        getattr(lib, prefix + f).argtypes = [ctypes.c_void_p]
    getattr(lib, prefix + "n_blocks").argtypes = [ctypes.c_void_p]
    getattr(lib, prefix + "block_dims").argtypes = [ctypes.c_void_p, _ip]
    getattr(lib, prefix + "destroy").argtypes = [ctypes.c_void_p]
    getattr(lib, prefix + "Au").argtypes = [ctypes.c_void_p, _dp, _dp]
    getattr(lib, prefix + "ATu").argtypes = [ctypes.c_void_p, _dp, _dp]
    getattr(lib, prefix + "create").restype = ctypes.c_void_p


def _lib(kind):
    if kind not in _libs:
        if kind == "oracle":
            lib = ctypes.CDLL(build_oracle())
            _bind(lib, "dco_")
            lib.dco_create.argtypes = [ctypes.c_int] * 5
            lib.dco_build_b.argtypes = [ctypes.c_void_p, _dp]
            lib.dco_build_c.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
            lib.dco_guess.argtypes = [ctypes.c_void_p, _dp]
        else:
            if not ref_available():
                raise FileNotFoundError("reference DOCI library not built: run oracle/build_ref.sh")
            lib = ctypes.CDLL(REF_SO)
            _bind(lib, "doci_ref_")
            lib.doci_ref_create.argtypes = ([ctypes.c_int] * 3 + [ctypes.c_char_p, ctypes.c_int]
                                            + [ctypes.c_void_p] * 2)
            lib.doci_ref_last_error.restype = ctypes.c_char_p
            for f in ("get_b", "get_c", "get_x"):
                getattr(lib, "doci_ref_" + f).argtypes = [ctypes.c_void_p, _dp]
            lib.doci_ref_pack_dims.restype = ctypes.c_long
            lib.doci_ref_pack_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
            lib.doci_ref_pack_spatial.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        _libs[kind] = lib
    return _libs[kind]


def _split(positivity):
    pos, *extras = positivity.upper().split("+")
    if pos not in POSITIVITY or not set(extras) <= {"D3"}:
        raise ValueError(f"unknown DOCI POSITIVITY {positivity}")
    return pos, bool(extras)


class _Base:
    def close(self):
        if getattr(self, "_h", None):
            getattr(self._lib, self._prefix + "destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _sizes(self):
        lib, pre = self._lib, self._prefix
        self.n_primal = getattr(lib, pre + "n_primal")(self._h)
        self.n_dual = getattr(lib, pre + "n_dual")(self._h)
        self.dims = np.zeros(getattr(lib, pre + "n_blocks")(self._h), np.int32)
        getattr(lib, pre + "block_dims")(self._h, self.dims)

    def Au(self, x):
        out = np.zeros(self.n_dual)
        getattr(self._lib, self._prefix + "Au")(self._h, np.ascontiguousarray(x, np.float64), out)
        return out

    def ATu(self, y):
        out = np.zeros(self.n_primal)
        getattr(self._lib, self._prefix + "ATu")(self._h, np.ascontiguousarray(y, np.float64), out)
        return out


class DociOracle(_Base):
    """The C restatement of one v2RDM-DOCI problem (test-side checker)."""
    _prefix = "dco_"

    def __init__(self, n, na, nb, positivity="DQG"):
        self._lib = _lib("oracle")
        pos, d3 = _split(positivity)
        self._h = self._lib.dco_create(n, na, nb, POSITIVITY[pos], int(d3))
        if not self._h:
            raise ValueError(f"DOCI oracle refuses n={n} na={na} nb={nb} {positivity}")
        self._sizes()

    def b(self):
        out = np.zeros(self.n_dual)
        self._lib.dco_build_b(self._h, out)
        return out

    def c(self, h, g):
        out = np.zeros(self.n_primal)
        self._lib.dco_build_c(self._h, np.ascontiguousarray(h, np.float64),
                              np.ascontiguousarray(g, np.float64), out)
        return out

    def guess(self):
        out = np.zeros(self.n_primal)
        self._lib.dco_guess(self._h, out)
        return out


class DociRef(_Base):
    """hilbert's own compiled DOCI code for one problem (h, g optional)."""
    _prefix = "doci_ref_"

    def __init__(self, n, na, nb, positivity="DQG", h=None, g=None):
        self._lib = lib = _lib("ref")
        pos, d3 = _split(positivity)
        hh = None if h is None else np.ascontiguousarray(h, np.float64)
        gg = None if g is None else np.ascontiguousarray(g, np.float64)
        self._h = lib.doci_ref_create(n, na, nb, pos.encode(), int(d3),
                                      None if hh is None else hh.ctypes.data,
                                      None if gg is None else gg.ctypes.data)
        if not self._h:
            raise RuntimeError(lib.doci_ref_last_error().decode())
        self._sizes()
        self.b, self.x0 = np.zeros(self.n_dual), np.zeros(self.n_primal)
        lib.doci_ref_get_b(self._h, self.b)
        lib.doci_ref_get_x(self._h, self.x0)
        self.c = None
        if hh is not None:
            self.c = np.zeros(self.n_primal)
            lib.doci_ref_get_c(self._h, self.c)


def _ref_pack(self, x):
    """hilbert's DOCI PackSpatialDensity (v2rdm_doci_solver.cc:1568-1703) of x:
    the packed spin-summed active D2 and D1"""
    d1n = ctypes.c_long()
    d2n = self._lib.doci_ref_pack_dims(self._h, ctypes.byref(d1n))
    d2, d1 = np.zeros(d2n), np.zeros(d1n.value)
    self._lib.doci_ref_pack_spatial(self._h, np.ascontiguousarray(x, np.float64), d2, d1)
    return d2, d1


DociRef.pack_spatial_density = _ref_pack


def _ref_write_tpdm(self, x):
    """Runs the reference DOCI WriteTPDM on x; {file: {entry: bytes}} for the
    D2aa (unit 270), D2ab (271) and D2bb (272) files it writes."""
    lib = self._lib
    lib.doci_ref_write_tpdm.argtypes = [ctypes.c_void_p, _dp]
    lib.doci_ref_psio_entry.restype = ctypes.c_long
    lib.doci_ref_psio_entry.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p]
    lib.doci_ref_write_tpdm(self._h, np.ascontiguousarray(x, np.float64))
    out = {}
    for name, unit in (("D2aa", 270), ("D2ab", 271), ("D2bb", 272)):
        out[name] = {}
        for key in (name, "length", "NUMBER ACTIVE ORBITALS", "ACTIVE ORBITALS",
                    "NUMBER INACTIVE ORBITALS", "INACTIVE ORBITALS"):
            size = lib.doci_ref_psio_entry(unit, key.encode(), None)
            if size < 0:
                continue
            buf = ctypes.create_string_buffer(max(size, 1))
            lib.doci_ref_psio_entry(unit, key.encode(), buf)
            out[name][key] = buf.raw[:size]
    return out


DociRef.write_tpdm = _ref_write_tpdm


def symmetric_integrals(rng, n):
    """Random real h and (ij|kl) with the 8-fold symmetry of real orbitals."""
    h = rng.standard_normal((n, n))
    g = rng.standard_normal((n,) * 4)
    g = g + g.transpose(1, 0, 2, 3)
    g = g + g.transpose(0, 1, 3, 2)
    g = g + g.transpose(2, 3, 0, 1)
    return h + h.T, g


def seniority_zero_ci(h, g, npair):
    """Exact DOCI energy: the lowest eigenvalue of the Hamiltonian in the
    basis of closed-shell pair determinants (each orbital empty or doubly
    occupied).  <I|H|I> = sum_i (2 h_ii + (ii|ii)) + sum_{i<j} (4 (ii|jj) - 2 (ij|ij))
    over the pairs of I; moving one pair i -> a couples I and J by (ia|ia)."""
    import itertools
    n = h.shape[0]
    dets = list(itertools.combinations(range(n), npair))
    index = {d: k for k, d in enumerate(dets)}
    H = np.zeros((len(dets), len(dets)))
    for k, d in enumerate(dets):
        occ = set(d)
        H[k, k] = (sum(2.0 * h[i, i] + g[i, i, i, i] for i in d)
                   + sum(4.0 * g[i, i, j, j] - 2.0 * g[i, j, i, j] for i, j in itertools.combinations(d, 2)))
        for i in d:
            for a in range(n):
                if a not in occ:
                    H[index[tuple(sorted((occ - {i}) | {a}))], k] = g[i, a, i, a]
    return float(np.linalg.eigvalsh(H)[0])

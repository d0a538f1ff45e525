"""ORACLE -- test infrastructure only.

ctypes bindings for the C restatement (``v2rdm_oracle.c``) and for the
reference build (``_ref/libv2rdm_ref.so``), both exposing the same problem
interface: sizes, block dimensions, index tables, b, c, guesses, A.x, A^T.y.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libv2rdm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libv2rdm_ref.so")

POSITIVITY = {"D": 0, "DQ": 1, "DG": 2, "DQG": 3, "DQGT2": 4, "DQGT1": 5, "DQGT1T2": 6}
BLOCK_NAMES = ("d2ab", "d2aa", "d2bb", "d200", "d1a", "d1b", "q1a", "q1b",
               "q2ab", "q2aa", "q2bb", "g2ab", "g2ba", "g2aa", "t2aaa", "t2bbb", "t2aab", "t2bba",
               "t1aaa", "t1bbb", "t1aab", "t1bba", "d3aaa", "d3bbb", "d3aab", "d3bba",
               "q3aaa", "q3bbb", "q3aab", "q3bba", "e3aaa", "e3bbb", "e3aab", "e3bba",
               "f3aaa", "f3bbb", "f3aab", "f3bba", "d4aaaa", "d4aaab", "d4aabb", "d4bbba", "d4bbbb")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build_oracle(force=False):
    """Compile v2rdm_oracle.c with gcc (no FMA contraction, like the reference build)."""
    src = os.path.join(HERE, "v2rdm_oracle.c")
    if not force and os.path.exists(ORACLE_SO) and os.path.getmtime(ORACLE_SO) >= os.path.getmtime(src):
        return ORACLE_SO
    os.makedirs(os.path.dirname(ORACLE_SO), exist_ok=True)
    subprocess.check_call(["gcc", "-std=c99", "-O2", "-fPIC", "-ffp-contract=off", "-shared",
                           src, "-o", ORACLE_SO, "-lm"])
    return ORACLE_SO


_olib = None
_rlib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        lib = ctypes.CDLL(build_oracle())
        lib.v2o_create.restype = ctypes.c_void_p
        lib.v2o_create.argtypes = [ctypes.c_int] * 7
        lib.v2o_destroy.argtypes = [ctypes.c_void_p]
        for f in ("v2o_n_primal", "v2o_n_dual"):
            getattr(lib, f).restype = ctypes.c_long
            getattr(lib, f).argtypes = [ctypes.c_void_p]
        lib.v2o_n_blocks.argtypes = [ctypes.c_void_p]
        lib.v2o_block_dims.argtypes = [ctypes.c_void_p, _ip]
        lib.v2o_gems.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        lib.v2o_tables.argtypes = [ctypes.c_void_p, _ip, _ip, _ip, _ip]
        lib.v2o_offsets.argtypes = [ctypes.c_void_p, _lp]
        lib.v2o_build_b.argtypes = [ctypes.c_void_p, _dp]
        lib.v2o_build_c_hubbard.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp]
        lib.v2o_build_c_external.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        lib.v2o_guess_random.argtypes = [ctypes.c_void_p, _dp]
        lib.v2o_guess_hf.argtypes = [ctypes.c_void_p, _dp]
        lib.v2o_Au.argtypes = [ctypes.c_void_p, _dp, _dp]
        lib.v2o_ATu.argtypes = [ctypes.c_void_p, _dp, _dp]
        _olib = lib
    return _olib


def ref_available():
    return os.path.exists(REF_SO)


def _ref_lib():
    global _rlib
    if _rlib is None:
        if not ref_available():
            raise FileNotFoundError("reference oracle not built: run oracle/build_ref.sh")
        lib = ctypes.CDLL(REF_SO)
        lib.v2b_ref_create.restype = ctypes.c_void_p
        lib.v2b_ref_create.argtypes = ([ctypes.c_int] * 3 + [ctypes.c_char_p] + [ctypes.c_int] * 3
                                       + [ctypes.c_double] * 2 + [ctypes.c_void_p] * 2 + [ctypes.c_int])
        lib.v2b_ref_destroy.argtypes = [ctypes.c_void_p]
        lib.v2b_ref_last_error.restype = ctypes.c_char_p
        for f in ("v2b_ref_n_primal", "v2b_ref_n_dual"):
            getattr(lib, f).restype = ctypes.c_long
            getattr(lib, f).argtypes = [ctypes.c_void_p]
        lib.v2b_ref_n_blocks.argtypes = [ctypes.c_void_p]
        lib.v2b_ref_block_dims.argtypes = [ctypes.c_void_p, _ip]
        lib.v2b_ref_block_offset.restype = ctypes.c_long
        lib.v2b_ref_block_offset.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        for f in ("v2b_ref_get_b", "v2b_ref_get_c", "v2b_ref_get_x"):
            getattr(lib, f).argtypes = [ctypes.c_void_p, _dp]
        lib.v2b_ref_Au.argtypes = [ctypes.c_void_p, _dp, _dp]
        lib.v2b_ref_ATu.argtypes = [ctypes.c_void_p, _dp, _dp]
        lib.v2b_ref_pack_dims.restype = ctypes.c_long
        lib.v2b_ref_pack_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
        lib.v2b_ref_pack_spatial.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        lib.v2b_ref_gems.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        lib.v2b_ref_tables.argtypes = [ctypes.c_void_p, _ip, _ip, _ip, _ip]
        _rlib = lib
    return _rlib


class OracleProblem:
    """C restatement of one C1 v2RDM problem (test-side checker)."""

    def __init__(self, n, na, nb, positivity="DQG", constrain_spin=True, constrain_sz=True,
                 hubbard=None, h=None, g=None):
        lib = _oracle_lib()
        self.n, self.na, self.nb = n, na, nb
        self.positivity = positivity
        self.hubbard = hubbard
        base, *extras = positivity.split("+")
        if not set(extras) <= {"D3", "Q3", "E3", "F3", "D4"}:
            raise ValueError(f"unknown constraint suffix in {positivity!r}")
        code = (POSITIVITY[base] | (16 if "D3" in extras else 0) | (32 if "Q3" in extras else 0)
                | (64 if "E3" in extras else 0) | (128 if "F3" in extras else 0)
                | (256 if "D4" in extras else 0))
        p = lib.v2o_create(n, na, nb, code, int(constrain_spin),
                           int(constrain_sz), int(hubbard is not None))
        if not p:
            raise ValueError("invalid problem")
        self._p = ctypes.c_void_p(p)
        self._lib = lib
        self.n_primal = lib.v2o_n_primal(self._p)
        self.n_dual = lib.v2o_n_dual(self._p)
        nbk = lib.v2o_n_blocks(self._p)
        self.dims = np.zeros(nbk, np.int32)
        lib.v2o_block_dims(self._p, self.dims)
        gab, gaa = ctypes.c_int(), ctypes.c_int()
        lib.v2o_gems(self._p, ctypes.byref(gab), ctypes.byref(gaa))
        self.gab, self.gaa = gab.value, gaa.value
        offs = np.zeros(len(BLOCK_NAMES), np.int64)
        lib.v2o_offsets(self._p, offs)
        self.offsets = {k: int(v) for k, v in zip(BLOCK_NAMES, offs) if v >= 0}
        self.b = np.zeros(self.n_dual)
        lib.v2o_build_b(self._p, self.b)
        self.c = np.zeros(self.n_primal)
        if hubbard is not None:
            t, U = hubbard
            lib.v2o_build_c_hubbard(self._p, float(t), float(U), self.c)
        elif h is not None:
            lib.v2o_build_c_external(self._p, np.ascontiguousarray(h, np.float64).ravel(),
                                     np.ascontiguousarray(g, np.float64).ravel(), self.c)

    def __del__(self):
        try:
            self._lib.v2o_destroy(self._p)
        except Exception:
            pass

    def tables(self):
        n = self.n
        bas_ab = np.zeros(2 * max(self.gab, 1), np.int32)
        bas_aa = np.zeros(2 * max(self.gaa, 1), np.int32)
        ibas_ab = np.zeros(n * n, np.int32)
        ibas_aa = np.zeros(n * n, np.int32)
        self._lib.v2o_tables(self._p, bas_ab, ibas_ab, bas_aa, ibas_aa)
        return (bas_ab[:2 * self.gab].reshape(-1, 2), ibas_ab.reshape(n, n),
                bas_aa[:2 * self.gaa].reshape(-1, 2), ibas_aa.reshape(n, n))

    def guess(self, kind="random"):
        x = np.zeros(self.n_primal)
        (self._lib.v2o_guess_hf if kind == "hf" else self._lib.v2o_guess_random)(self._p, x)
        return x

    def Au(self, x):
        out = np.zeros(self.n_dual)
        self._lib.v2o_Au(self._p, np.ascontiguousarray(x, np.float64), out)
        return out

    def ATu(self, y):
        out = np.zeros(self.n_primal)
        self._lib.v2o_ATu(self._p, np.ascontiguousarray(y, np.float64), out)
        return out


class RefProblem:
    """hilbert's own map code compiled by build_ref.sh (the pin for OracleProblem)."""

    def __init__(self, n, na, nb, positivity="DQG", constrain_spin=True, constrain_sz=True,
                 hubbard=None, h=None, g=None, guess="random"):
        lib = _ref_lib()
        self._lib = lib
        hp = gp = None
        if hubbard is None:
            self._h = np.ascontiguousarray(h, np.float64).ravel()
            self._g = np.ascontiguousarray(g, np.float64).ravel()
            hp, gp = self._h.ctypes.data, self._g.ctypes.data
            t, U = 0.0, 0.0
        else:
            t, U = hubbard
        p = lib.v2b_ref_create(n, na, nb, positivity.encode(), int(constrain_spin), int(constrain_sz),
                               int(hubbard is not None), float(t), float(U), hp, gp,
                               int(guess == "hf"))
        if not p:
            raise RuntimeError(lib.v2b_ref_last_error().decode())
        self._p = ctypes.c_void_p(p)
        self.n = n
        self.n_primal = lib.v2b_ref_n_primal(self._p)
        self.n_dual = lib.v2b_ref_n_dual(self._p)
        nbk = lib.v2b_ref_n_blocks(self._p)
        self.dims = np.zeros(nbk, np.int32)
        lib.v2b_ref_block_dims(self._p, self.dims)
        gab, gaa = ctypes.c_int(), ctypes.c_int()
        lib.v2b_ref_gems(self._p, ctypes.byref(gab), ctypes.byref(gaa))
        self.gab, self.gaa = gab.value, gaa.value
        self.offsets = {}
        for k in BLOCK_NAMES:
            v = lib.v2b_ref_block_offset(self._p, k.encode())
            if v >= 0:
                self.offsets[k] = int(v)
        self.b = np.zeros(self.n_dual)
        lib.v2b_ref_get_b(self._p, self.b)
        self.c = np.zeros(self.n_primal)
        lib.v2b_ref_get_c(self._p, self.c)
        self.x0 = np.zeros(self.n_primal)
        lib.v2b_ref_get_x(self._p, self.x0)

    def __del__(self):
        try:
            self._lib.v2b_ref_destroy(self._p)
        except Exception:
            pass

    def tables(self):
        n = self.n
        bas_ab = np.zeros(2 * max(self.gab, 1), np.int32)
        bas_aa = np.zeros(2 * max(self.gaa, 1), np.int32)
        ibas_ab = np.zeros(n * n, np.int32)
        ibas_aa = np.zeros(n * n, np.int32)
        self._lib.v2b_ref_tables(self._p, bas_ab, ibas_ab, bas_aa, ibas_aa)
        return (bas_ab[:2 * self.gab].reshape(-1, 2), ibas_ab.reshape(n, n),
                bas_aa[:2 * self.gaa].reshape(-1, 2), ibas_aa.reshape(n, n))

    def Au(self, x):
        out = np.zeros(self.n_dual)
        if self._lib.v2b_ref_Au(self._p, out, np.ascontiguousarray(x, np.float64)):
            raise RuntimeError(self._lib.v2b_ref_last_error().decode())
        return out

    def pack_spatial_density(self, x):
        """hilbert's PackSpatialDensity (v2rdm_solver.cc:3110-3219) of x: the
        packed spin-summed active D2 (n(n+1)/2 geminals, lower triangle) and D1"""
        d1n = ctypes.c_long()
        d2n = self._lib.v2b_ref_pack_dims(self._p, ctypes.byref(d1n))
        d2 = np.zeros(d2n)
        d1 = np.zeros(d1n.value)
        if self._lib.v2b_ref_pack_spatial(self._p, np.ascontiguousarray(x, np.float64), d2, d1):
            raise RuntimeError(self._lib.v2b_ref_last_error().decode())
        return d2, d1

    # PSIO units and entries of hilbert's RDM writers (misc/hilbert_psifiles.h:33-42)
    RDM_UNITS = {"D2aa": 270, "D2ab": 271, "D2bb": 272, "D1a": 277, "D1b": 278, "D2": 279,
                 "D3aaa": 273, "D3aab": 274, "D3bba": 275, "D3bbb": 276}
    TPDM = np.dtype([("i", np.int32), ("j", np.int32), ("k", np.int32), ("l", np.int32),
                     ("value", np.float64)])
    OPDM = np.dtype([("i", np.int32), ("j", np.int32), ("value", np.float64)])
    DM3 = np.dtype([("i", np.int32), ("j", np.int32), ("k", np.int32), ("l", np.int32),
                    ("m", np.int32), ("n", np.int32), ("value", np.float64)])

    def write_rdms(self, x, ncore=0):
        """Runs the reference's WriteTPDM, WriteTPDMSpinFree, WriteOPDM and
        WriteTPDM_IWL on x, with ncore restricted doubly occupied orbitals
        numbered first, and returns what the PSIO writers wrote: {file:
        records} and {file: {entry: bytes}} (iwl_records has the rest)"""
        lib = self._lib
        lib.v2b_ref_write_rdms.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int]
        lib.v2b_ref_psio_entry.restype = ctypes.c_long
        lib.v2b_ref_psio_entry.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p]
        if lib.v2b_ref_write_rdms(self._p, np.ascontiguousarray(x, np.float64), int(ncore)):
            raise RuntimeError(lib.v2b_ref_last_error().decode())
        records, entries = {}, {}
        for name, unit in self.RDM_UNITS.items():
            entries[name] = {}
            for key in (name, "length", "NUMBER ACTIVE ORBITALS", "ACTIVE ORBITALS",
                        "NUMBER INACTIVE ORBITALS", "INACTIVE ORBITALS"):
                size = lib.v2b_ref_psio_entry(unit, key.encode(), None)
                if size < 0:
                    continue
                buf = ctypes.create_string_buffer(max(size, 1))
                lib.v2b_ref_psio_entry(unit, key.encode(), buf)
                entries[name][key] = buf.raw[:size]
            if not entries[name]:   # a file this problem's writers do not write
                del entries[name]
                continue
            raw = entries[name].get(name, b"")
            dt = self.TPDM if name.startswith("D2") else self.DM3 if name.startswith("D3") else self.OPDM
            records[name] = np.frombuffer(raw, dt).copy()
        return records, entries

    def iwl_records(self):
        """After write_rdms: the reference IWL writer's write_value calls per
        file, {"D2aa", "D2ab", "D2bb"}: (labels (n, 4), values (n,)), and the
        files' cutoff."""
        lib = self._lib
        lib.v2b_ref_iwl_records.restype = ctypes.c_long
        lib.v2b_ref_iwl_records.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p]
        out, cutoff = {}, ctypes.c_double()
        for name, spin in (("D2aa", b"aa"), ("D2ab", b"ab"), ("D2bb", b"bb")):
            count = lib.v2b_ref_iwl_records(spin, None, None)
            buf = np.zeros((max(count, 0), 5))
            lib.v2b_ref_iwl_records(spin, buf.ctypes.data, ctypes.byref(cutoff))
            out[name] = (buf[:, :4].astype(np.int64), buf[:, 4].copy())
        return out, cutoff.value

    def ATu(self, y):
        out = np.zeros(self.n_primal)
        if self._lib.v2b_ref_ATu(self._p, out, np.ascontiguousarray(y, np.float64)):
            raise RuntimeError(self._lib.v2b_ref_last_error().decode())
        return out

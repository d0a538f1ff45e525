"""ORACLE -- test infrastructure only.

ctypes binding of focas's C++ orbital optimizer compiled from the reference
sources (oracle/_ref/libfocas_ref.so, built by oracle/build_ref.sh with the
harness oracle/focas_harness.cc): the DF orbital step v2RDM-CASSCF runs
(OrbitalOptimizer::optimize_orbitals, src/focas/C_files/orbopt_optimize.cc:
25-98) and the gradient / diagonal Hessian it starts from (Compute_EGH).

Inputs are in the layouts hilbert hands to focas (v2rdm_solver.cc:3257):
d2 and d1 from PackSpatialDensity (active orbitals), the three-index
integrals Q-major over the packed lower triangle of all orbitals
(tei.cc:281-283), the one-electron integrals as a packed lower triangle, and
the transformation matrix (the identity on the first call), C1 orbitals
numbered core, active, virtual.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_ref", "libfocas_ref.so")
_lib = None


def available():
    return os.path.exists(SO)


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(SO)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.v2b_focas_create.restype = ctypes.c_void_p
        lib.v2b_focas_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        lib.v2b_focas_destroy.argtypes = [ctypes.c_void_p]
        lib.v2b_focas_nrot.restype = ctypes.c_int
        lib.v2b_focas_nrot.argtypes = [ctypes.c_void_p, dp, dp, dp, dp]
        lib.v2b_focas_egh.restype = ctypes.c_double
        lib.v2b_focas_egh.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp, dp, dp, dp]
        lib.v2b_focas_optimize.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp, dp, dp,
                                           ctypes.POINTER(ctypes.c_int)]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def pack_lower(m):
    """lower triangle of a symmetric matrix, INDEX(i, j) = i (i + 1) / 2 + j, i >= j"""
    i, j = np.tril_indices(m.shape[0])
    return np.ascontiguousarray(m[i, j])


def pack_df(B):
    """(naux, n, n) factors, Q-major over the packed lower triangle"""
    i, j = np.tril_indices(B.shape[1])
    return np.ascontiguousarray(B[:, i, j].reshape(-1))


class Focas:
    """One compiled focas optimizer for C1 orbitals (ncore, nact, nvirt)."""

    def __init__(self, ncore, nact, nvirt, naux, active_active=False, exact_diagonal_hessian=True,
                 maxiter=10, g_conv=1e-4, e_conv=1e-8):
        lib = _load()
        self._lib = lib
        self.nmo = ncore + nact + nvirt
        self._h = lib.v2b_focas_create(ncore, nact, nvirt, naux, int(active_active),
                                       int(exact_diagonal_hessian), maxiter, g_conv, e_conv)

    def __del__(self):
        try:
            self._lib.v2b_focas_destroy(self._h)
        except Exception:
            pass

    def _inputs(self, h, B, d2p, d1p):
        return (np.array(d2p, dtype=np.float64), np.array(d1p, dtype=np.float64), pack_df(np.asarray(B)),
                pack_lower(np.asarray(h)), np.eye(self.nmo))

    def gradient_hessian(self, h, B, d2p, d1p):
        """(E, gradient over focas's rotation pairs, diagonal Hessian, |g|) at the given orbitals"""
        d2, d1, tei, oei, U = self._inputs(h, B, d2p, d1p)
        nrot = self._lib.v2b_focas_nrot(self._h, _p(d2), _p(d1), _p(oei), _p(U))
        g = np.zeros(nrot)
        hd = np.zeros(nrot)
        gn = ctypes.c_double()
        E = self._lib.v2b_focas_egh(self._h, _p(d2), _p(d1), _p(tei), _p(oei), _p(U), _p(g), _p(hd),
                                    ctypes.byref(gn))
        return E, g, hd, gn.value

    def optimize(self, h, B, d2p, d1p):
        """One call of optimize_orbitals: (transformation matrix, dE, |g|, iterations)"""
        d2, d1, tei, oei, U = self._inputs(h, B, d2p, d1p)
        dE, gn, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._lib.v2b_focas_optimize(self._h, _p(d2), _p(d1), _p(tei), _p(oei), _p(U), ctypes.byref(dE),
                                     ctypes.byref(gn), ctypes.byref(it))
        return U, dE.value, gn.value, it.value

"""ctypes binding of the in-tree C-ABI library (include/v2rdm_b200.h).

The product path has no fallback: if the compiled library is missing or no
CUDA device is visible, loading or calling it raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libv2rdm_b200.so")

V2B_OK = 0
V2B_NOT_CONVERGED = 1
V2B_BAD_ARG = 2
V2B_NAN = 3
V2B_DEVICE_TIMEOUT = 4
V2B_CUDA_ERROR = 5
V2B_NO_DEVICE = 6
V2B_INTERNAL = 7

STATUS_NAMES = {0: "OK", 1: "NOT_CONVERGED", 2: "BAD_ARG", 3: "NAN", 4: "DEVICE_TIMEOUT",
                5: "CUDA_ERROR", 6: "NO_DEVICE", 7: "INTERNAL"}

POSITIVITY = {"D": 0, "DQ": 1, "DG": 2, "DQG": 3, "DQGT2": 4, "DQGT1": 5, "DQGT1T2": 6, "DQGT": 6}
V2B_CONSTRAIN_D3 = 16   # OR-ed into a POSITIVITY value
V2B_CONSTRAIN_Q3 = 32   # (implies D3)
V2B_CONSTRAIN_E3 = 64   # (implies D3)
V2B_CONSTRAIN_F3 = 128  # (implies D3)
V2B_CONSTRAIN_D4 = 256  # (implies D3)

#: every symbol declared in include/v2rdm_b200.h
EXPORTS = (
    "v2b_last_error", "v2b_version",
    "v2b_bpsdp_create", "v2b_bpsdp_solve", "v2b_bpsdp_is_converged", "v2b_bpsdp_get_mu",
    "v2b_bpsdp_set_mu", "v2b_bpsdp_get_y", "v2b_bpsdp_get_z", "v2b_bpsdp_set_y",
    "v2b_bpsdp_set_z", "v2b_bpsdp_iiter_total", "v2b_bpsdp_oiter_total", "v2b_bpsdp_destroy",
    "v2b_problem_create", "v2b_doci_problem_create", "v2b_problem_destroy", "v2b_problem_n_primal", "v2b_problem_n_dual",
    "v2b_problem_n_blocks", "v2b_problem_block_dims", "v2b_problem_build_b",
    "v2b_problem_build_c_hubbard", "v2b_problem_build_c_external", "v2b_problem_guess",
    "v2b_problem_Au", "v2b_problem_ATu", "v2b_problem_project", "v2b_problem_project_warm",
    "v2b_problem_solve",
    "v2b_problem_solve_device", "v2b_problem_get_y", "v2b_problem_get_z", "v2b_problem_get_mu",
    "v2b_problem_kernel_launches", "v2b_problem_operator_size", "v2b_problem_operator",
    "v2b_problem_set_profiling", "v2b_problem_profile", "v2b_problem_stream",
    "v2b_problem_projection_counts", "v2b_problem_refine_counts", "v2b_problem_set_projection_mode", "v2b_problem_set_gemm_split", "v2b_problem_gemm_split_choice", "v2b_problem_pack_dims", "v2b_problem_projection_profile",
    "v2b_problem_cg_profile",
    "v2b_problem_pack_spatial_density", "v2b_project_block_noalloc",
    "v2b_problem_rdm_counts", "v2b_problem_rdm_records", "v2b_problem_set_state", "v2b_problem_continue",
    "v2b_problem_set_wait_limit", "v2b_df_transform", "v2b_df_transform_adjoint",
    "v2b_doci_v2rdm_layout", "v2b_batch_problem_create", "v2b_problem_palette",
    "v2b_problem_tpdm_iwl_records", "v2b_problem_d3_counts", "v2b_problem_d3_records",
)


class V2BError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class SDPOptions(ctypes.Structure):
    """libsdp::SDPOptions as hilbert sets it (v2rdm_solver.cc:426-431)."""
    _fields_ = [("sdp_objective_convergence", ctypes.c_double),
                ("sdp_error_convergence", ctypes.c_double),
                ("cg_convergence", ctypes.c_double),
                ("cg_maxiter", ctypes.c_int),
                ("maxiter", ctypes.c_int)]


SDP_CALLBACK = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)
SDP_MONITOR = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_void_p)

_lib = None


def load(path=LIB_PATH):
    """Load the library (built by hilbert_b200.build); raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is not built; run `python -m hilbert_b200.build` "
                          "(there is no CPU fallback for the B200 path)")
    lib = ctypes.CDLL(path)
    vp, dp, ip, lp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), \
        ctypes.POINTER(ctypes.c_long)
    sig = {
        "v2b_last_error": (ctypes.c_char_p, []),
        "v2b_version": (ctypes.c_int, []),
        "v2b_bpsdp_create": (ctypes.c_int, [ctypes.c_long, ctypes.c_long, ctypes.POINTER(SDPOptions),
                                            ctypes.POINTER(vp)]),
        "v2b_bpsdp_solve": (ctypes.c_int, [vp, dp, dp, dp, ip, ctypes.c_int, ctypes.c_int,
                                           SDP_CALLBACK, SDP_CALLBACK, SDP_MONITOR, ctypes.c_int, vp]),
        "v2b_bpsdp_is_converged": (ctypes.c_int, [vp]),
        "v2b_bpsdp_get_mu": (ctypes.c_double, [vp]),
        "v2b_bpsdp_set_mu": (ctypes.c_int, [vp, ctypes.c_double]),
        "v2b_bpsdp_get_y": (ctypes.c_int, [vp, dp]),
        "v2b_bpsdp_get_z": (ctypes.c_int, [vp, dp]),
        "v2b_bpsdp_set_y": (ctypes.c_int, [vp, dp]),
        "v2b_bpsdp_set_z": (ctypes.c_int, [vp, dp]),
        "v2b_bpsdp_iiter_total": (ctypes.c_long, [vp]),
        "v2b_bpsdp_oiter_total": (ctypes.c_long, [vp]),
        "v2b_bpsdp_destroy": (None, [vp]),
        "v2b_problem_create": (ctypes.c_int, [ctypes.c_int] * 7 + [ctypes.POINTER(vp)]),
        "v2b_doci_problem_create": (ctypes.c_int, [ctypes.c_int] * 4 + [ctypes.POINTER(vp)]),
        "v2b_problem_destroy": (None, [vp]),
        "v2b_problem_n_primal": (ctypes.c_long, [vp]),
        "v2b_problem_n_dual": (ctypes.c_long, [vp]),
        "v2b_problem_n_blocks": (ctypes.c_int, [vp]),
        "v2b_problem_block_dims": (ctypes.c_int, [vp, ip]),
        "v2b_problem_build_b": (ctypes.c_int, [vp, dp]),
        "v2b_problem_build_c_hubbard": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_double, dp]),
        "v2b_problem_build_c_external": (ctypes.c_int, [vp, dp, dp, dp]),
        "v2b_problem_guess": (ctypes.c_int, [vp, ctypes.c_int, dp]),
        "v2b_problem_Au": (ctypes.c_int, [vp, vp, vp, vp]),
        "v2b_problem_ATu": (ctypes.c_int, [vp, vp, vp, vp]),
        "v2b_problem_project": (ctypes.c_int, [vp, vp, ctypes.c_double, vp, vp, vp]),
        "v2b_problem_project_warm": (ctypes.c_int, [vp, vp, ctypes.c_double, vp, vp, vp]),
        "v2b_problem_solve": (ctypes.c_int, [vp, dp, dp, dp, ctypes.POINTER(SDPOptions), ctypes.c_int,
                                             SDP_MONITOR, ctypes.c_int, vp, lp, lp, dp]),
        "v2b_problem_solve_device": (ctypes.c_int, [vp, vp, vp, vp, ctypes.POINTER(SDPOptions),
                                                    ctypes.c_int, SDP_MONITOR, ctypes.c_int, vp, lp,
                                                    lp, dp]),
        "v2b_problem_get_y": (ctypes.c_int, [vp, dp]),
        "v2b_problem_get_z": (ctypes.c_int, [vp, dp]),
        "v2b_problem_get_mu": (ctypes.c_double, [vp]),
        "v2b_problem_kernel_launches": (ctypes.c_long, [vp]),
        "v2b_problem_set_profiling": (ctypes.c_int, [vp, ctypes.c_int]),
        "v2b_problem_profile": (ctypes.c_int, [vp, dp, lp]),
        "v2b_problem_stream": (ctypes.c_void_p, [vp]),
        "v2b_problem_projection_counts": (ctypes.c_int, [vp, lp, lp, lp]),
        "v2b_problem_refine_counts": (ctypes.c_int, [vp, lp, ctypes.c_int]),
        "v2b_problem_set_projection_mode": (ctypes.c_int, [vp, ctypes.c_int]),
        "v2b_problem_set_gemm_split": (ctypes.c_int, [vp, ctypes.c_int]),
        "v2b_problem_gemm_split_choice": (ctypes.c_int, [vp, ip, ip]),
        "v2b_problem_pack_dims": (ctypes.c_int, [vp, lp, lp]),
        "v2b_problem_rdm_counts": (ctypes.c_int, [vp, ctypes.c_int, vp]),
        "v2b_problem_set_state": (ctypes.c_int, [vp, ctypes.c_double, dp, dp]),
        "v2b_problem_continue": (ctypes.c_int, [vp]),
        "v2b_problem_set_wait_limit": (ctypes.c_int, [vp, ctypes.c_longlong]),
        "v2b_df_transform": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, ctypes.c_int, vp]),
        "v2b_df_transform_adjoint": (ctypes.c_int, [vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp]),
        "v2b_doci_v2rdm_layout": (ctypes.c_int, [vp, vp, vp, lp]),
        "v2b_batch_problem_create": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(vp)]),
        "v2b_problem_palette": (ctypes.c_int, [vp, ctypes.c_int, vp, ip]),
        "v2b_problem_tpdm_iwl_records": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp, vp]),
        "v2b_problem_d3_counts": (ctypes.c_int, [vp, vp]),
        "v2b_problem_d3_records": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp, vp, vp]),
        "v2b_problem_rdm_records": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp]),
        "v2b_problem_projection_profile": (ctypes.c_int, [vp, dp, lp, ctypes.c_int]),
        "v2b_problem_cg_profile": (ctypes.c_int, [vp, dp, ctypes.c_int]),
        "v2b_problem_pack_spatial_density": (ctypes.c_int, [vp, vp, vp, vp, vp]),
        "v2b_project_block_noalloc": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, vp, vp, vp]),
        "v2b_problem_operator_size": (ctypes.c_int, [vp, ctypes.c_int, lp, lp, ip]),
        "v2b_problem_operator": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_uint32),
                                                ctypes.POINTER(ctypes.c_uint32), dp]),
    }
    for name in EXPORTS:
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = sig[name]
    _lib = lib
    return lib


def check(code, allow=(V2B_OK,)):
    if code not in allow:
        msg = _lib.v2b_last_error().decode() if _lib is not None else ""
        raise V2BError(code, msg)
    return code

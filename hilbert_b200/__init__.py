"""hilbert_b200 -- B200-native boundary-point SDP path for hilbert's v2RDM-CASSCF.

The compute path is the C-ABI library ``_lib/libv2rdm_b200.so`` (CUDA kernels
for sm_100a, C++ host orchestration; entry points in include/v2rdm_b200.h).
This package mirrors hilbert's Python-facing interface on top of it.
"""
from ._capi import LIB_PATH, V2BError, load  # noqa: F401
from .v2rdm import (BatchProblem, BPSDPSolver, DOCIProblem, Options, V2RDMProblem, block_layout,  # noqa: F401
                    block_offsets, v2RDM_DOCIHelper, v2RDMHelper)

__all__ = ["BatchProblem", "BPSDPSolver", "DOCIProblem", "Options", "V2RDMProblem", "v2RDMHelper", "v2RDM_DOCIHelper", "block_layout",
           "block_offsets", "load", "LIB_PATH", "V2BError"]

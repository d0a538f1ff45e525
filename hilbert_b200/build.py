"""Build the in-tree C-ABI library hilbert_b200/_lib/libv2rdm_b200.so for sm_100a.

The library has no Python or torch dependency: it is a plain shared object
with the entry points declared in include/v2rdm_b200.h.  Python reaches it
through ctypes (hilbert_b200/_capi.py); a C or C++ host links it directly.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libv2rdm_b200.so")
SOURCES = ["v2rdm_problem.cpp", "doci_problem.cpp", "rdm_records.cpp", "batch_problem.cpp", "v2b_kernels.cu", "v2b_eig.cu", "v2b_bigjacobi.cu", "v2b_refine.cu",
           "v2b_orbital.cu", "v2b_transform.cu", "v2b_solver.cu", "v2b_noalloc.cu"]
HEADERS = ["v2rdm_problem.h", "doci_problem.h", "rdm_records.h", "v2b_kernels.cuh", "v2b_device.cuh", "v2b_eig.cuh", "v2b_bigjacobi.cuh",
           "v2b_refine.cuh", "v2b_orbital.cuh", "v2b_transform.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "v2rdm_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    nvcc = nvcc_path()
    common = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc] + ARCH + common + ["-Xptxas", "-v" if verbose else "-O3", "-c",
                                        os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-rdc=false"]
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

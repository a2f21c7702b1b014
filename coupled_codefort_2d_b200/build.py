"""Build the in-tree CUDA library ``libfugu_gpu.so`` for sm_100a.

Run as ``python -m coupled_codefort_2d_b200.build`` (or through
``__graft_entry__.build()``).  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfugu_gpu.so")
SOURCES = ["fugu_gpu.cu"]
HEADERS = ["fugu_internal.cuh", "kernels.cuh", "persistent.cuh", "pcg_cluster.cuh", "scalars.cuh", "fgmres.cuh", "adjoint.cuh",
           "dual.cuh", "step_vjp.cuh", "lockstep.cuh", "lockstep_host.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # FP64 plain form: no contraction, so each a*b+c rounds twice as the
    # reference (and the CPU oracle) does.
    "--fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "fugu_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


DRIVER = os.path.join(HERE, "fugu2d")
DRIVER_SRC = os.path.join(CSRC, "fugu2d_main.cpp")


def build_driver(verbose: bool = False) -> str:
    """The fugu2d driver (input.nml -> time loop) linked against the library."""
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), DRIVER_SRC, "-o", DRIVER,
           "-L", HERE, "-lfugu_gpu", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return DRIVER


ROWBENCH = os.path.join(HERE, "rowbench")
ROWBENCH_SRC = os.path.join(CSRC, "rowbench.cu")


def build_rowbench(verbose: bool = False) -> str:
    """The row-kernel timing program (csrc/rowbench.cu): the same kernels and
    flags as the library, as a stand-alone executable."""
    nvcc = os.environ.get("NVCC", "nvcc")
    flags = [f for f in NVCC_FLAGS if f not in ("-shared", "-Xcompiler", "-fPIC")]
    cmd = [nvcc, *flags, "-I", os.path.join(ROOT, "include"), ROWBENCH_SRC, "-o", ROWBENCH]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return ROWBENCH


def build(force: bool = False, verbose: bool = False) -> str:
    if force or _stale():
        nvcc = os.environ.get("NVCC", "nvcc")
        cmd = [nvcc, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-o", LIB]
        cmd += [os.path.join(CSRC, f) for f in SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(DRIVER) or os.path.getmtime(DRIVER) < max(os.path.getmtime(LIB),
                                                                             os.path.getmtime(DRIVER_SRC)):
        build_driver(verbose)
    return LIB


if __name__ == "__main__":
    if "--rowbench" in sys.argv:
        print(build_rowbench(verbose=True))
    else:
        print(build(force="--force" in sys.argv, verbose=True))

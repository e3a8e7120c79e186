"""Build libheat_b200.so and the heat_solver_b200 CLI in-tree for sm_100a.

The library is compiled with ``--fmad=false`` (every fused multiply-add in the
kernels is an explicit ``__fma_rn``) and host code with
``-ffp-contract=off``, so the deterministic path is a fixed function of its
inputs on any build machine.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libheat_b200.so")
CLI = os.path.join(HERE, "heat_solver_b200")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["hs_solver.cu", "hs_setup.cpp", "hs_cli.cpp"]
HEADERS = ["hs_kernels.cuh", "hs_types.h", "hs_host.h", "hs_cli.h", "hs_noalloc.cu", "hs_campaign.cu", "hs_batch.cu", "hs_batch_kernels.cuh", "hs_csum.h", "hs_field.cu"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _host_compiler() -> list:
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def _stale(target: str, deps: list) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the shared library and the CLI; returns the library path."""
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "heat_b200.h"))
    deps.append(os.path.abspath(__file__))
    nvcc = _nvcc()
    common = ARCH + _host_compiler() + [
        "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
        "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    ]
    if force or _stale(LIB, deps):
        cmd = [nvcc] + common + ["-shared", "-o", LIB] + [os.path.join(CSRC, f) for f in SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
    cli_src = os.path.join(CSRC, "heat_solver_b200.cpp")
    if force or _stale(CLI, [LIB, cli_src]):
        cmd = [nvcc] + ARCH + _host_compiler() + ["-O2", "-std=c++17", "-o", CLI, cli_src, "-L" + HERE,
                                                  "-lheat_b200", "-Xlinker", "-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

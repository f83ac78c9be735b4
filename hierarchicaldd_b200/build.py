"""Builds the CUDA library libhdd_b200.so in-tree for sm_100a, and the
hdd_test_bench command line (the reference's Test_Bench_3D flags) linked to it.

Usage: python -m hierarchicaldd_b200.build  (or build() from Python).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libhdd_b200.so")
# The reference's Test_Bench_3D command line over the C ABI.
CLI = os.path.join(HERE, "hdd_test_bench")
BUILD = os.path.join(HERE, "_build")

SOURCES = [
    "host_setup.cpp",
    "host_interface.cpp",
    "host_cholesky.cpp",
    "host_interface_io.cpp",
    "capi.cpp",
    "server.cpp",
    "kernels_vcycle.cu",
    "kernels_vcycle_global.cu",
    "kernels_pcg.cu",
    "sigma.cu",
    "sn_plan.cpp",
    "sn_solve.cu",
    "solver.cu",
    "noalloc.cu",
    "velocity.cu",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # A host compiler whose OpenMP runtime is installed.
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc, cxx = _nvcc(), _host_cxx()
    common = ["-std=c++17", "-O3", "-ccbin", cxx, "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off"]
    objs = []
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "hdd.h"))
    newest_header = max(os.path.getmtime(h) for h in headers)
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
                and os.path.getmtime(obj) >= newest_header):
            continue
        cmd = [nvcc] + common + ARCH + ["-lineinfo", "-c", path, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-O3"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [nvcc] + ARCH + ["-shared", "-ccbin", cxx, "-o", OUT] + objs + ["-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    cli_src = os.path.join(CSRC, "test_bench_main.cpp")
    if force or not os.path.exists(CLI) or any(os.path.getmtime(f) > os.path.getmtime(CLI)
                                               for f in (cli_src, OUT)):
        cmd = [cxx, "-std=c++17", "-O2", "-fopenmp", "-I", os.path.join(os.path.dirname(HERE), "include"),
               cli_src, "-o", CLI, "-L", HERE, "-l:libhdd_b200.so", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(OUT)

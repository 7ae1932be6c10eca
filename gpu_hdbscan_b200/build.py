"""Builds libhdb_b200.so (all CUDA sources, sm_100a only) and the hdbscan_ CLI.

Usage: python -m gpu_hdbscan_b200.build   (or __graft_entry__.build()).
The shared library is written next to this file so it travels with the
source tree; nothing is installed.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libhdb_b200.so")
CLI = os.path.join(HERE, "hdbscan_")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-I", os.path.join(ROOT, "include")]


def _sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = _sources()
    deps = srcs + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [
        os.path.join(ROOT, "include", "hdb", "hdb.h")]
    if force or _stale(LIB, deps):
        cmd = [NVCC, *ARCH, *FLAGS, "-shared", "-o", LIB, *srcs, "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    cli_src = os.path.join(HERE, "cli", "hdbscan_main.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB])):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
               "-I", "/usr/local/cuda/include", "-o", CLI, cli_src, "-L", HERE, "-lhdb_b200",
               "-Wl,-rpath,$ORIGIN", "-L/usr/local/cuda/lib64", "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

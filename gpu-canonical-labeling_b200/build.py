"""Build the native parts of the package in-tree.

* ``libgcl_b200.so`` -- the CUDA kernels and the C ABI (include/gcl.h), built
  for sm_100a only.
* ``bin/gpu_canon_label`` -- the command-line front-end (same usage as the
  reference's ``gpu_canon_label``), linked against ``libgcl_b200.so``.

Usage: ``python gpu-canonical-labeling_b200/build.py [--force]``.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libgcl_b200.so")
CLI_SRC = os.path.join(PKG, "cli", "gpu_canon_label.cpp")
CLI_BIN = os.path.join(PKG, "bin", "gpu_canon_label")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr"]
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cuh", ".h", ".cpp")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force: bool = False, verbose: bool = False) -> str:
    deps = _sources() + [os.path.join(ROOT, "include", "gcl.h")]
    if force or _stale(LIB, deps):
        units = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
        cmd = [NVCC, *ARCH, *NVCC_FLAGS, "-ccbin", HOST_CXX, "-shared", "-o", LIB, *units]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    return LIB


def build_cli(force: bool = False) -> str:
    if not os.path.exists(CLI_SRC):
        return ""
    deps = [CLI_SRC, LIB, os.path.join(ROOT, "include", "gcl.h"), os.path.join(CSRC, "gcl_dimacs.h"),
            os.path.join(CSRC, "gcl_format.h")]
    if force or _stale(CLI_BIN, deps):
        os.makedirs(os.path.dirname(CLI_BIN), exist_ok=True)
        cmd = [HOST_CXX, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), CLI_SRC,
               "-o", CLI_BIN, "-L", PKG, "-lgcl_b200", "-Wl,-rpath,$ORIGIN/..",
               ]
        subprocess.run(cmd, check=True)
    return CLI_BIN


def build(force: bool = False, verbose: bool = False) -> None:
    build_lib(force, verbose)
    build_cli(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)

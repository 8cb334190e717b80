"""Build the sm_100a shared library ql_dns_b200/_lib/libqlgpu.so in-tree.

Usage: python -m ql_dns_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libqlgpu.so")
MAIN = os.path.join(OUT_DIR, "ql_main")

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def sources():
    return [os.path.join(CSRC, "qlgpu.cu")]


def deps():
    return (glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(CSRC, "examples", "*")) +
            glob.glob(os.path.join(ROOT, "include", "*")))


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in deps())


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and not stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + (extra or []) + ["-I" + os.path.join(ROOT, "include"), "-o", LIB + ".tmp"] + sources()
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    build_main(verbose)
    return LIB


def build_main(verbose: bool = False) -> str:
    """The C++ driver (csrc/examples/ql_main.cpp) linked against libqlgpu.so."""
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    src = os.path.join(CSRC, "examples", "ql_main.cpp")
    cmd = [cxx, "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), src, "-o", MAIN,
           "-L" + OUT_DIR, "-lqlgpu", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return MAIN


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    build(force=a.force or a.ptxas_v, verbose=a.verbose, extra=(["-Xptxas", "-v"] if a.ptxas_v else None))
    print(LIB)
    sys.exit(0)

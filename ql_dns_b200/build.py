"""Build the sm_100a shared library ql_dns_b200/_lib/libqlgpu.so in-tree.

Usage: python -m ql_dns_b200.build [--force] [--verbose] [--debug]

--debug builds ql_dns_b200/_lib/libqlgpu_debug.so with -DQLGPU_DEBUG: device
bounds checks on the index math of every kernel family (a failed check sets a
status bit and the access is redirected in bounds, no trap) and canary-guarded
device buffers checked after every launch.  QLGPU_DEBUG=1 in the environment
makes the Python binding load it.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libqlgpu.so")
DEBUG_LIB = os.path.join(OUT_DIR, "libqlgpu_debug.so")
MAIN = os.path.join(OUT_DIR, "ql_main")

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]
OBJ_DIR = os.path.join(OUT_DIR, "obj")
DEBUG_OBJ_DIR = os.path.join(OUT_DIR, "obj_debug")


def sources():
    """Translation units of libqlgpu.so: the host code and one file per kernel family, compiled in parallel."""
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def deps():
    return (glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(CSRC, "examples", "*")) +
            glob.glob(os.path.join(ROOT, "include", "*")))


def stale(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(d) > t for d in deps())


def _headers_mtime() -> float:
    hs = [d for d in deps() if not d.endswith((".cu", ".cpp")) and os.path.isfile(d)]
    return max(os.path.getmtime(h) for h in hs) if hs else 0.0


def build(force: bool = False, verbose: bool = False, extra=None, jobs: int | None = None,
          debug: bool = False) -> str:
    lib = DEBUG_LIB if debug else LIB
    obj_dir = DEBUG_OBJ_DIR if debug else OBJ_DIR
    if not force and not stale(lib):
        return lib
    os.makedirs(obj_dir, exist_ok=True)
    flags = NVCC_FLAGS + (["-DQLGPU_DEBUG"] if debug else [])
    nvcc = os.environ.get("NVCC", "nvcc")
    hdr_t = _headers_mtime()
    inc = ["-I" + os.path.join(ROOT, "include")]

    def compile_one(src):
        obj = os.path.join(obj_dir, os.path.splitext(os.path.basename(src))[0] + ".o")
        if (not force and extra is None and os.path.exists(obj) and os.path.getmtime(obj) > os.path.getmtime(src)
                and os.path.getmtime(obj) > hdr_t):
            return obj
        cmd = [nvcc] + flags + (extra or []) + inc + ["-c", "-o", obj + ".tmp.o", src]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.stdout or r.stderr:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, cmd)
        os.replace(obj + ".tmp.o", obj)
        return obj

    # the kernel translation units are the slow ones: start them first
    srcs = sorted(sources(), key=lambda f: -os.path.getsize(f) if f.endswith(".cu") and
                  os.path.basename(f) != "qlgpu.cu" else 0)
    n = jobs or max(1, min(len(srcs), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(max_workers=n) as ex:
        objs = list(ex.map(compile_one, srcs))
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-o",
           lib + ".tmp"] + objs
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(lib + ".tmp", lib)
    if not debug:
        build_main(verbose)
    return lib


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
    ap.add_argument("--debug", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose, extra=(["-Xptxas", "-v"] if a.ptxas_v else None),
                debug=a.debug))
    sys.exit(0)

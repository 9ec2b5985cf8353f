"""In-tree build of the engine and its command-line drivers.

Compiles every CUDA source under ``csrc/`` for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) and the host sources with g++/OpenMP, then
links ``lib/libmapgraph_b200.so`` with the CUDA runtime linked statically. The
shared library is the product: Python, the C++ header shims and the CLI drivers
all reach the engine through its C ABI (``include/mapgraph_b200.h``).

Run ``python -m mirrorofmapgraph_b200._build`` or call :func:`build`.
Rebuilds only when a source or header is newer than the library.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
BINDIR = os.path.join(PKG, "bin")
OBJDIR = os.path.join(PKG, "_build")
LIB = os.path.join(LIBDIR, "libmapgraph_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fopenmp,-O3",
    "-I" + INCLUDE, "-I" + CSRC,
]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-I" + INCLUDE, "-I" + CSRC,
             "-I" + os.path.join(CUDA_HOME, "include")]


def _sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    return cu, cpp


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(INCLUDE, "*.h")))


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _obj(src):
    return os.path.join(OBJDIR, os.path.basename(src) + ".o")


def build_library(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    """Compiles and links lib/libmapgraph_b200.so when out of date; returns its path."""
    cu, cpp = _sources()
    hdr_time = _newest(_headers())
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    todo = []
    for src in cu + cpp:
        o = _obj(src)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(src), hdr_time):
            todo.append(src)

    def compile_one(src):
        o = _obj(src)
        if src.endswith(".cu"):
            cmd = [NVCC] + NVCC_FLAGS + ["-Xptxas", "-v", "-c", src, "-o", o] if verbose else \
                [NVCC] + NVCC_FLAGS + ["-c", src, "-o", o]
        else:
            cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", o]
        return _run(cmd, verbose)

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, len(todo))) as ex:
            for out in ex.map(compile_one, todo):
                if verbose and out.strip():
                    print(out)
    objs = [_obj(s) for s in cu + cpp]
    if force or todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        tmp = LIB + ".tmp"
        _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs +
             ["-cudart", "static", "-Xcompiler", "-fopenmp", "-lgomp"], verbose)
        os.replace(tmp, LIB)
    return LIB


def build_cli(force: bool = False, verbose: bool = False) -> list[str]:
    """Builds the BFS/SSSP/CC/PageRank command-line drivers against the library."""
    srcdir = os.path.join(CSRC, "cli")
    outs = []
    if not os.path.isdir(srcdir):
        return outs
    os.makedirs(BINDIR, exist_ok=True)
    common = sorted(glob.glob(os.path.join(srcdir, "common", "*.cpp")))
    deps = common + glob.glob(os.path.join(srcdir, "common", "*.h")) + _headers() + [LIB]
    for main in sorted(glob.glob(os.path.join(srcdir, "*.cpp"))):
        name = os.path.splitext(os.path.basename(main))[0]
        exe = os.path.join(BINDIR, name)
        if not force and os.path.exists(exe) and os.path.getmtime(exe) >= _newest(deps + [main]):
            outs.append(exe)
            continue
        _run(["g++", "-O2", "-std=c++17", "-I" + INCLUDE, "-I" + os.path.join(srcdir, "common"), main] + common +
             ["-o", exe, "-L" + LIBDIR, "-lmapgraph_b200", "-Wl,-rpath,$ORIGIN/../lib"], verbose)
        outs.append(exe)
    return outs


def build(force: bool = False, verbose: bool = False) -> str:
    lib = build_library(force=force, verbose=verbose)
    build_cli(force=force, verbose=verbose)
    return lib


def clean() -> None:
    for d in (OBJDIR, LIBDIR, BINDIR):
        shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    force = "--force" in sys.argv
    verbose = "-v" in sys.argv
    print(build(force=force, verbose=verbose))

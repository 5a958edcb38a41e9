"""Build recipe for libstkfmm_b200.so (sm_100a, in-tree).

Every CUDA / C++ source under stkfmm_b200/csrc is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and linked into
``stkfmm_b200/libstkfmm_b200.so`` with a static CUDA runtime; the far field's
dense translations and operator pseudo-inverses link cuBLAS and cuSOLVER from
the CUDA toolkit (an rpath points there).  Objects go to
``stkfmm_b200/_build`` and are rebuilt only when a source or header changed.

The host-only octree and list builder (stk_tree.cpp, stk_octree_capi.cpp) is
also built on its own, by the host C++ compiler and without CUDA, into
``stkfmm_b200/libstk_octree.so``: the tree C ABI (``stk_octree_*``) for
programs that have no GPU or must not map the GPU library.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libstkfmm_b200.so")
OCTREE_LIB = os.path.join(HERE, "libstk_octree.so")
OCTREE_SOURCES = ("stk_tree.cpp", "stk_octree_capi.cpp")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build stkfmm_b200")


def host_compiler() -> list:
    # the system g++ (the image's default $CXX wrapper is not usable as nvcc's host compiler)
    for cand in ("/usr/bin/g++",):
        if os.path.exists(cand):
            return ["-ccbin", cand]
    return []


def _cuda_libs() -> list:
    libdir = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc()))), "lib64")
    return ["-L" + libdir, "-Xlinker", "-rpath=" + libdir, "-lcublas", "-lcusolver"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.h*")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                  + glob.glob(os.path.join(INCLUDE, "*.h")))


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def _compile(src: str, obj: str, verbose: bool) -> None:
    cmd = [nvcc()] + host_compiler() + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s%s" % (os.path.basename(src), r.stdout, r.stderr))
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)


def build_octree(force: bool = False) -> str:
    """Compile (if needed) and return the path of the host-only libstk_octree.so."""
    srcs = [os.path.join(CSRC, f) for f in OCTREE_SOURCES]
    deps = srcs + [os.path.join(CSRC, "stk_tree.hpp"), os.path.join(INCLUDE, "stkfmm_b200.h")]
    if force or not os.path.exists(OCTREE_LIB) or os.path.getmtime(OCTREE_LIB) < _newest(deps):
        cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "c++")
        tmp = OCTREE_LIB + ".tmp"
        cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + INCLUDE, "-o", tmp] + srcs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("g++ failed on libstk_octree.so:\n%s%s" % (r.stdout, r.stderr))
        os.replace(tmp, OCTREE_LIB)
    return OCTREE_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile (if needed) and return the path of libstkfmm_b200.so (and build libstk_octree.so)."""
    build_octree(force)
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    hdr_time = _newest(_headers())
    objs = []
    todo = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_time):
            todo.append((s, o))
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            list(ex.map(lambda so: _compile(so[0], so[1], verbose), todo))
    if force or todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        tmp = LIB + ".tmp"
        cmd = ([nvcc()] + host_compiler() + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
               + _cuda_libs())
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc link failed:\n%s%s" % (r.stdout, r.stderr))
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

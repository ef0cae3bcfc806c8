"""Builds libmfree.so (the C-ABI library) in-tree for sm_100a, and its
bounds-checked debug build libmfree_checked.so (-DMFREE_BOUNDS_CHECK: indices
computed from data are tested and counted instead of faulting; the tests run
small cases through it as the stand-in for a memory checker).

CUDA sources are compiled by nvcc with ``-gencode arch=compute_100a,code=sm_100a``
(default IEEE division/square root: the cell hash must be bit-exact); host C++
sources by g++.  Usage: ``python -m iwf_mfree_gpu_3d_b200.build [--force]``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmfree.so")
LIB_CHECKED = os.path.join(PKG, "libmfree_checked.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["mfree_sort.cu", "mfree_interact.cu", "mfree_contact.cu", "mfree_host.cu", "mfree_batch.cu",
              "mfree_output.cu", "mfree_state.cu", "mfree_probe.cu", "mfree_static.cu"]
CPP_SOURCES = ["mfree_tool.cpp", "mfree_io.cpp"]


def _newer(out: str, deps) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hs + [os.path.join(INCLUDE, "mfree.h")]


def _compile(src: str, force: bool, verbose_ptxas: bool, checked: bool = False):
    name = os.path.basename(src)
    obj = os.path.join(BUILD, "checked" if checked else "", name + ".o")
    if not force and _newer(obj, [src] + _headers()):
        return obj, ""
    defs = ["-DMFREE_BOUNDS_CHECK"] if checked else []
    if src.endswith(".cu"):
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", *defs, "-I" + INCLUDE,
               "-I" + CSRC, "-c", src, "-o", obj]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", *defs, "-I" + INCLUDE, "-I" + CSRC,
               "-I" + os.path.join(CUDA_HOME, "include"), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose_ptxas: bool = False, checked: bool = False) -> str:
    """Compile and link libmfree.so (checked: libmfree_checked.so); returns its path."""
    lib = LIB_CHECKED if checked else LIB
    os.makedirs(os.path.join(BUILD, "checked") if checked else BUILD, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES + CPP_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose_ptxas, checked), srcs))
    objs = [o for o, _ in results]
    if verbose_ptxas:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    if force or not _newer(lib, objs):
        tmp = lib + ".tmp"
        cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        shutil.move(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv, checked="--checked" in sys.argv))

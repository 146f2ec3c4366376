"""Builds libnnkifmm.so in-tree (stokes-nnkifmm_b200/nnkifmm/libnnkifmm.so).

CUDA sources are compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); host sources with g++ and
``-ffp-contract=off`` so the tree midpoints and the nearest-neighbour
distances round like the reference's separate FP64 operations.

Usage: python stokes-nnkifmm_b200/build_lib.py [-j N] [--verbose]
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "nnkifmm")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libnnkifmm.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
            "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fopenmp", "-fmad=true"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
             f"-I{CUDA}/include"]


def sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def newer(src_files, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_files)


def run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(jobs=8, verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp = sources()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "nnkifmm.h"))
    objs, cmds = [], []
    for f in cu:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or newer([src] + headers, obj):
            cmds.append([NVCC, *ARCH, *CU_FLAGS, "-c", src, "-o", obj])
    for f in cpp:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or newer([src] + headers, obj):
            cmds.append(["g++", *CXX_FLAGS, "-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        list(ex.map(lambda c: run(c, verbose), cmds))
    if force or cmds or newer(objs, LIB):
        run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, f"-L{CUDA}/lib64", "-lcublas", "-lcusolver", "-lgomp",
             "-Xlinker", f"-rpath={CUDA}/lib64"], verbose)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.verbose, a.force))

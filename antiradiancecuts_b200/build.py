"""Build recipe for libarc.so: every CUDA source compiled for sm_100a with nvcc, the CPU scene
generator with g++, linked in-tree into antiradiancecuts_b200/libarc.so.

    python -m antiradiancecuts_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libarc.so")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp", f"-I{INCLUDE}", f"-I{CSRC}",
                     "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-fPIC", "-fopenmp", "-std=c++17", f"-I{INCLUDE}", f"-I{CSRC}"]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "arc_api.h"))
    return max(os.path.getmtime(h) for h in hs)


def _needs(obj: str, src: str, hdr_mtime: float) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return t < os.path.getmtime(src) or t < hdr_mtime


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return r


def build(force: bool = False, verbose: bool = False, extra_nvcc=()) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp = _sources()
    hdr = _headers_mtime()
    jobs = []
    objs = []
    for f in cu:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _needs(obj, src, hdr):
            # the GPU scene generator reproduces the CPU one bit for bit: no FMA contraction
            per_file = ["-fmad=false"] if f == "scene_gpu.cu" else []
            jobs.append([NVCC, *NVCC_FLAGS, *per_file, *extra_nvcc, "-c", src, "-o", obj])
    for f in cpp:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _needs(obj, src, hdr):
            jobs.append(["g++", *CXX_FLAGS, "-c", src, "-o", obj])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    if jobs or not os.path.exists(LIB):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fopenmp", "-lgomp"], verbose)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills per kernel")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_info else []
    print(build(force=a.force or a.ptxas_info, verbose=a.verbose or a.ptxas_info, extra_nvcc=extra))


if __name__ == "__main__":
    sys.exit(main())

"""Builds libfeatb200.so in-tree (feat3.doxytest_b200/featb200/libfeatb200.so) for sm_100a.

    python feat3.doxytest_b200/build.py [--force]

CUDA sources are compiled by nvcc for sm_100a only; the host set-up code by g++ without FP
contraction (the coarse-grid inverse must round like the reference's own C++).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OUT_DIR = os.path.join(HERE, "featb200")
LIB = os.path.join(OUT_DIR, "libfeatb200.so")
OBJ_DIR = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["fb_arch.cu", "fb_mg.cu", "fb_mrhs.cu", "fb_noalloc.cu", "fb_batch.cu", "fb_assemble.cu", "fb_unet.cu"]
CPP_SOURCES = ["fb_setup.cpp"]


def _sources():
    cu = [s for s in CU_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    cpp = [s for s in CPP_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    return cu, cpp


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, force):
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in os.listdir(CSRC)
                                         if h.endswith((".h", ".cuh"))] + [os.path.join(INCLUDE, "featb200.h")]
    if not force and not _stale(obj, deps):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC] + ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
                               "-I", INCLUDE, "-c", os.path.join(CSRC, src), "-o", obj]
    else:
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", INCLUDE, "-c",
               os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile of {src} failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force=False):
    os.makedirs(OBJ_DIR, exist_ok=True)
    cu, cpp = _sources()
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), cu + cpp))
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))

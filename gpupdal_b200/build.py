"""Builds the native library in-tree: gpupdal_b200/_lib/libnbg_b200.so.

    python -m gpupdal_b200.build [--verbose-ptxas]

Every CUDA source is compiled for sm_100a only (no PTX for other targets),
with the CUDA runtime linked statically so the library needs only the driver.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libnbg_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
              "-I", INCLUDE, "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-I", INCLUDE]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    return cmd, r


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    cu, cpp = sources()
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "nbg_b200.h")]
    newest_dep = max(os.path.getmtime(p) for p in deps)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest_dep:
        return LIB
    jobs = []
    objs = []
    for f in cu:
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", os.path.join(CSRC, f), "-o", obj]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        jobs.append(cmd)
    for f in cpp:
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        jobs.append([nvcc(), *ARCH, "-x", "cu", *NVCC_FLAGS, "-c", os.path.join(CSRC, f), "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for cmd, r in ex.map(_compile, jobs):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("compile failed: " + " ".join(cmd[-3:]))
            if verbose_ptxas:
                sys.stderr.write(r.stderr)
    tmp = LIB + ".tmp"
    link = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, "-lpthread"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose_ptxas, a.force))

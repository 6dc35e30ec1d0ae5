#!/usr/bin/env python3
"""Build libatsc3_fec.so (all CUDA kernels + the C ABI) for sm_100a, in tree.

    python atsc3_b200/csrc/build.py [--force]

Every translation unit is compiled with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` only, ``-fmad=false`` (the
parity kernels must round each float op separately), ``-lineinfo``; the
objects are linked into ``atsc3_b200/_lib/libatsc3_fec.so``.  Rebuilds only
when a source or header is newer than the library.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libatsc3_fec.so")
OBJDIR = os.path.join(PKG, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler",
         "-fPIC", "-Xcompiler", "-fvisibility=default", "--use_fast_math=false"]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def sources():
    return sorted(glob.glob(os.path.join(HERE, "*.cu")))


def deps():
    return (sources() + glob.glob(os.path.join(HERE, "*.cuh")) +
            glob.glob(os.path.join(HERE, "*.h")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in deps())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    cc = nvcc()
    flags = [f for f in FLAGS if f != "--use_fast_math=false"]

    def one(src):
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
        cmd = [cc] + ARCH + flags + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(one, sources()))
    tmp = LIB + ".tmp"
    cmd = [cc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

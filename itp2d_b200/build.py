"""Builds the sm_100a CUDA library libitp2d_b200.so in-tree with nvcc.

    python -m itp2d_b200.build            # incremental
    python -m itp2d_b200.build --force    # rebuild everything
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libitp2d_b200.so")

SOURCES = ["split.cu", "contract.cu", "jacobi.cu", "ctx.cu", "probe.cu", "noalloc.cu", "bjacobi.cu", "tc.cu", "rfft.cu", "bjacobi32.cu", "potential.cu", "lowdin.cu", "batch.cu", "cholesky.cu", "oz.cu"]
HOST_SOURCES = [os.path.join("host", "itp2d_host.cpp"), os.path.join("host", "itp2d_serve.cpp"),
                os.path.join("host", "itp2d_datafile.cpp")]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-I", os.path.join(ROOT, "include")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")]:
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps(src: str) -> list:
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(ROOT, "include", "itp2d_gpu.h"), src]


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    objs = []
    procs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s.replace(".cu", ".o"))
        objs.append(obj)
        stale = force or not os.path.exists(obj) or \
            max(os.path.getmtime(d) for d in _deps(src)) > os.path.getmtime(obj)
        if stale:
            cmd = [nvcc(), *ARCH, *FLAGS, "-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for h in HOST_SOURCES:
        src = os.path.join(HERE, h)
        obj = os.path.join(OBJ, os.path.basename(h).replace(".cpp", ".o"))
        objs.append(obj)
        deps = [src, os.path.join(HERE, "host", "itp2d_host.hpp"), os.path.join(ROOT, "include", "itp2d_gpu.h"),
                os.path.join(ROOT, "include", "itp2d_host.h"), os.path.join(ROOT, "include", "itp2d_datafile.h")]
        if force or not os.path.exists(obj) or max(os.path.getmtime(d) for d in deps) > os.path.getmtime(obj):
            cmd = ["g++", *CXX_FLAGS, "-c", src, "-o", obj]
            procs.append((h, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for s, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out)
            raise RuntimeError(f"nvcc failed on {s}")
        if verbose and out:
            sys.stderr.write(out)
    relink = force or procs or not os.path.exists(LIB) or \
        max(os.path.getmtime(o) for o in objs) > os.path.getmtime(LIB)
    if relink:
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-lpthread", "-ldl", "-lz"]
        # the host objects are plain g++ output; nvcc links them with the device code
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))

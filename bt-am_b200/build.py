"""Build step of the package: compiles libbtam.so for sm_100a with nvcc.

Usage: python bt-am_b200/build.py   (or __graft_entry__.build()).
The shared library lands in bt-am_b200/lib/ inside the tree, next to the
Python bindings that load it.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libbtam.so")
SOURCES = ["btam_capi.cu", "adp_kernels.cu", "topo_kernels.cu", "solvers.cu", "batch.cu",
           "server.cu", "noalloc.cu", "point.cu", "mf_hessian.cu", "multipole.cu"]
# multipole.cu restates the finite-difference Hessians of the multipole
# rule, whose 1/(12 dr^2) amplifies the last bit of every term: no FMA
# contraction there, so each operation rounds as the reference's does.
EXTRA = {"multipole.cu": ["--fmad=false"]}
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
         "-ffp-contract=off"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    os.makedirs(LIB_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "btam.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    objs = [os.path.join(LIB_DIR, src.replace(".cu", ".o")) for src in SOURCES]
    cmds = [[NVCC, *ARCH, *FLAGS, *EXTRA.get(src, []), "-c", os.path.join(CSRC, src), "-o", obj]
            for src, obj in zip(SOURCES, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd))
    # the translation units are independent: compile them concurrently
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for r in ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args)
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))

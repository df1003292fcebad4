"""Builds libswb_cuda.so in-tree with nvcc for sm_100a.

    python -m swiftbwa_b200.build [--debug] [--ptxas-v]

The library is a plain C-ABI shared object (include/swb_cuda.h): no torch,
no Python.  cudart is linked statically so the .so only needs the driver.
Each .cu file compiles to its own object (in parallel, rebuilt when the file
or any header is newer than the object) and one nvcc call links them.
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
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libswb_cuda.so")
SOURCES = ["swb_runtime.cu", "swb_ext.cu", "swb_global.cu", "swb_local.cu", "swb_probe.cu", "swb_noalloc.cu",
           "swb_cigar.cu", "swb_serve.cu", "swb_extend.cu", "swb_rescue.cu", "swb_seed.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


WORKLOAD_SRC = os.path.join(CSRC, "swb_workload.cpp")
WORKLOAD_OUT = os.path.join(HERE, "libswb_workload.so")


def build_workload() -> str:
    """Host-only synthetic workload generator (g++)."""
    deps = [WORKLOAD_SRC, os.path.join(HERE, "..", "include", "swb_cuda.h")]
    if os.path.exists(WORKLOAD_OUT) and all(os.path.getmtime(d) <= os.path.getmtime(WORKLOAD_OUT) for d in deps):
        return WORKLOAD_OUT
    cxx = shutil.which("g++") or "g++"
    subprocess.run([cxx, "-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-shared", "-pthread",
                    "-o", WORKLOAD_OUT + ".tmp", WORKLOAD_SRC], check=True)
    os.replace(WORKLOAD_OUT + ".tmp", WORKLOAD_OUT)
    return WORKLOAD_OUT


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(debug: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    build_workload()
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "swb_cuda.h"))
    force = debug or ptxas_v
    if not force and not _stale(OUT, srcs + headers):
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    extra = (["-DSWB_DEBUG=1"] if debug else []) + (["-Xptxas", "-v"] if ptxas_v else [])
    objs, jobs = [], []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers]):
            jobs.append([nvcc(), *ARCH, *FLAGS, *extra, "-c", "-o", o + ".tmp", s])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(cmd[cmd.index("-o") + 1], cmd[cmd.index("-o") + 1][:-4])

    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            for f in [ex.submit(run, j) for j in jobs]:
                f.result()
    if jobs or _stale(OUT, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", OUT + ".tmp", *objs]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    args = ap.parse_args()
    print(build(debug=args.debug, verbose=True, ptxas_v=args.ptxas_v))

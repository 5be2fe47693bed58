"""Builds ``libhislam2_b200.so`` (all CUDA kernels + the C ABI) for sm_100a.

Usage: ``python hi-slam2_b200/hislam2_b200/build.py [-j N] [--force]``.
The library is written next to this file so that it travels with the source
tree; ``hislam2_b200._lib`` loads it from there.
"""

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.normpath(os.path.join(HERE, "..", "..", "include"))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhislam2_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--use_fast_math", "-Xcompiler", "-fPIC",
              "-Xptxas", "-warn-spills", "-I", INCLUDE]
# FP32 kernels are compiled without fast-math: the BA numerics follow IEEE division/sqrt.
NVCC_FLAGS.remove("--use_fast_math")


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build hislam2_b200")
    return exe


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(jobs=None, force=False, verbose=False, extra_flags=()):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "hislam2_b200.h"))
    objs, todo = [], []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            todo.append((src, obj))

    def compile_one(job):
        src, obj = job
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + list(extra_flags) + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
        return src, r.stderr

    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        for src, err in ex.map(compile_one, todo):
            if verbose and err.strip():
                print(os.path.basename(src), err, file=sys.stderr)
    if todo or force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print register/smem usage per kernel")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_info else []
    print(build(a.jobs, a.force or a.ptxas_info, a.verbose or a.ptxas_info, extra))

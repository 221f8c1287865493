"""Build the in-tree sm_100a library ``lib/libmomgpu.so`` and the ``mom_b200`` driver.

Every CUDA source is compiled with ``-gencode arch=compute_100a,code=sm_100a``
by nvcc (cross-compiles without a GPU); host C++ is compiled by nvcc's host
compiler with ``-ffp-contract=off`` so the geometry matches the reference's
FP64 arithmetic.  Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libmomgpu.so")
EXE = os.path.join(HERE, "bin", "mom_b200")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off",
           "-Xptxas", "-warn-spills"] + ARCH


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return (glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    nvcc = _nvcc()
    hdr = _headers()
    srcs = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu"))) + [os.path.join(HERE, "host", "problem.cpp")]
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if _stale(o, [s] + hdr):
            jobs.append([nvcc] + CUFLAGS + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcublas"])
    main = os.path.join(HERE, "host", "mom_main.cpp")
    if os.path.exists(main) and _stale(EXE, [main, LIB] + hdr):
        _run([nvcc, "-O2", "-std=c++17", "-o", EXE, main, "-L" + os.path.dirname(LIB), "-lmomgpu",
              "-Xlinker", "-rpath,$ORIGIN/../lib"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

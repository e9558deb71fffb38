"""Build libcxg.so (the CUDA kernels + C ABI) for sm_100a, in-tree.

    python -m calculixpp_b200.build [--verbose]

Output: calculixpp_b200/_lib/libcxg.so. nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libcxg.so")
SOURCES = ["cxg_api.cu", "cxg_kernels.cu", "cxg_pattern.cu", "cxg_v2.cu", "cxg_solve.cu", "cxg_batch.cu", "cxg_recover.cu",
           "cxg_refpattern.cu", "cxg_mpc.cu", "cxg_sparse_solve.cu", "cxg_film.cu"]
# Per-file flags: the reference-pattern mask evaluates K_e in the reference's own FP64
# operation order, so it must not contract multiply-adds.
EXTRA_FLAGS = {"cxg_refpattern.cu": ["-fmad=false"]}
HEADERS = ["cxg_internal.cuh", "cxg_elements.hpp", "cxg_plan.hpp", os.path.join("..", "..", "include", "cxg.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.exists(cand) or cand == "nvcc"):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS]
    if not force and not _stale(LIB, deps):
        return LIB
    objs, procs = [], []
    for src in srcs:  # the translation units compile in parallel
        obj = os.path.join(OUT_DIR, os.path.basename(src).replace(".cu", ".o"))
        cmd = [_nvcc(), *NVCC_FLAGS, *EXTRA_FLAGS.get(os.path.basename(src), []), "-dc", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
           *objs, "-o", LIB, "-lcusolver", "-lcusparse"]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))

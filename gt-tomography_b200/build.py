"""Builds the CUDA library libcbct.so in-tree for sm_100a.

    python gt-tomography_b200/build.py [--force]

Each csrc/*.cu is compiled by nvcc for `-gencode arch=compute_100a,code=sm_100a`
with -lineinfo and linked into gt-tomography_b200/_build/libcbct.so together
with the static CUDA runtime.  Rebuilds only what changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libcbct.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I", os.path.join(HERE, "..", "include"),
]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(HERE, "..", "include", "*.h"))


def _compile(src: str, obj: str, extra: list[str]) -> str:
    cmd = [NVCC, *NVCC_FLAGS, *extra, "-c", src, "-o", obj + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    os.replace(obj + ".tmp", obj)
    return r.stderr


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    extra = list(extra or [])
    os.makedirs(OUT_DIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_mtime = max(os.path.getmtime(h) for h in _headers() + [__file__])
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(OUT_DIR, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_mtime):
            jobs.append((s, o))
    if jobs:
        # The plain reference-replica path is compiled with --use_fast_math, as the
        # reference itself is (its CMakeLists.txt:52); the product kernels are not.
        def flags(src):
            return extra + (["--use_fast_math"] if os.path.basename(src).startswith("plain_") else [])
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for msg in ex.map(lambda j: _compile(j[0], j[1], flags(j[0])), jobs):
                if verbose and msg:
                    print(msg, file=sys.stderr)
    if force or jobs or not os.path.exists(LIB):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
               "-cudart", "static", *objs, "-o", LIB + ".tmp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    ptxas = "--ptxas-v" in sys.argv
    print(build(force="--force" in sys.argv or ptxas, verbose=ptxas,
                extra=["-Xptxas", "-v"] if ptxas else None))

"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/cbct_oracle.cpp into oracle/_build/liboracle.so with g++ and
OpenMP.  The reference itself is not built: it needs the Gadgetron toolbox,
Boost and HDF5, and its kernels use CUDA texture references that CUDA 12
removed, so there is no oracle/_ref recipe.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cbct_oracle.cpp")
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "liboracle.so")

# x86-64-v3 (AVX2/FMA) so that a library built on one host loads on another.
CXXFLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
            "-fno-fast-math", "-Wall", "-Wno-unknown-pragmas"]


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if (not force and os.path.exists(OUT)
            and os.path.getmtime(OUT) >= os.path.getmtime(SRC)
            and os.path.getmtime(OUT) >= os.path.getmtime(__file__)):
        return OUT
    cmd = ["g++", *CXXFLAGS, SRC, "-o", OUT + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))

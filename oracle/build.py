"""Build recipe of liboracle.so (the C++ FP64 oracle, OpenMP).  Test infrastructure.

-ffp-contract=off keeps the arithmetic unfused, like the reference's Julia code.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SRCS = [HERE / "oracle.cpp", HERE / "poisson.cpp", HERE / "fluid.cpp"]


def build(verbose: bool = False) -> Path:
    deps = SRCS + [HERE / "oracle.h"]
    if LIB.exists() and LIB.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-Wall",
           "-o", str(LIB)] + [str(x) for x in SRCS]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)

"""Build recipe of the engine's shared library (sm_100a, in-tree).

    python -m garli_b200.build          # builds garli_b200/libgarli_b200.so

The library is a plain C-ABI .so (include/garli_b200.h); nvcc compiles the
CUDA translation unit for sm_100a only and the host-side C++ (model math and
the tree driver) with the same toolchain.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgarli_b200.so")

SOURCES = ["gb_engine.cu", "gb_model.cpp", "gb_tree.cpp", "gb_modelopt.cpp", "gb_population.cpp", "gb_noalloc.cu"]
HEADERS = ["gb_common.cuh", "gb_dna.cuh", "gb_nstate.cuh", "gb_pmat.cuh", "gb_newton.h", "gb_graph.cuh",
           "gb_newton_dna.cuh", "gb_persist.cuh", "gb_batch.cuh", "gb_batch_mixed.cuh", "gb_tc.cuh", "gb_persist_mixed.cuh", "gb_eigen.cuh", "gb_stage.cuh"]
GENCODE = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def nvcc_available() -> bool:
    try:
        nvcc()
        return True
    except RuntimeError:
        return False


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "garli_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [
        nvcc(), GENCODE, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O2,-fopenmp",
        "-Xptxas", "-v" if verbose else "-O3",
        "-I", os.path.join(ROOT, "include"),
        "-o", LIB + ".tmp",
    ] + [os.path.join(CSRC, s) for s in SOURCES] + ["-lcudart", "-lgomp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

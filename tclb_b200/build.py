"""Build the CUDA extension libtclb_b200.so in-tree for sm_100a.

    python -m tclb_b200.build [--force] [--verbose]

The library is a plain CUDA/C++ shared object with a C ABI (include/tclb_b200.h);
it does not link against PyTorch.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtclb_b200.so")
SOURCES = ["tclb_b200.cu", "batch.cu", "case.cpp"]
HEADERS = ["lbm_kernels.cuh", "lbm_batch.cuh", "lbm_tma.cuh", "f32x2.cuh", "tclb_models.h", "cumulant_gen.cuh", "xml.hpp"]
RUNNER = os.path.join(HERE, "tclb_run")
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "tclb_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and not _stale():
        return LIB
    cmd = [_nvcc()] + NVCC_FLAGS + (extra or []) + ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES] + ["-lz"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd, cwd=CSRC)
    # the case-file runner executable, linked against the library
    runner = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-o", RUNNER, os.path.join(CSRC, "tclb_run.cpp"), "-L" + HERE,
              "-ltclb_b200", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN"]
    if verbose:
        print(" ".join(runner), flush=True)
    subprocess.check_call(runner, cwd=CSRC)
    return LIB


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--force", action="store_true")
    p.add_argument("--verbose", action="store_true")
    p.add_argument("--ptxas-v", action="store_true", help="print register/spill usage")
    a = p.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_v else None
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose, extra=extra))


if __name__ == "__main__":
    sys.exit(main())

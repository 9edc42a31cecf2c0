"""Build the sm_100a shared library ``bart_b200/lib/libbnufft.so`` in-tree.

``python -m bart_b200.build`` (or ``build()``) runs nvcc directly; the
library has a plain C ABI (include/bnufft.h, include/bespirit.h) and links only the CUDA
runtime; the ESPIRiT calibration loads cuSOLVER on first use.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "lib", "libbnufft.so")
SOURCES = [os.path.join(HERE, "csrc", "bnufft.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("fft_core.cuh", "nufft_kernels.cuh", "cg_kernels.cuh", "gridding.cuh",
                                                   "precnet.cuh", "nudft.cuh", "precond_cluster.cuh", "fft512.cuh",
                                                   "precnet_tc.cuh", "espirit.cuh", "cgext.cuh")] + \
    [os.path.join(ROOT, "include", f) for f in ("bnufft.h", "bespirit.h")]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "--cudart", "shared",
         "-I" + os.path.join(ROOT, "include")]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + SOURCES + ["-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose:
        sys.stderr.write(r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

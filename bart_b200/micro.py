"""Microbenchmarks that give the rooflines of this library's kernels.

    python -m bart_b200.micro atomics

``atomics`` builds (nvcc, sm_100a) and runs csrc/micro_atomics.cu: atomic-add
throughput in shared and global memory, the bound of the gridding scatter.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def build_atomics() -> str:
    src = os.path.join(HERE, "csrc", "micro_atomics.cu")
    exe = os.path.join(HERE, "lib", "micro_atomics")
    if not os.path.exists(exe) or os.path.getmtime(exe) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(exe), exist_ok=True)
        subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-o", exe, src], check=True)
    return exe


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if not argv or argv[0] != "atomics":
        print(__doc__)
        return 2
    r = subprocess.run([build_atomics()])
    return r.returncode


if __name__ == "__main__":
    sys.exit(main())

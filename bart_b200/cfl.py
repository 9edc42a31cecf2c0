"""BART ``.cfl`` / ``.hdr`` file I/O (src/misc/mmio.c, src/misc/io.c:379-400).

A ``.cfl`` file is raw complex64 in column-major order; the ``.hdr`` text
file holds ``# Dimensions`` and the dims (16 of them as written here).
"""

from __future__ import annotations

import numpy as np

DIMS = 16


def readcfl(name: str) -> np.ndarray:
    """Read ``name.hdr`` / ``name.cfl`` into an F-ordered complex64 array."""
    with open(name + ".hdr") as f:
        lines = f.read().split("\n")
    i = lines.index("# Dimensions")
    dims = [int(x) for x in lines[i + 1].split()]
    n = int(np.prod(dims))
    data = np.fromfile(name + ".cfl", dtype=np.complex64, count=n)
    if data.size != n:
        raise ValueError(f"{name}.cfl holds {data.size} values, header says {n}")
    return data.reshape(dims, order="F")


def writecfl(name: str, array: np.ndarray) -> None:
    """Write an array (BART dim order) as ``name.hdr`` / ``name.cfl``."""
    a = np.asarray(array, dtype=np.complex64)
    dims = list(a.shape) + [1] * (DIMS - a.ndim)
    with open(name + ".hdr", "w") as f:
        f.write("# Dimensions\n" + " ".join(str(d) for d in dims) + " \n")
    np.asfortranarray(a).ravel(order="F").tofile(name + ".cfl")


def dims16(shape) -> list:
    """Pad a shape to BART's 16 dims."""
    s = [int(d) for d in shape]
    if len(s) > DIMS:
        raise ValueError("more than 16 dims")
    return s + [1] * (DIMS - len(s))

"""PLOT3D multi-block grid files (famrdp_jax ``mesh/io_grd.py:5-29``).

Layout (little-endian binary stream, no record markers): int32 nblocks; then
int32 (ni, nj, nk) per block; then per block the x, y and z coordinate arrays
of ni*nj*nk float64 values each, in Fortran (column-major, i fastest) order.
Blocks come back as float64 arrays of shape (3, ni, nj, nk), axis 0 = x, y, z.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np


def read_grd(path) -> list[np.ndarray]:
    """The blocks of a PLOT3D grid file, each (3, ni, nj, nk) float64."""
    raw = Path(path).read_bytes()
    head = np.frombuffer(raw, dtype="<i4", count=1)
    if head.size != 1 or head[0] < 0:
        raise ValueError(f"{path}: not a PLOT3D grid file")
    nb = int(head[0])
    dims = np.frombuffer(raw, dtype="<i4", count=3 * nb, offset=4).reshape(nb, 3).astype(int)
    off = 4 + 12 * nb
    blocks = []
    for ni, nj, nk in dims:
        n = int(ni) * int(nj) * int(nk)
        if off + 24 * n > len(raw):
            raise ValueError(f"{path}: truncated coordinate data")
        xyz = np.frombuffer(raw, dtype="<f8", count=3 * n, offset=off).reshape(3, n)
        off += 24 * n
        blocks.append(np.stack([c.reshape((ni, nj, nk), order="F") for c in xyz]).astype(np.float64))
    return blocks


def write_grd(path, blocks) -> None:
    """Writes blocks of shape (3, ni, nj, nk) in the layout read_grd reads."""
    with open(path, "wb") as f:
        np.asarray([len(blocks)], dtype="<i4").tofile(f)
        for b in blocks:
            np.asarray(b.shape[1:], dtype="<i4").tofile(f)
        for b in blocks:
            for c in range(3):
                np.asarray(b[c], dtype="<f8").ravel(order="F").tofile(f)

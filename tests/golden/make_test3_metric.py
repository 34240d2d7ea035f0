"""Writes tests/golden/test3_metric.npz from the reference's Fortran probe data.

Source (read only, in the reference checkout):
  validation/references/test3/xyz/block_000{1,2}.bin     -- coordinates
  validation/references/test3/metric/block_000{1,2}_jac.bin -- Jacobian
in the probe format of validation/fortran_ref.py:6-31 (int32 shape header,
float64 data in Fortran order).  Both blocks are 51 x 51 x 11 nodes.  The
reference's own check (tests/validation/test_m11_metric_match.py:23-36)
compares compute_metrics(xyz).jac against this Jacobian with atol 1e-13.

    python tests/golden/make_test3_metric.py REFERENCE_ROOT

REFERENCE_ROOT is the root of a famrdp_jax checkout (or set
FAMRDP_JAX_REFERENCE).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np


def _read_probe(path: Path, ndim: int) -> np.ndarray:
    with open(path, "rb") as f:
        shape = tuple(int(x) for x in np.fromfile(f, dtype="<i4", count=ndim))
        return np.fromfile(f, dtype="<f8", count=int(np.prod(shape))).reshape(shape, order="F")


def _read_xyz(path: Path) -> np.ndarray:
    with open(path, "rb") as f:
        ni, nj, nk = (int(x) for x in np.fromfile(f, dtype="<i4", count=3))
        comps = [np.fromfile(f, dtype="<f8", count=ni * nj * nk).reshape((ni, nj, nk), order="F")
                 for _ in range(3)]
    return np.stack(comps, axis=0)


def main(ref_root: str | None = None) -> Path:
    import os
    ref_root = ref_root or os.environ.get("FAMRDP_JAX_REFERENCE")
    if not ref_root:
        raise SystemExit("usage: make_test3_metric.py REFERENCE_ROOT (or set FAMRDP_JAX_REFERENCE)")
    base = Path(ref_root) / "validation" / "references" / "test3"
    out = {}
    for b in (1, 2):
        out[f"xyz{b}"] = np.ascontiguousarray(_read_xyz(base / "xyz" / f"block_{b:04d}.bin"))
        out[f"jac{b}"] = np.ascontiguousarray(_read_probe(base / "metric" / f"block_{b:04d}_jac.bin", 3))
    dst = Path(__file__).resolve().parent / "test3_metric.npz"
    np.savez_compressed(dst, **out)
    return dst


if __name__ == "__main__":
    print(main(*sys.argv[1:]))

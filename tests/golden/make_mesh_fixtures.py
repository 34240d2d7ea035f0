"""Writes the grid/topology fixtures of tests/test_mesh_io.py:

  mini.grd  PLOT3D, two blocks of (4, 3, 2) and (3, 3, 2) nodes on the unit
            cube (x, y, z = linspace(0, 1) per axis), written with
            famrdp_jax_b200.mesh.io_grd.write_grd;
  mini.inp  GridGen topology of two 5 x 5 x 3 blocks A and B joined JMAX(A) ->
            JMIN(B) and JMIN(A) <- JMAX(B) (a periodic pair in j), with WALL on
            the k faces and SYMMETRY / FARFIELD on the i faces.

Run from the repository root:  python tests/golden/make_mesh_fixtures.py
"""
from pathlib import Path
import sys

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from famrdp_jax_b200.mesh.io_grd import write_grd  # noqa: E402


def grid():
    out = []
    for ni, nj, nk in ((4, 3, 2), (3, 3, 2)):
        axes = [np.linspace(0.0, 1.0, n) for n in (ni, nj, nk)]
        out.append(np.stack(np.meshgrid(*axes, indexing="ij")))
    write_grd(HERE / "mini.grd", out)


def topology():
    def line(v):
        return " ".join(f"{x:7d}" for x in v)

    rows = ["1", "2"]
    for name, nbr in (("A", 2), ("B", 1)):
        rows += ["5 5 3", name, "6",
                 line([1, 5, 1, 5, 1, 1, 2]),      # KMIN wall
                 line([1, 5, 1, 5, 3, 3, 2]),      # KMAX wall
                 line([1, 1, 1, 5, 1, 3, 3]),      # IMIN symmetry
                 line([5, 5, 1, 5, 1, 3, 4]),      # IMAX farfield
                 line([1, 5, 5, 5, -3, -1, -1]),   # JMAX interface ...
                 line([1, 5, 1, 1, -3, -1, nbr]),  # ... with the neighbour's JMIN
                 line([1, 5, 1, 1, -3, -1, -1]),   # JMIN interface ...
                 line([1, 5, 5, 5, -3, -1, nbr])]  # ... with the neighbour's JMAX
    (HERE / "mini.inp").write_text("\n".join(rows) + "\n")


if __name__ == "__main__":
    grid()
    topology()
    print("wrote", HERE / "mini.grd", HERE / "mini.inp")

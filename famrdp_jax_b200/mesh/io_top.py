"""GridGen ``.inp`` block topology files (famrdp_jax ``mesh/io_top.py``).

Grammar (whitespace-separated integers, blank lines ignored):
  line 1      a header value (ignored)
  line 2      nblocks
  per block   ni nj nk / a label line / nbc, then nbc logical face entries,
              each ``is ie js je ks ke value``:
                value > 1   a physical boundary (BCType value) on the face the
                            degenerate index range names;
                value == -1 (CUT1TO1) an interface: a second line follows with
                            the neighbour's face range and, as its value, the
                            neighbour's 1-based block number.
The face of a range is the axis whose start equals its end, on absolute
values (interface lines may carry negative placeholders): the MIN face when
that index is 1 (for k also when it is 0), the MAX face otherwise; a range
with no degenerate axis falls back to the axis of smallest extent, MIN when
its start is at most half the current block's extent (mesh/io_top.py:36-90;
the current block's extents are used for the neighbour's line too, as there).

Orientation.  The reference stores every interface as orientation 1
(mesh/io_top.py:183), which its halo fill rejects (mesh/halo.py:86-87), so no
parsed multi-block topology can be stepped there.  Here an interface whose
two faces lie on the same axis with both tangential index ranges running the
same way is stored as orientation 0, the aligned copy the halo fill performs;
any other interface keeps the reference's 1, and the halo fill rejects it
with NotImplementedError as the reference does.
"""
from __future__ import annotations

from pathlib import Path

from famrdp_jax_b200.core.constants import BCType, Face
from famrdp_jax_b200.core.types import BlockTopology

_AXIS_FACES = ((Face.IMIN, Face.IMAX), (Face.JMIN, Face.JMAX), (Face.KMIN, Face.KMAX))


def _face(rng, dims) -> Face:
    """Face of a 6-value index range (absolute values, mesh/io_top.py:36-90)."""
    lo = [abs(rng[0]), abs(rng[2]), abs(rng[4])]
    hi = [abs(rng[1]), abs(rng[3]), abs(rng[5])]
    for a in range(3):
        if lo[a] == hi[a]:
            is_min = lo[a] == 1 or (a == 2 and lo[a] <= 0)
            return _AXIS_FACES[a][0] if is_min else _AXIS_FACES[a][1]
    ext = [abs(hi[a] - lo[a]) for a in range(3)]
    a = ext.index(min(ext))
    return _AXIS_FACES[a][0] if lo[a] <= dims[a] // 2 else _AXIS_FACES[a][1]


def _orientation(mine, nbr, my_face: Face, nbr_face: Face) -> int:
    """0 when the two faces share their axis and both tangential ranges run the
    same way (the aligned copy), else the reference's marker 1."""
    ax = int(my_face) // 2 if isinstance(my_face, Face) else None
    if ax is None or ax != int(nbr_face) // 2:
        return 1
    for t in range(3):
        if t == ax:
            continue
        d1 = abs(mine[2 * t + 1]) - abs(mine[2 * t])
        d2 = abs(nbr[2 * t + 1]) - abs(nbr[2 * t])
        if (d1 > 0) != (d2 > 0) or (d1 < 0) != (d2 < 0):
            return 1
    return 0


def parse_topology(path) -> list[BlockTopology]:
    """One BlockTopology per block of a GridGen .inp file (0-based ids)."""
    rows = [ln.split() for ln in Path(path).read_text().splitlines() if ln.strip()]
    pos = 1  # the header line is ignored
    nblocks = int(rows[pos][0])
    pos += 1
    out = []
    for bid in range(nblocks):
        dims = [int(x) for x in rows[pos][:3]]
        pos += 2  # dimensions, label
        nbc = int(rows[pos][0])
        pos += 1
        bc_type, neighbors = {}, {}
        for _ in range(nbc):
            row = [int(x) for x in rows[pos][:7]]
            pos += 1
            face = _face(row[:6], dims)
            if row[6] == int(BCType.CUT1TO1):
                nrow = [int(x) for x in rows[pos][:7]]
                pos += 1
                nface = _face(nrow[:6], dims)
                bc_type[face] = BCType.CUT1TO1
                neighbors[face] = (nrow[6] - 1, nface, _orientation(row[:6], nrow[:6], face, nface))
            else:
                bc_type[face] = BCType(row[6])
                neighbors[face] = None
        out.append(BlockTopology(block_id=bid, neighbors=neighbors, bc_type=bc_type))
    return out

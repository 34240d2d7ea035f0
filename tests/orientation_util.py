"""NumPy statement of the mapped interface orientation (no test functions).

The reference's halo fill only copies equal-shaped slabs element by element
(orientation 0, mesh/halo.py:36-53) and rejects every other orientation
(mesh/halo.py:86-87); ``core.constants.ORIENT_MAPPED`` codes are this
library's extension.  This module writes their definition out cell by cell,
independently of the CUDA code's affine index map, for the tests to compare
against:

* the target ghost layer at distance d (1..g) from the interface takes the
  source's interior layer at distance d;
* the target face's tangential axes (t0 < t1) map onto the source face's
  (s0 < s1), swapped when ORIENT_SWAP is set; ORIENT_REV_A / ORIENT_REV_B run
  t0 / t1 backwards over the source's full extent;
* links apply in order, all reading the pre-exchange arrays (the reference's
  rule), so a later link wins where ghost slabs overlap.
"""
import numpy as np

from famrdp_jax_b200.core.constants import ORIENT_REV_A, ORIENT_REV_B, ORIENT_SWAP, Face


def _tangential(axis):
    return [a for a in range(3) if a != axis]


def mapped_copy(tgt, src, tgt_face, src_face, orient, g):
    """tgt (5, n...) with the ghost slab of tgt_face filled from src through
    the mapped orientation ``orient``; returns a new array."""
    out = tgt.copy()
    ta, sa = int(tgt_face) // 2, int(src_face) // 2
    tn, sn = tgt.shape[1:], src.shape[1:]
    tt, st = _tangential(ta), _tangential(sa)
    if orient & ORIENT_SWAP:
        st = st[::-1]
    rev = [bool(orient & ORIENT_REV_A), bool(orient & ORIENT_REV_B)]
    for m in range(2):
        if tn[tt[m]] != sn[st[m]]:
            raise ValueError("halo slab shape mismatch")
    for d in range(1, g + 1):
        t_layer = g - d if int(tgt_face) % 2 == 0 else tn[ta] - g - 1 + d
        s_layer = g + d - 1 if int(src_face) % 2 == 0 else sn[sa] - g - d
        for u in range(tn[tt[0]]):
            for v in range(tn[tt[1]]):
                ti = [0, 0, 0]
                ti[ta], ti[tt[0]], ti[tt[1]] = t_layer, u, v
                si = [0, 0, 0]
                si[sa] = s_layer
                si[st[0]] = sn[st[0]] - 1 - u if rev[0] else u
                si[st[1]] = sn[st[1]] - 1 - v if rev[1] else v
                out[(slice(None),) + tuple(ti)] = src[(slice(None),) + tuple(si)]
    return out


def mapped_halo(qs, links, g):
    """All links (tgt_block, tgt_face, src_block, src_face, orient) in order,
    every source read from the pre-exchange arrays; orientation 0 links use
    the oracle's statement of the reference's copy (mesh/halo.py:36-53)."""
    from oracle.ref import NP
    orig = [q.copy() for q in qs]
    out = [q.copy() for q in qs]
    for tb, tf, sb, sf, o in links:
        if o == 0:
            out[tb] = np.asarray(NP._copy_face(out[tb].copy(), orig[sb], Face(tf), Face(sf), g))
        else:
            out[tb] = mapped_copy(out[tb], orig[sb], tf, sf, o, g)
    return out


def relabel(arr, perm, flip, lead=1):
    """A block's array with its spatial axes relabelled: new axis a is old axis
    perm[a], run backwards where flip[a].  ``lead`` = number of leading
    non-spatial axes (1 for q, 2 for kxyz, 0 for vol)."""
    x = np.transpose(arr, tuple(range(lead)) + tuple(lead + p for p in perm))
    for a in range(3):
        if flip[a]:
            x = np.flip(x, axis=lead + a)
    return np.ascontiguousarray(x)


def relabel_kxyz(kxyz, perm, flip):
    """Metrics of the relabelled block: kxyz[l][m] = d xi_l / d x_m, so row l
    of the new block is row perm[l] of the old one, negated where the axis runs
    backwards; the cells are relabelled like q's."""
    rows = np.stack([(-1.0 if flip[l] else 1.0) * kxyz[perm[l]] for l in range(3)])
    return relabel(rows, perm, flip, lead=2)


def unrelabel(arr, perm, flip, lead=1):
    """Inverse of relabel."""
    x = arr
    for a in range(3):
        if flip[a]:
            x = np.flip(x, axis=lead + a)
    inv = [perm.index(a) for a in range(3)]
    return np.ascontiguousarray(np.transpose(x, tuple(range(lead)) + tuple(lead + p for p in inv)))

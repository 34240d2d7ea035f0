"""Enumerations of the block/face/boundary vocabulary.

Values and names follow famrdp_jax ``core/constants.py:4-64`` exactly, so a
topology written for the reference (``Face`` keys, ``BCType`` values,
``orient`` flags) means the same thing here.
"""
from enum import IntEnum


class BCType(IntEnum):
    """Boundary types (core/constants.py:4-12).  CUT1TO1 is a block interface."""
    CUT1TO1 = -1
    WALL = 2
    SYMMETRY = 3
    FARFIELD = 4
    INFLOW = 5
    OUTFLOW = 6
    POLE = 7
    PATCHED = 8


class WallSubType(IntEnum):
    """core/constants.py:15-18"""
    ADIABATIC = 1
    ISOTHERMAL = 2
    SLIP = 3


class Face(IntEnum):
    """Block faces (core/constants.py:54-60); the array axis of IMIN/IMAX is 1
    of q's (5, ni, nj, nk), of JMIN/JMAX 2 and of KMIN/KMAX 3."""
    IMIN = 0
    IMAX = 1
    JMIN = 2
    JMAX = 3
    KMIN = 4
    KMAX = 5


N_EQN = 5  # rho, rho*u, rho*v, rho*w, rho*E
N_DIM = 3

# Interface orientation codes (``neighbors[face] = (block_id, face, orient)``):
# 0 is the reference's element-by-element slab copy (mesh/halo.py:36-53); the
# reference rejects every other value (mesh/halo.py:86-87), including the 1 its
# topology reader stores.  ORIENT_MAPPED | bits is this library's face-to-face
# mapping, for interfaces whose index directions differ between the two
# blocks (no counterpart in the reference): the ghost layer at distance d from
# the interface takes the source's interior layer at distance d, and the
# target face's two tangential axes, in i, j, k order, map onto the source
# face's, ORIENT_SWAP pairing the first with the second and ORIENT_REV_A /
# ORIENT_REV_B running the target's first / second one backwards on the source.
ORIENT_MAPPED = 8
ORIENT_SWAP = 1
ORIENT_REV_A = 2
ORIENT_REV_B = 4


def mapped_orientation(swap: bool = False, reverse_a: bool = False, reverse_b: bool = False) -> int:
    """The orientation code of a mapped interface (see ORIENT_MAPPED)."""
    return ORIENT_MAPPED | (ORIENT_SWAP if swap else 0) | (ORIENT_REV_A if reverse_a else 0) | \
        (ORIENT_REV_B if reverse_b else 0)


def orientation_supported(orient: int) -> bool:
    """0 (the reference's copy) or a mapped code ORIENT_MAPPED | bits."""
    return orient == 0 or (int(orient) & ~7) == ORIENT_MAPPED

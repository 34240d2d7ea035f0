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

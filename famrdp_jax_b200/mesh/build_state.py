"""Initial multi-block state from a PLOT3D grid and a GridGen topology
(famrdp_jax ``mesh/build_state.py``).

Each block's coordinates are padded by ``ghost`` layers per side by edge
replication; q comes from ``q_init_fn((5, ni, nj, nk))`` on the padded shape.
Like the reference, the metrics are placeholders (jac = vol = 1, kxyz = 0):
edge-replicated ghost coordinates have zero spacing, so metrics of the padded
coordinates would be singular there; callers compute metrics from
coordinates with proper ghost layers (compute_metrics).
"""
from __future__ import annotations

import numpy as np
import torch

from famrdp_jax_b200.core.types import Block, Metrics, State
from famrdp_jax_b200.mesh.io_grd import read_grd
from famrdp_jax_b200.mesh.io_top import parse_topology


def _pad_xyz(xyz: np.ndarray, ghost: int) -> np.ndarray:
    return np.pad(xyz, ((0, 0),) + ((ghost, ghost),) * 3, mode="edge")


def build_initial_state(grd_path, inp_path, ghost: int, q_init_fn, *, device="cpu"):
    """(State, topologies) for the grid and topology files."""
    blocks, metrics = [], []
    for xyz in read_grd(grd_path):
        pad = _pad_xyz(xyz, ghost)
        shape = pad.shape[1:]
        q = torch.as_tensor(np.asarray(q_init_fn((5,) + shape)), dtype=torch.float64, device=device)
        x = torch.as_tensor(pad, dtype=torch.float64, device=device)
        blocks.append(Block(q=q, xyz=x))
        metrics.append(Metrics(jac=torch.ones(shape, dtype=torch.float64, device=device),
                               kxyz=torch.zeros((3, 3) + shape, dtype=torch.float64, device=device),
                               vol=torch.ones(shape, dtype=torch.float64, device=device)))
    return State(blocks=tuple(blocks), metrics=tuple(metrics), t=0.0, step=0), tuple(parse_topology(inp_path))

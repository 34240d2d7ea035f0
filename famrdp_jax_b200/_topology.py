"""Topology marshalling: BlockTopology / Config -> the C ABI's link, boundary
and block tables.

The order of the tables carries the reference's semantics:
  * links follow (block order, ``neighbors`` dict insertion order)
    (mesh/halo.py:76-90); a later link overwrites an earlier one where their
    ghost slabs overlap;
  * boundary faces follow (block, Face enum order) (physics/bc/dispatch.py:15);
    CUT1TO1, absent faces and types the reference does not dispatch are
    skipped.
"""
from __future__ import annotations

import ctypes

import torch

from famrdp_jax_b200 import _capi
from famrdp_jax_b200.core.constants import BCType, Face, orientation_supported


def links(topos) -> list[tuple[int, int, int, int, int]]:
    """(tgt_block, tgt_face, src_block, src_face, orient) in halo order.
    An orientation other than 0 (the reference's copy) or a mapped code
    (``core.constants.ORIENT_MAPPED``) raises NotImplementedError
    (mesh/halo.py:86-87)."""
    id_to_idx = {t.block_id: i for i, t in enumerate(topos)}
    out = []
    for i, topo in enumerate(topos):
        for face, info in topo.neighbors.items():
            if info is None:
                continue
            if topo.bc_type.get(face) != BCType.CUT1TO1:
                continue
            nb_id, src_face, orient = info
            if not orientation_supported(orient):
                raise NotImplementedError(f"orient={orient} not supported in stage 1")
            out.append((i, int(face), id_to_idx[nb_id], int(src_face), int(orient)))
    return out


def bcs(topos, cfg) -> list[tuple]:
    """(block, face, type, isothermal, T_wall, q_inf) in dispatch order."""
    out = []
    for b, topo in enumerate(topos):
        for face in Face:
            bct = topo.bc_type.get(face)
            if bct is None or bct == BCType.CUT1TO1:
                continue
            bc_p = cfg.bc_params.get(face, {})
            if bct == BCType.WALL:
                iso = bc_p.get("wall_type", "adiabatic") == "isothermal"
                out.append((b, int(face), int(BCType.WALL), int(iso), float(bc_p.get("T_wall", 300.0)),
                            (0.0,) * 5))
            elif bct == BCType.SYMMETRY:
                out.append((b, int(face), int(BCType.SYMMETRY), 0, 0.0, (0.0,) * 5))
            elif bct == BCType.FARFIELD:
                qi = bc_p.get("q_inf", [1.0, 0.0, 0.0, 0.0, 2.5])
                if isinstance(qi, torch.Tensor):
                    qi = qi.detach().cpu().tolist()
                qi = tuple(float(x) for x in list(qi))
                if len(qi) != 5:
                    raise ValueError("q_inf must have 5 entries")
                out.append((b, int(face), int(BCType.FARFIELD), 0, 0.0, qi))
    return out


def link_array(ls):
    arr = (_capi.FjLink * max(1, len(ls)))()
    for n, (t, tf, s, sf, o) in enumerate(ls):
        arr[n].tgt_block, arr[n].tgt_face, arr[n].src_block, arr[n].src_face, arr[n].orient = t, tf, s, sf, o
    return arr


def bc_array(bs):
    arr = (_capi.FjBc * max(1, len(bs)))()
    for n, (b, f, ty, iso, tw, qi) in enumerate(bs):
        arr[n].block, arr[n].face, arr[n].type, arr[n].isothermal, arr[n].T_wall = b, f, ty, iso, tw
        for v in range(5):
            arr[n].q_inf[v] = qi[v]
    return arr


def block_array(qs, metrics=None):
    """fj_block table for a sequence of q tensors (and optional Metrics)."""
    arr = (_capi.FjBlock * len(qs))()
    for b, q in enumerate(qs):
        if q.dim() != 4 or q.shape[0] != 5:
            raise ValueError(f"block {b}: q must have shape (5, ni, nj, nk), got {tuple(q.shape)}")
        arr[b].q = _capi.dev_ptr(q, f"blocks[{b}].q")
        arr[b].ni, arr[b].nj, arr[b].nk = q.shape[1], q.shape[2], q.shape[3]
        if metrics is not None:
            m = metrics[b]
            if tuple(m.kxyz.shape) != (3, 3) + tuple(q.shape[1:]) or tuple(m.vol.shape) != tuple(q.shape[1:]):
                raise ValueError(f"block {b}: metrics shape does not match q")
            arr[b].kxyz = _capi.dev_ptr(m.kxyz, f"metrics[{b}].kxyz")
            arr[b].vol = _capi.dev_ptr(m.vol, f"metrics[{b}].vol")
    return arr


def ptr_array(ts):
    arr = (ctypes.c_void_p * len(ts))()
    for n, t in enumerate(ts):
        arr[n] = _capi.dev_ptr(t, f"out[{n}]")
    return arr

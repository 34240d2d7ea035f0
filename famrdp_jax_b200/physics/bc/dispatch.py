"""Boundary-condition dispatch (famrdp_jax ``physics/bc/dispatch.py:11-32``) on
the GPU: faces in Face enum order, CUT1TO1 and absent faces skipped; WALL
(adiabatic mirror or isothermal), SYMMETRY (mirror, normal velocity negated)
and FARFIELD (ghost layers := q_inf)."""
from __future__ import annotations

from famrdp_jax_b200 import _capi, _topology
from famrdp_jax_b200.core.types import Block, BlockTopology, Config


def apply_bc_blocks(qs, topos, cfg: Config) -> None:
    """In place on a list of q tensors (all blocks, one launch per face)."""
    bs = _topology.bcs(topos, cfg)
    if not bs:
        return
    dev = qs[0].device
    c = _capi.ctx(dev)
    p = _capi.params(cfg.gas, limiter=cfg.scheme.limiter, ghost=cfg.ghost,
                     precision=getattr(cfg, "precision", "f64"))
    _capi.check(_capi.lib().fj_apply_bc_f64(c, _topology.block_array(qs), len(qs), _topology.bc_array(bs),
                                            len(bs), p, _capi.stream(dev)), "fj_apply_bc_f64", c)


def apply_bc(block: Block, topo: BlockTopology, cfg: Config) -> Block:
    """New block with its physical boundary ghosts filled (input unchanged)."""
    q = block.q.clone()
    apply_bc_blocks([q], (topo,), cfg)
    return Block(q=q, xyz=block.xyz)

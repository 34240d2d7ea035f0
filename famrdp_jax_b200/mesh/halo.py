"""Inter-block halo fill (famrdp_jax ``mesh/halo.py:56-92``) on the GPU.

Every CUT1TO1 face copies the source block's 2-layer slab next to the source
face into the target's ghost slab (full extent along the other two axes),
reading all sources from the pre-exchange arrays; faces apply in (block,
neighbors-dict) order so later faces overwrite edges and corners.
Orientation 0 is the reference's element-by-element copy; a mapped code
(``core.constants.mapped_orientation``, no counterpart in the reference)
connects faces whose index directions differ; any other value raises
NotImplementedError as the reference does.
"""
from __future__ import annotations

from famrdp_jax_b200 import _capi, _topology
from famrdp_jax_b200.core.types import Block, BlockTopology


def halo_exchange(blocks: tuple[Block, ...], topos: tuple[BlockTopology, ...],
                  ghost: int) -> tuple[Block, ...]:
    """New blocks with their CUT1TO1 ghost layers filled (inputs unchanged)."""
    ls = _topology.links(topos)
    qs = [b.q.clone() for b in blocks]
    if ls:
        dev = qs[0].device
        c = _capi.ctx(dev)
        arr = _topology.block_array(qs)
        _capi.check(_capi.lib().fj_halo_exchange_f64(c, arr, len(qs), _topology.link_array(ls), len(ls),
                                                     int(ghost), _capi.stream(dev)),
                    "fj_halo_exchange_f64", c)
    return tuple(Block(q=qs[i], xyz=blocks[i].xyz) for i in range(len(blocks)))

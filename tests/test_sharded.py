"""Block sharding's host side on CPU: the partition, the per-rank halo
schedule and the exchange over two gloo ranks (127.0.0.1).  The packing and
unpacking of the slabs are restated here in NumPy for the reference's
element-by-element links (orient 0), so that a sharded halo fill can be
compared with the oracle's fill of all blocks (mesh/halo.py:56-92); the CUDA
pack/unpack kernels are compared with the unsharded step on the GPU
(tests/test_gpu_sharded.py)."""
import datetime
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from famrdp_jax_b200 import _topology, cases
from famrdp_jax_b200.solver import sharded
from oracle.ref import NP

ROOT = Path(__file__).resolve().parent.parent


def _case(name):
    if name == "tree24":
        return cases.tree24(nblocks=24, lo=6, hi=20, seed=3)
    if name == "wavy4":
        return cases.wavy4(n=10, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2))
    if name == "tgv":
        return cases.tgv(n=8)
    if name == "ragged":
        return cases.tree24(nblocks=7, lo=3, hi=23, seed=7)
    raise KeyError(name)


CASES = ["tree24", "wavy4", "tgv", "ragged"]


def test_partition_balances_and_is_deterministic():
    c = _case("tree24")
    shapes = [q.shape for q in c.qs]
    links = _topology.links(c.cfg.topology)
    cells = [int(np.prod(s[1:])) for s in shapes]
    for world in (1, 2, 3, 4, 8):
        owner = sharded.partition(shapes, links, world)
        assert owner == sharded.partition(shapes, links, world)
        assert sorted(set(owner)) == list(range(min(world, len(shapes))))
        load = [sum(cl for cl, o in zip(cells, owner) if o == r) for r in range(world)]
        # largest-first greedy: no rank exceeds the average by more than the slack plus one block
        assert max(load) <= sum(cells) / world * 1.05 + max(cells)
    assert sharded.partition(shapes, links, 1) == [0] * len(shapes)
    with pytest.raises(ValueError):
        sharded.partition(shapes, links, 0)


def test_partition_keeps_linked_equal_blocks_together():
    # four equal blocks in a ring (0-1-2-3-0) on two ranks: each rank gets two
    # linked blocks, so two of the four links are cut, not all four
    links = [(0, 1, 1, 0, 0), (1, 0, 0, 1, 0), (1, 1, 2, 0, 0), (2, 0, 1, 1, 0),
             (2, 1, 3, 0, 0), (3, 0, 2, 1, 0), (3, 1, 0, 0, 0), (0, 0, 3, 1, 0)]
    owner = sharded.partition([(5, 8, 8, 8)] * 4, links, 2)
    cut = sum(1 for (t, _tf, s, _sf, _o) in links if owner[t] != owner[s])
    assert sorted(owner) == [0, 0, 1, 1] and cut == 4


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_schedule_covers_every_link_once(name, world):
    c = _case(name)
    shapes = [q.shape for q in c.qs]
    links = _topology.links(c.cfg.topology)
    owner = sharded.partition(shapes, links, world)
    sch = [sharded.halo_schedule(shapes, links, owner, r, c.cfg.ghost) for r in range(world)]
    unpacked = sorted(L for s in sch for L, _ in s.unpack)
    packed = sorted(L for s in sch for L, _ in s.pack_local + s.pack_export)
    assert unpacked == list(range(len(links))) and packed == list(range(len(links)))
    for r, s in enumerate(sch):
        # unpack in link-list order; slabs aligned, inside the buffers, disjoint
        assert [L for L, _ in s.unpack] == sorted(L for L, _ in s.unpack)
        for pairs, size in ((s.unpack, s.fill_doubles), (s.pack_export, s.export_doubles)):
            spans = sorted((o, o + sharded._slab_doubles(shapes[links[L][0]], links[L][1], 2)) for L, o in pairs)
            assert all(o % sharded.ALIGN == 0 and e <= size for o, e in spans)
            assert all(a[1] <= b[0] for a, b in zip(spans, spans[1:]))
        for p in range(world):
            if p == r:
                continue
            # what r sends p is what p receives from r: same links, same order, same length
            sent = [L for L, o in s.pack_export if s.send[p][0] <= o < s.send[p][0] + s.send[p][1]] if p in s.send else []
            q = sch[p]
            got = ([L for L, o in q.unpack if q.recv[r][0] <= o < q.recv[r][0] + q.recv[r][1]]
                   if r in q.recv else [])
            assert sent == got
            assert s.send.get(p, (0, 0))[1] == q.recv.get(r, (0, 0))[1]


# ---- the exchange and a sharded fill over two gloo ranks -------------------
def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _box(shape, face, g, source):
    n = shape[-3:]
    ax = face >> 1
    sl = [slice(0, n[0]), slice(0, n[1]), slice(0, n[2])]
    if source:
        lo = g if face % 2 == 0 else n[ax] - 2 * g
    else:
        lo = 0 if face % 2 == 0 else n[ax] - g
    sl[ax] = slice(lo, lo + g)
    return (slice(None),) + tuple(sl)


def _sharded_fill(rank, world, name, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        c = _case(name)
        g = c.cfg.ghost
        shapes = [q.shape for q in c.qs]
        links = _topology.links(c.cfg.topology)
        owner = sharded.partition(shapes, links, world)
        s = sharded.halo_schedule(shapes, links, owner, rank, g)
        local = {b: np.array(c.qs[b]) for b in range(len(shapes)) if owner[b] == rank}
        fill = torch.zeros(max(s.fill_doubles, 1), dtype=torch.float64)
        export = torch.zeros(max(s.export_doubles, 1), dtype=torch.float64)
        # pack (the pre-exchange sources), the exchange, then unpack in link order
        for pairs, buf in ((s.pack_local, fill), (s.pack_export, export)):
            for L, o in pairs:
                t, tf, src, sf, _ = links[L]
                slab = local[src][_box(shapes[src], sf, g, True)].reshape(-1)
                buf[o:o + slab.size] = torch.from_numpy(slab.copy())
        dist.barrier()
        sharded.exchange(s, export, fill)
        for L, o in s.unpack:
            t, tf, _src, _sf, _ = links[L]
            box = _box(shapes[t], tf, g, False)
            n = local[t][box].size
            local[t][box] = fill[o:o + n].numpy().reshape(local[t][box].shape)
        out.put((rank, {b: a for b, a in local.items()}))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["tree24", "wavy4", "ragged"])
def test_two_rank_fill_matches_the_oracle(name):
    c = _case(name)
    ref = NP.halo_exchange([np.array(q) for q in c.qs], c.cfg.topology, c.cfg.ghost)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_sharded_fill, args=(r, 2, name, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        _r, blocks = q.get(timeout=180)
        got.update(blocks)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(got) == list(range(len(c.qs)))
    for b in range(len(c.qs)):
        np.testing.assert_array_equal(got[b], np.asarray(ref[b]))

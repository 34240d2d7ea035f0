"""The time step with the blocks of one topology spread over several devices
(one process per GPU, ``torch.distributed`` for the plumbing).

The reference steps every block on one device (solver/step.py:18-56) and fills
the halo once per step (solver/step.py:32, mesh/halo.py:56-92); it has no
multi-device path.  Here each rank owns some of the blocks (``partition``),
steps them with a local StepPlan, and the one halo fill per step moves the
face slabs of links that cross ranks with one grouped send/receive per peer:

  1. the step's start state is copied into the output arrays (the local
     plan then steps them in place);
  2. pack: the source slab of every link whose source block is local is
     gathered -- into the fill buffer when its target is local too, else into
     the export buffer's region for the target's rank.  All packs run before
     any ghost cell is written, so every slab holds pre-exchange values, as in
     the reference;
  3. exchange: per peer, the export region for that peer is sent and the fill
     buffer's region for that peer received (on both sides the links of a
     region are in link-list order and have the same lengths, so one message
     per direction and peer suffices);
  4. unpack: every link whose target is local is written in link-list order,
     a later link overwriting an earlier one where their ghost boxes overlap;
  5. the local plan (no links) applies the boundary conditions of its blocks
     and runs the three stages.

The slabs land in the rank's own memory before any kernel reads them (no
kernel reads a peer's memory).  The dt of a sharded run is the minimum over
the ranks (``cfl_dt``); FP32-flux plans share one pressure offset
(``StepPlan``'s p_ref: the mean pressure over all blocks), so that a sharded
step matches the step of one plan over all blocks bit for bit.
"""
from __future__ import annotations

import ctypes
import dataclasses

import torch

from famrdp_jax_b200 import _capi, _topology
from famrdp_jax_b200.core.types import BlockTopology, Config, State
from famrdp_jax_b200.solver import diagnostics
from famrdp_jax_b200.solver.step import StepPlan

ALIGN = 32  # doubles: every slab starts on a 256-byte boundary


def _cells(shape) -> int:
    n = 1
    for x in shape:
        n *= int(x)
    return n


def partition(shapes, links, world: int) -> list[int]:
    """Owner rank of every block.  Blocks go out by decreasing cell count
    (ties by index); each goes to one of the ranks whose load is within 5 % of
    the per-rank average above the least loaded one: the rank holding most
    links to the block, then the less loaded, then the lower rank.  So the
    balance comes first and, within it, cuts follow the link graph.
    ``shapes``: (ni, nj, nk) or (5, ni, nj, nk) per block."""
    if world < 1:
        raise ValueError("world must be >= 1")
    dims = [tuple(s[-3:]) for s in shapes]
    nb = len(dims)
    cells = [_cells(d) for d in dims]
    slack = 0.05 * sum(cells) / world
    nbr = [dict() for _ in range(nb)]
    for (t, _tf, s, _sf, _o) in links:
        if t != s:
            nbr[t][s] = nbr[t].get(s, 0) + 1
            nbr[s][t] = nbr[s].get(t, 0) + 1
    owner = [-1] * nb
    load = [0] * world
    for b in sorted(range(nb), key=lambda b: (-cells[b], b)):
        lo = min(load)
        cand = [r for r in range(world) if load[r] <= lo + slack]
        ties = {r: 0 for r in cand}
        for o, w in nbr[b].items():
            if owner[o] in ties:
                ties[owner[o]] += w
        best = max(cand, key=lambda r: (ties[r], -load[r], -r))
        owner[b] = best
        load[best] += cells[b]
    return owner


def _slab_doubles(shape, face: int, ghost: int) -> int:
    ext = list(shape[-3:])
    ext[face >> 1] = ghost
    return 5 * _cells(ext)


def _aligned(n: int) -> int:
    return (n + ALIGN - 1) // ALIGN * ALIGN


@dataclasses.dataclass
class HaloSchedule:
    """Where each link's slab lives on one rank (all offsets in doubles).

    pack_local:  (link, fill offset) of the links with source and target local
    pack_export: (link, export offset) of the links with a local source and a
                 target on another rank
    unpack:      (link, fill offset) of every link with a local target, in
                 link-list order
    recv / send: peer -> (offset, length) of the fill / export region that
                 peer's message fills / carries
    """
    rank: int
    pack_local: list
    pack_export: list
    unpack: list
    recv: dict
    send: dict
    fill_doubles: int
    export_doubles: int


def halo_schedule(shapes, links, owner, rank: int, ghost: int) -> HaloSchedule:
    """The rank's part of the halo fill of ``links`` (the topology's link list,
    in halo order) for the blocks placed by ``owner``."""
    dims = [tuple(s[-3:]) for s in shapes]
    world = max(owner) + 1 if owner else 1
    slab = [_slab_doubles(dims[t], tf, ghost) for (t, tf, _s, _sf, _o) in links]
    fill_off = {}
    pos = 0
    for L, (t, _tf, s, _sf, _o) in enumerate(links):
        if owner[t] == rank and owner[s] == rank:
            fill_off[L] = pos
            pos += _aligned(slab[L])
    recv = {}
    for p in range(world):
        if p == rank:
            continue
        start = pos
        for L, (t, _tf, s, _sf, _o) in enumerate(links):
            if owner[t] == rank and owner[s] == p:
                fill_off[L] = pos
                pos += _aligned(slab[L])
        if pos > start:
            recv[p] = (start, pos - start)
    fill_doubles = pos
    export = []
    send = {}
    pos = 0
    for p in range(world):
        if p == rank:
            continue
        start = pos
        for L, (t, _tf, s, _sf, _o) in enumerate(links):
            if owner[s] == rank and owner[t] == p:
                export.append((L, pos))
                pos += _aligned(slab[L])
        if pos > start:
            send[p] = (start, pos - start)
    pack_local = [(L, fill_off[L]) for L, (t, _tf, s, _sf, _o) in enumerate(links)
                  if owner[t] == rank and owner[s] == rank]
    unpack = [(L, fill_off[L]) for L, (t, _tf, _s, _sf, _o) in enumerate(links) if owner[t] == rank]
    return HaloSchedule(rank, pack_local, export, unpack, recv, send, fill_doubles, pos)


def exchange(sched: HaloSchedule, export_buf: torch.Tensor, fill_buf: torch.Tensor, group=None) -> None:
    """Step 3: one send per peer of its export region and one receive per peer
    into the fill buffer's region (torch.distributed P2P, batched so that NCCL
    runs them as one group; gloo moves CPU tensors the same way)."""
    import torch.distributed as dist
    ops = []
    for p in sorted(set(sched.send) | set(sched.recv)):
        if p in sched.send:
            o, n = sched.send[p]
            ops.append(dist.P2POp(dist.isend, export_buf[o:o + n], p, group))
        if p in sched.recv:
            o, n = sched.recv[p]
            ops.append(dist.P2POp(dist.irecv, fill_buf[o:o + n], p, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


def exchange_in_process(steps) -> None:
    """Step 3 for shards that live in one process (``steps[r]`` the
    ShardedStep of rank r, all on one device): region copies on the current
    stream, the same data movement as ``exchange``."""
    for r, st in enumerate(steps):
        for p, (o, n) in st.schedule.send.items():
            ro, rn = steps[p].schedule.recv[r]
            if rn != n:
                raise RuntimeError(f"region of ranks {r} -> {p} differs in length ({n} vs {rn})")
            steps[p].fill[ro:ro + n].copy_(st.export[o:o + n])


def local_config(cfg: Config, ids) -> Config:
    """The configuration of the blocks ``ids`` without their inter-block
    links: CUT1TO1 faces keep their type (no boundary condition) and lose their
    neighbour, so a StepPlan over these blocks applies only their boundary
    conditions; the halo is the ShardedStep's."""
    topo = tuple(BlockTopology(cfg.topology[b].block_id, {f: None for f in cfg.topology[b].neighbors},
                               dict(cfg.topology[b].bc_type)) for b in ids)
    return dataclasses.replace(cfg, topology=topo)


class ShardedStep:
    """One rank's share of a step over the topology ``cfg.topology``.

    shapes: (5, ni, nj, nk) of EVERY block of the topology; owner: rank per
    block (``partition``); local: State of this rank's blocks in increasing
    block order (their q give the shapes and device; their metrics the local
    plan's).  ``run(qs, outs, dt)`` steps the local blocks qs -> outs.  With
    ``group`` the exchange goes through torch.distributed; shards of one
    process are stepped with ``pack``, ``exchange_in_process`` and ``finish``.
    """

    def __init__(self, shapes, owner, rank: int, local: State, cfg: Config, group=None):
        self.cfg = cfg
        self.rank = rank
        self.group = group
        self.shapes = [tuple(s) for s in shapes]
        self.owner = list(owner)
        self.ids = [b for b in range(len(self.shapes)) if self.owner[b] == rank]
        if len(local.blocks) != len(self.ids):
            raise ValueError(f"rank {rank} owns {len(self.ids)} blocks, got {len(local.blocks)}")
        for b, blk in zip(self.ids, local.blocks):
            if tuple(blk.q.shape) != self.shapes[b]:
                raise ValueError(f"block {b}: shape {tuple(blk.q.shape)} differs from {self.shapes[b]}")
        self.links = _topology.links(cfg.topology)
        self.schedule = halo_schedule(self.shapes, self.links, self.owner, rank, cfg.ghost)
        self.device = local.blocks[0].q.device if local.blocks else torch.device("cpu")
        self.plan = StepPlan(local, local_config(cfg, self.ids)) if self.ids else None
        self.fill = torch.zeros(max(self.schedule.fill_doubles, 1), dtype=torch.float64, device=self.device)
        self.export = torch.zeros(max(self.schedule.export_doubles, 1), dtype=torch.float64, device=self.device)
        # the C table: every block's dimensions; q of the local ones is set per
        # call to the arrays being filled (_bind), the others stay NULL
        self._blocks = (_capi.FjBlock * len(self.shapes))()
        for b, s in enumerate(self.shapes):
            self._blocks[b].ni, self._blocks[b].nj, self._blocks[b].nk = s[1], s[2], s[3]
        self._links = _topology.link_array(self.links)

        def sel(pairs):
            n = len(pairs)
            return ((ctypes.c_int * max(n, 1))(*[L for L, _ in pairs]),
                    (ctypes.c_int64 * max(n, 1))(*[o for _, o in pairs]), n)

        self._connected = False
        self._pack_local = sel(self.schedule.pack_local)
        self._pack_export = sel(self.schedule.pack_export)
        self._unpack = sel(self.schedule.unpack)

    # -- the plan's pressure offset (FP32-flux) --------------------------------
    def p_ref(self) -> float:
        """The local plan's pressure offset (0.0 without local blocks)."""
        return self.plan.p_ref() if self.plan is not None else 0.0

    def set_p_ref(self, value: float) -> None:
        if self.plan is not None:
            self.plan.set_p_ref(value)

    def share_p_ref(self) -> float:
        """Sets every rank's offset to the cell-weighted mean of the ranks'
        offsets (an all-reduce over ``group``) and returns it."""
        import torch.distributed as dist
        cells = float(sum(_cells(self.shapes[b][1:]) for b in self.ids))
        t = torch.tensor([self.p_ref() * cells, cells], dtype=torch.float64,
                         device=self.device if self.device.type == "cuda" else "cpu")
        dist.all_reduce(t, group=self.group)
        value = float(t[0] / t[1])
        self.set_p_ref(value)
        return value

    def set_ensemble(self, mu0=None, dt=None) -> None:
        """Per-block viscosity scale and time step for independent instances
        (StepPlan.set_ensemble), given for EVERY block of the topology; each
        rank keeps its own blocks' values."""
        n = len(self.shapes)
        for name, x in (("mu0", mu0), ("dt", dt)):
            if x is not None and len(x) != n:
                raise ValueError(f"{name}: one value per block of the topology expected ({n})")
        if self.plan is not None:
            pick = (lambda x: None if x is None else [x[b] for b in self.ids])  # noqa: E731
            self.plan.set_ensemble(pick(mu0), pick(dt))

    # -- one step --------------------------------------------------------------
    def _halo_part(self, which, buf: torch.Tensor, unpack: bool) -> None:
        idx, off, n = which
        if n == 0:
            return
        c = _capi.ctx(self.device)
        fn = _capi.lib().fj_halo_unpack_f64 if unpack else _capi.lib().fj_halo_pack_f64
        name = "fj_halo_unpack_f64" if unpack else "fj_halo_pack_f64"
        _capi.check(fn(c, self._blocks, len(self.shapes), self._links, len(self.links), int(self.cfg.ghost), idx,
                       off, n, _capi.dev_ptr(buf, "slab buffer"), buf.numel(), _capi.stream(self.device)), name, c)

    def _bind(self, arrays) -> None:
        if len(arrays) != len(self.ids):
            raise ValueError(f"one state per local block expected ({len(self.ids)}), got {len(arrays)}")
        for b, a in zip(self.ids, arrays):
            if tuple(a.shape) != self.shapes[b]:
                raise ValueError(f"block {b}: shape {tuple(a.shape)} differs from {self.shapes[b]}")
            self._blocks[b].q = _capi.dev_ptr(a, f"state[{b}]")

    def pack(self, qs, outs) -> None:
        """Steps 1-2: qs (the local blocks' start states) into outs and every
        locally sourced slab into the fill or export buffer."""
        self._bind(outs)
        for o, q in zip(outs, qs):
            if o.data_ptr() != q.data_ptr():
                o.copy_(q)
        self._halo_part(self._pack_local, self.fill, False)
        self._halo_part(self._pack_export, self.export, False)

    def finish(self, outs, dt: float, graph: bool = False) -> None:
        """Steps 4-5: the ghost slabs of the local blocks (outs, as left by
        ``pack``), then the local plan's boundary conditions and stages, in
        place on outs."""
        self._bind(outs)
        self._halo_part(self._unpack, self.fill, True)
        if self.plan is not None:
            self.plan.run(outs, outs, dt, graph=graph)

    def run(self, qs, outs, dt: float, graph: bool = False) -> None:
        """One step of the local blocks, exchanging with the other ranks of
        ``group`` (every rank of the group calls it once per step)."""
        if not self._connected:
            # the first batched P2P call of a NCCL group must involve all of its
            # ranks: a barrier first sets up the communicator on every rank
            import torch.distributed as dist
            dist.barrier(group=self.group)
            self._connected = True
        self.pack(qs, outs)
        exchange(self.schedule, self.export, self.fill, self.group)
        self.finish(outs, dt, graph=graph)


def cfl_dt(local: State, cfg: Config, cfl: float | None = None, group=None) -> float:
    """The CFL time step of the whole topology: each rank's minimum over its
    blocks, then the minimum over the ranks (an all-reduce)."""
    import torch.distributed as dist
    dt = diagnostics.cfl_dt(local, cfg, cfl) if local.blocks else float("inf")
    return _all_reduce([dt], local, group, dist.ReduceOp.MIN)[0]


def _all_reduce(values, local: State, group, op=None):
    import torch.distributed as dist
    dev = local.blocks[0].q.device if local.blocks else torch.device("cpu")
    t = torch.tensor(values, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM if op is None else op, group=group)
    return t.tolist()


def kinetic_energy(local: State, ghost: int = 2, group=None) -> float:
    """J over the whole topology: the ranks' sums over their blocks' interior
    cells, added (an all-reduce)."""
    j = diagnostics.kinetic_energy(local, ghost) if local.blocks else 0.0
    return _all_reduce([j], local, group)[0]


def residual(local: State, prev, dt: float, ghost: int = 2, group=None) -> list[float]:
    """diagnostics.residual over the whole topology: each rank's per-component
    RMS weighted by its interior cells, combined (an all-reduce)."""
    n = float(sum((b.q.shape[1] - 2 * ghost) * (b.q.shape[2] - 2 * ghost) * (b.q.shape[3] - 2 * ghost)
                  for b in local.blocks))
    r = diagnostics.residual(local, prev, dt, ghost) if local.blocks else [0.0] * 5
    tot = _all_reduce([x * x * n for x in r] + [n], local, group)
    return [(x / tot[5]) ** 0.5 for x in tot[:5]]


def shard_state(state: State, owner, rank: int) -> State:
    """The blocks (and metrics) of ``state`` that ``owner`` gives ``rank``."""
    ids = [b for b in range(len(state.blocks)) if owner[b] == rank]
    return State(blocks=tuple(state.blocks[b] for b in ids), metrics=tuple(state.metrics[b] for b in ids),
                 t=state.t, step=state.step)


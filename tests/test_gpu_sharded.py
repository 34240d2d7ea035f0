"""Block sharding on the GPU: the blocks of a topology split over 2-4 shards
that live in one process (one device; the exchange is ``exchange_in_process``,
the same data movement as the NCCL send/receive of a multi-GPU run) step
exactly like one plan over all blocks -- bit for bit in FP64 and, with the
shared pressure offset, in FP32-flux -- for periodic curvilinear blocks,
uneven trees with farfield faces, ragged blocks and links in mapped
orientations.  Also: the pack/unpack entry points' refusals and the
torch.distributed path with a one-rank NCCL group."""
import ctypes
import dataclasses
import datetime
import socket

import pytest
import torch

from famrdp_jax_b200 import _capi, _topology, cases
from famrdp_jax_b200.solver import diagnostics, sharded
from famrdp_jax_b200.solver.step import StepPlan
from oracle.ref import NP

pytestmark = pytest.mark.gpu


def _case(name, precision, dev):
    if name == "box":
        from test_gpu_orientation import RELABELS, _box, _cfg, _state
        qs, mets, topos = _box(*RELABELS[3])  # the second block in mapped orientations
        return _state(qs, mets), _cfg(topos, precision), 0.3
    if name == "wavy4":
        c = cases.wavy4(n=12, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2))
    elif name == "tree24":
        c = cases.tree24(nblocks=24, lo=6, hi=14, seed=3)
    elif name == "ragged":
        c = cases.tree24(nblocks=5, lo=3, hi=23, seed=7)
    else:
        raise KeyError(name)
    return cases.to_state(c, dev), dataclasses.replace(c.cfg, precision=precision), c.cfl


def _shards(state, cfg, world):
    shapes = [tuple(b.q.shape) for b in state.blocks]
    owner = sharded.partition(shapes, _topology.links(cfg.topology), world)
    steps = [sharded.ShardedStep(shapes, owner, r, sharded.shard_state(state, owner, r), cfg)
             for r in range(world)]
    return owner, steps


@pytest.mark.parametrize("name,world", [("wavy4", 2), ("wavy4", 4), ("tree24", 2), ("tree24", 3),
                                        ("ragged", 2), ("box", 2)])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_sharded_steps_match_one_plan(cuda_device, name, world, precision):
    state, cfg, cfl = _case(name, precision, cuda_device)
    dt = diagnostics.cfl_dt(state, cfg, cfl)
    full = StepPlan(state, cfg)
    owner, steps = _shards(state, cfg, world)
    assert len(set(owner)) > 1  # links do cross shards
    for s in steps:
        s.set_p_ref(full.p_ref())
    qa = [b.q.clone() for b in state.blocks]
    qb = [torch.empty_like(q) for q in qa]
    sa = [[qa[b].clone() for b in s.ids] for s in steps]
    sb = [[torch.empty_like(q) for q in x] for x in sa]
    for n in range(3):
        full.run(qa, qb, dt)
        qa, qb = qb, qa
        for s, x, y in zip(steps, sa, sb):
            s.pack(x, y)
        sharded.exchange_in_process(steps)
        for s, y in zip(steps, sb):
            s.finish(y, dt, graph=n > 0)
        sa, sb = sb, sa
        for s, x in zip(steps, sa):
            for b, q in zip(s.ids, x):
                assert torch.equal(q, qa[b]), (name, world, precision, n, b)
    assert not torch.equal(qa[0], state.blocks[0].q)  # the state did evolve


def test_shared_pressure_offset_is_the_plans(cuda_device):
    state, cfg, _ = _case("tree24", "f32", cuda_device)
    full = StepPlan(state, cfg)
    _, steps = _shards(state, cfg, 3)
    assert full.p_ref() != 0.0
    assert all(s.p_ref() != full.p_ref() for s in steps)  # each shard's own mean differs
    for s in steps:
        s.set_p_ref(full.p_ref())
    assert all(s.p_ref() == full.p_ref() for s in steps)
    assert StepPlan(*_case("tree24", "f64", cuda_device)[:2]).p_ref() == 0.0
    with pytest.raises(ValueError):
        full.set_p_ref(float("nan"))


def test_pack_and_unpack_refuse_what_they_cannot_do(cuda_device):
    state, cfg, _ = _case("wavy4", "f64", cuda_device)
    links = _topology.links(cfg.topology)
    blocks = _topology.block_array([b.q for b in state.blocks])
    blocks[links[0][0]].q = None  # the first link's target is not on this device
    buf = torch.zeros(1 << 16, dtype=torch.float64, device=cuda_device)
    c = _capi.ctx(cuda_device)
    la = _topology.link_array(links)
    sel = (ctypes.c_int * 1)(0)
    off = (ctypes.c_int64 * 1)(0)
    lib = _capi.lib()
    args = (c, blocks, len(state.blocks), la, len(links), 2, sel, off, 1, _capi.dev_ptr(buf, "buf"))
    assert lib.fj_halo_unpack_f64(*args, buf.numel(), None) == _capi.FJ_ERR_INVALID_ARGUMENT
    assert lib.fj_halo_pack_f64(*args, 10, None) == _capi.FJ_ERR_INVALID_ARGUMENT  # slab outside the buffer
    off[0] = -32
    assert lib.fj_halo_pack_f64(*args, buf.numel(), None) == _capi.FJ_ERR_INVALID_ARGUMENT
    sel[0] = len(links)
    off[0] = 0
    assert lib.fj_halo_pack_f64(*args, buf.numel(), None) == _capi.FJ_ERR_INVALID_ARGUMENT
    sel[0] = 0
    src = links[0][2]
    if blocks[src].q:  # the source is set: packing works
        assert lib.fj_halo_pack_f64(*args, buf.numel(), None) == _capi.FJ_OK
    torch.cuda.synchronize()


def test_sharded_run_through_a_process_group(cuda_device):
    """ShardedStep.run and sharded.cfl_dt over a one-rank NCCL group: the
    collective path without peers (a multi-GPU run adds one send and one
    receive per peer)."""
    import torch.distributed as dist
    state, cfg, cfl = _case("wavy4", "f64", cuda_device)
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=cuda_device)
    try:
        dt = sharded.cfl_dt(state, cfg, cfl)
        assert dt == diagnostics.cfl_dt(state, cfg, cfl)
        shapes = [tuple(b.q.shape) for b in state.blocks]
        owner = sharded.partition(shapes, _topology.links(cfg.topology), 1)
        st = sharded.ShardedStep(shapes, owner, 0, state, cfg)
        full = StepPlan(state, cfg)
        assert st.share_p_ref() == full.p_ref()
        qa = [b.q.clone() for b in state.blocks]
        qb = [torch.empty_like(q) for q in qa]
        sa = [q.clone() for q in qa]
        sb = [torch.empty_like(q) for q in qa]
        for _ in range(2):
            full.run(qa, qb, dt)
            st.run(sa, sb, dt)
            qa, qb, sa, sb = qb, qa, sb, sa
        torch.cuda.synchronize()
        assert all(torch.equal(a, b) for a, b in zip(sa, qa))
        done = sharded.shard_state(dataclasses.replace(state, blocks=tuple(
            dataclasses.replace(b, q=q) for b, q in zip(state.blocks, sa))), owner, 0)
        assert sharded.kinetic_energy(done) == diagnostics.kinetic_energy(done)
        res = sharded.residual(done, sb, dt)
        ref = diagnostics.residual(done, sb, dt)
        assert all(abs(a - b) <= 1e-12 * abs(b) for a, b in zip(res, ref)) and max(ref) > 0
    finally:
        dist.destroy_process_group()


def test_sharded_ensemble_matches_one_plan(cuda_device):
    """Independent instances (each block its own mu0 and dt, no links between
    blocks) spread over three shards step like one plan over all of them."""
    from famrdp_jax_b200.core.types import State
    c = cases.ensemble(ninst=7, n=10, seed=2)
    state = cases.to_state(c, cuda_device)
    cfg = c.cfg
    mu0 = c.meta["mu0"]
    dts = [diagnostics.cfl_dt(State(blocks=(b,), metrics=(m,)), cfg, c.cfl)
           for b, m in zip(state.blocks, state.metrics)]
    full = StepPlan(state, cfg)
    full.set_ensemble(mu0, dts)
    _, steps = _shards(state, cfg, 3)
    assert cfg.precision == "f32"
    for s in steps:
        s.set_ensemble(mu0, dts)
        s.set_p_ref(full.p_ref())
        assert not s.schedule.send and not s.schedule.recv  # nothing crosses shards
    with pytest.raises(ValueError):
        steps[0].set_ensemble(mu0[:-1], None)
    qa = [b.q.clone() for b in state.blocks]
    qb = [torch.empty_like(q) for q in qa]
    sa = [[qa[b].clone() for b in s.ids] for s in steps]
    sb = [[torch.empty_like(q) for q in x] for x in sa]
    for _ in range(3):
        full.run(qa, qb, 0.0)
        qa, qb = qb, qa
        for s, x, y in zip(steps, sa, sb):
            s.pack(x, y)
        sharded.exchange_in_process(steps)
        for s, y in zip(steps, sb):
            s.finish(y, 0.0)
        sa, sb = sb, sa
    for s, x in zip(steps, sa):
        for b, q in zip(s.ids, x):
            assert torch.equal(q, qa[b]), b

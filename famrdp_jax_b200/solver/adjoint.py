"""Hand-written adjoint of the RHS and of the TVD-RK3 step, with checkpointed
reverse sweeps, exposed to torch.autograd.

The reference differentiates ``step`` with ``jax.grad`` (tests/solver/
test_grad.py:30-35): reverse-mode AD through every jnp operation of every
step, storing everything.  Here the reverse mode is written by hand in CUDA
(``fj_rhs_vjp_f64``, ``fj_step_vjp_f64``) and the trajectory keeps only one
state every ``checkpoint_every`` steps: the reverse sweep recomputes each
segment's states from its checkpoint and runs the step adjoints backwards
through it.

    qN = integrate(state, cfg, dt, nsteps, checkpoint_every=10)   # differentiable
    J = kinetic_energy(State(qN...)) ...; J.backward()

or, without torch autograd,

    J, dJ_dq0, dJ_dmu0 = adjoint_kinetic_energy(state, cfg, dt, nsteps, 10)
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from famrdp_jax_b200 import _capi, _topology
from famrdp_jax_b200.core.types import Block, Config, Metrics, State
from famrdp_jax_b200.solver.step import StepPlan, _params


def rhs_vjp(q: torch.Tensor, metrics: Metrics, cfg: Config, lam: torch.Tensor) -> torch.Tensor:
    """(dL/dq)^T lam for one block, L = _rhs_block (solver/step.py:10-15)."""
    p = _params(cfg)
    out = torch.empty_like(q)
    ni, nj, nk = q.shape[1:]
    c = _capi.ctx(q.device)
    _capi.check(_capi.lib().fj_rhs_vjp_f64(c, _capi.dev_ptr(q, "q"), _capi.dev_ptr(metrics.kxyz, "kxyz"),
                                           _capi.dev_ptr(metrics.vol, "vol"), _capi.dev_ptr(lam.contiguous(), "lam"),
                                           _capi.dev_ptr(out, "out"), ni, nj, nk, p, _capi.stream(q.device)),
                "fj_rhs_vjp_f64", c)
    return out


class _Tables:
    """Link / boundary tables of a configuration, marshalled once."""

    def __init__(self, cfg: Config):
        self.params = _params(cfg)
        self.links = _topology.links(cfg.topology)
        self.bcs = _topology.bcs(cfg.topology, cfg)
        self.link_arr = _topology.link_array(self.links)
        self.bc_arr = _topology.bc_array(self.bcs)


def step_vjp(qs, metrics, cfg: Config, dt: float, lams, *, tables: _Tables | None = None,
             dmu: torch.Tensor | None = None):
    """dJ/dq of one step's input from dJ/dq_new (lists over blocks).  When a
    one-element float64 CUDA tensor ``dmu`` is given, dJ/dmu0 of this step is
    added to it."""
    t = tables or _Tables(cfg)
    dev = qs[0].device
    c = _capi.ctx(dev)
    outs = [torch.empty_like(q) for q in qs]
    lam_c = [l.contiguous() for l in lams]
    lam_in = (ctypes.c_void_p * len(qs))(*[_capi.dev_ptr(l, "lam") for l in lam_c])
    blocks = _topology.block_array(list(qs), metrics)
    if dmu is None:
        st = _capi.lib().fj_step_vjp_f64(c, blocks, lam_in, _topology.ptr_array(outs), len(qs), t.link_arr,
                                         len(t.links), t.bc_arr, len(t.bcs), t.params, float(dt), _capi.stream(dev))
        _capi.check(st, "fj_step_vjp_f64", c)
    else:
        st = _capi.lib().fj_step_vjp_mu_f64(c, blocks, lam_in, _topology.ptr_array(outs), len(qs), t.link_arr,
                                            len(t.links), t.bc_arr, len(t.bcs), t.params, float(dt),
                                            _capi.dev_ptr(dmu, "dmu"), _capi.stream(dev))
        _capi.check(st, "fj_step_vjp_mu_f64", c)
    return outs


def step_vjp_saved(saved, metrics, cfg: Config, dt: float, lams, *, tables: _Tables | None = None,
                   dmu: torch.Tensor | None = None):
    """step_vjp on the states a StepPlan.run_save kept: saved = (q0s, q1s, q2s)
    with q0s the halo-filled start states; the step's forward is not rerun."""
    t = tables or _Tables(cfg)
    q0s, q1s, q2s = saved
    dev = q0s[0].device
    c = _capi.ctx(dev)
    outs = [torch.empty_like(q) for q in q0s]
    lam_c = [l.contiguous() for l in lams]
    lam_in = (ctypes.c_void_p * len(q0s))(*[_capi.dev_ptr(l, "lam") for l in lam_c])
    blocks = _topology.block_array(list(q0s), metrics)
    pa = _topology.ptr_array
    st = _capi.lib().fj_step_vjp_saved_f64(c, blocks, pa(q1s), pa(q2s), lam_in, pa(outs), len(q0s), t.link_arr,
                                           len(t.links), t.bc_arr, len(t.bcs), t.params, float(dt),
                                           _capi.dev_ptr(dmu, "dmu") if dmu is not None else None,
                                           _capi.stream(dev))
    _capi.check(st, "fj_step_vjp_saved_f64", c)
    return outs


def kinetic_energy_grad(qs, metrics, ghost: int = 2):
    """dJ/dq of J = sum over interior cells of vol * 0.5 |rho u|^2 / rho."""
    dev = qs[0].device
    c = _capi.ctx(dev)
    grads = [torch.empty_like(q) for q in qs]
    _capi.check(_capi.lib().fj_kinetic_energy_grad_f64(c, _topology.block_array(list(qs), metrics),
                                                       _topology.ptr_array(grads), len(qs), int(ghost),
                                                       _capi.stream(dev)), "fj_kinetic_energy_grad_f64", c)
    return grads


def _forward_segment(plan: StepPlan, qs, dt, nsteps, keep: bool):
    """nsteps steps from qs; returns the final state and, if keep, each step's
    saved intermediate states (halo-filled start state, stage 1 and 2)."""
    states = []
    cur = list(qs)
    for _ in range(nsteps):
        nxt = [torch.empty_like(q) for q in cur]
        if keep:
            saved = tuple([torch.empty_like(q) for q in cur] for _ in range(3))
            plan.run_save(cur, nxt, *saved, dt)
            states.append(saved)
        else:
            plan.run(cur, nxt, dt)
        cur = nxt
    return cur, states


@dataclass
class _Run:
    cfg: Config
    metrics: tuple
    dt: float
    nsteps: int
    every: int
    plan: StepPlan
    tables: _Tables
    dmu: torch.Tensor | None = None


def _reverse_sweep(run: _Run, checkpoints, lams):
    """Segments in reverse: recompute the segment's states from its checkpoint
    (keeping each step's stage states), then apply the step adjoints
    backwards, releasing each step's states once its adjoint has run."""
    nseg = len(checkpoints)
    for s in reversed(range(nseg)):
        seg_len = min(run.every, run.nsteps - s * run.every)
        _, states = _forward_segment(run.plan, checkpoints[s], run.dt, seg_len, keep=True)
        while states:
            lams = step_vjp_saved(states.pop(), run.metrics, run.cfg, run.dt, lams, tables=run.tables, dmu=run.dmu)
    return lams


def _forward_with_checkpoints(run: _Run, q0s):
    checkpoints = []
    cur = [q.detach() for q in q0s]
    done = 0
    while done < run.nsteps:
        checkpoints.append([q.clone() for q in cur])
        n = min(run.every, run.nsteps - done)
        cur, _ = _forward_segment(run.plan, cur, run.dt, n, keep=False)
        done += n
    return cur, checkpoints


class _Trajectory(torch.autograd.Function):
    @staticmethod
    def forward(ctx, run: _Run, *q0s):
        final, checkpoints = _forward_with_checkpoints(run, q0s)
        ctx.run = run
        ctx.checkpoints = checkpoints
        return tuple(final)

    @staticmethod
    def backward(ctx, *grads):
        lams = [g if g is not None else None for g in grads]
        run: _Run = ctx.run
        lams = [l if l is not None else torch.zeros_like(c) for l, c in zip(lams, ctx.checkpoints[0])]
        out = _reverse_sweep(run, ctx.checkpoints, lams)
        return (None, *out)


def integrate(state: State, cfg: Config, dt: float, nsteps: int, *, checkpoint_every: int = 10,
              plan: StepPlan | None = None) -> State:
    """nsteps TVD-RK3 steps, differentiable with respect to the blocks' q
    through the hand-written adjoint (one checkpoint every checkpoint_every
    steps, recomputation in the reverse sweep)."""
    plan = plan or StepPlan(state, cfg)
    run = _Run(cfg=cfg, metrics=state.metrics, dt=float(dt), nsteps=int(nsteps), every=max(1, int(checkpoint_every)),
               plan=plan, tables=_Tables(cfg))
    final = _Trajectory.apply(run, *[b.q for b in state.blocks])
    blocks = tuple(Block(q=q, xyz=b.xyz) for q, b in zip(final, state.blocks))
    return State(blocks=blocks, metrics=state.metrics, t=state.t + nsteps * dt, step=state.step + nsteps)


def adjoint_kinetic_energy(state: State, cfg: Config, dt: float, nsteps: int, checkpoint_every: int = 10,
                           plan: StepPlan | None = None):
    """(J, dJ/dq0 per block, dJ/dmu0) for J = the interior kinetic-energy
    integral after nsteps steps, by the checkpointed adjoint."""
    from famrdp_jax_b200.solver import diagnostics

    plan = plan or StepPlan(state, cfg)
    dev = state.blocks[0].q.device
    dmu = torch.zeros(1, dtype=torch.float64, device=dev)
    run = _Run(cfg=cfg, metrics=state.metrics, dt=float(dt), nsteps=int(nsteps), every=max(1, int(checkpoint_every)),
               plan=plan, tables=_Tables(cfg), dmu=dmu)
    final, checkpoints = _forward_with_checkpoints(run, [b.q for b in state.blocks])
    fstate = State(blocks=tuple(Block(q=q, xyz=b.xyz) for q, b in zip(final, state.blocks)), metrics=state.metrics)
    J = diagnostics.kinetic_energy(fstate, cfg.ghost)
    lams = kinetic_energy_grad(final, state.metrics, cfg.ghost)
    grads = _reverse_sweep(run, checkpoints, lams)
    return J, grads, float(dmu.item())

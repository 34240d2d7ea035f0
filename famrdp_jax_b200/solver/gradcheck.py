"""Central-difference check of the checkpointed adjoint of the kinetic-energy
objective (the reference's gradient test, tests/solver/test_grad.py:30-35,
takes jax.grad of ``step``; here the hand-written adjoint is checked against
central differences of the forward steps on the same device).

For seeded random directions d of unit L2 norm over the initial state,
    fd(d) = (J(q0 + eps d) - J(q0 - eps d)) / (2 eps)   and   ad(d) = <dJ/dq0, d>,
and two errors are reported per direction:
  * rel_direction = |fd - ad| / |ad|  -- the directional derivative's own
    relative error; for a random direction in a space of n values |ad| is
    about |grad J| / sqrt(n), so FP64 rounding of J (about 1e-16 J / eps)
    dominates it on large states;
  * rel_gradnorm  = |fd - ad| / |grad J| -- the same error against the
    derivative's bound for a unit direction.
The gradient direction itself (d = g / |g|, where fd should equal |g|) and
dJ/dmu0 (central differences in mu0 with step eps_mu * mu0) are checked too.
eps_mu defaults to 1e-3: J moves by about 2 eps_mu mu0 |dJ/dmu0| between the
two evaluations, and at 1e-6 that is within a few thousand FP64 roundings of
J on a 96^3 block over 50 steps (measured: a 2.3e-5 relative error that is
rounding, not the adjoint); J depends smoothly on mu0 (the viscous RHS is
linear in it), so the larger step costs no measurable truncation error.
J is only piecewise smooth (minmod switches where two slopes have equal
magnitude or a slope changes sign): a +-eps perturbation that crosses one of
those points biases fd, so single directions can disagree at any eps.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import torch

from famrdp_jax_b200.core.types import Block, State
from famrdp_jax_b200.solver import adjoint, diagnostics
from famrdp_jax_b200.solver.step import StepPlan


def _objective(plan: StepPlan, state: State, q0s, nsteps: int, dt: float, ghost: int, bufs) -> float:
    a = [q.clone() for q in q0s]
    b = bufs
    for _ in range(nsteps):
        plan.run(a, b, dt)
        a, b = b, a
    fs = State(blocks=tuple(Block(q=q, xyz=bl.xyz) for q, bl in zip(a, state.blocks)), metrics=state.metrics)
    return diagnostics.kinetic_energy(fs, ghost)


def fd_check_kinetic_energy(state: State, cfg, dt: float, nsteps: int, *, checkpoint_every: int = 10,
                            eps: float = 1e-6, ndirs: int = 16, seed: int = 0, eps_mu: float = 1e-3) -> dict:
    """Adjoint gradient of J = interior kinetic energy after nsteps steps
    against central differences; returns the per-direction errors and their
    maxima (see the module docstring)."""
    plan = StepPlan(state, cfg)
    J, grads, dmu = adjoint.adjoint_kinetic_energy(state, cfg, dt, nsteps, checkpoint_every=checkpoint_every,
                                                   plan=plan)
    q0s = [b.q for b in state.blocks]
    bufs = [torch.empty_like(q) for q in q0s]
    gnorm = math.sqrt(sum(float(torch.sum(g * g)) for g in grads))
    rng = np.random.default_rng(seed)

    def J_at(qs, p=plan):
        return _objective(p, state, qs, nsteps, dt, cfg.ghost, bufs)

    rows = []
    for _ in range(ndirs):
        ds = [torch.tensor(rng.standard_normal(tuple(q.shape)), dtype=torch.float64, device=q.device) for q in q0s]
        nrm = math.sqrt(sum(float(torch.sum(d * d)) for d in ds))
        ds = [d / nrm for d in ds]
        fd = (J_at([q + eps * d for q, d in zip(q0s, ds)]) - J_at([q - eps * d for q, d in zip(q0s, ds)])) / (2 * eps)
        ad = sum(float(torch.sum(g * d)) for g, d in zip(grads, ds))
        rows.append({"fd": fd, "ad": ad, "rel_direction": abs(fd - ad) / max(abs(ad), 1e-300),
                     "rel_gradnorm": abs(fd - ad) / gnorm})
    ds = [g / gnorm for g in grads]
    fd_g = (J_at([q + eps * d for q, d in zip(q0s, ds)]) - J_at([q - eps * d for q, d in zip(q0s, ds)])) / (2 * eps)
    h = eps_mu * cfg.gas.mu0
    fd_mu = []
    for s in (1.0, -1.0):
        c2 = dataclasses.replace(cfg, gas=dataclasses.replace(cfg.gas, mu0=cfg.gas.mu0 + s * h))
        fd_mu.append(J_at(q0s, StepPlan(state, c2)))
    fd_mu = (fd_mu[0] - fd_mu[1]) / (2 * h)
    return {"J": J, "grad_norm": gnorm, "eps": eps, "directions": ndirs, "seed": seed,
            "max_rel_direction": max(r["rel_direction"] for r in rows),
            "median_rel_direction": float(np.median([r["rel_direction"] for r in rows])),
            "max_rel_gradnorm": max(r["rel_gradnorm"] for r in rows),
            "gradient_direction_rel": abs(fd_g - gnorm) / gnorm,
            "dJ_dmu0": dmu, "dJ_dmu0_fd": fd_mu, "dJ_dmu0_rel": abs(fd_mu - dmu) / max(abs(dmu), 1e-300),
            "per_direction": rows}

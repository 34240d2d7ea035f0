"""A monitored time loop: fixed-dt TVD-RK3 steps with the state check and the
per-step residual log the reference plans (docs/requirements.md FR-61, FR-63,
NFR-31) but does not have; its Config.nan_check (core/types.py:187) is read
here.

    state, log = run(state, cfg, dt, nsteps, residual_every=1)
    write_residual_log("res.txt", log)

After every ``check_every`` steps (when cfg.nan_check) the state is checked
for non-finite values and non-positive density or pressure; on failure the
state before the failing step (the last good one when check_every is 1) and
the failing one are saved under ``dump_dir`` (when given) and
FloatingPointError names the step.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import torch

from famrdp_jax_b200.core.types import Block, Config, State
from famrdp_jax_b200.solver import diagnostics
from famrdp_jax_b200.solver.step import StepPlan


@dataclass
class ResidualLog:
    """One row per logged step: (step, t, [res rho, rho u, rho v, rho w, rho E])."""
    rows: list = field(default_factory=list)


def _dump(dump_dir, name, qs):
    d = Path(dump_dir)
    d.mkdir(parents=True, exist_ok=True)
    torch.save([q.detach().cpu() for q in qs], d / name)


def run(state: State, cfg: Config, dt: float, nsteps: int, *, plan: StepPlan | None = None, check_every: int = 1,
        residual_every: int = 1, graph: bool = True, dump_dir=None):
    """nsteps steps of fixed dt; returns (final State, ResidualLog)."""
    plan = plan or StepPlan(state, cfg)
    a = [b.q.clone() for b in state.blocks]
    b = [torch.empty_like(q) for q in a]
    log = ResidualLog()
    g = cfg.ghost
    for n in range(1, nsteps + 1):
        plan.run(a, b, dt, graph=graph)
        cur = State(blocks=tuple(Block(q=q, xyz=s.xyz) for q, s in zip(b, state.blocks)), metrics=state.metrics)
        if residual_every and n % residual_every == 0:
            log.rows.append((state.step + n, state.t + n * dt, diagnostics.residual(cur, a, dt, g)))
        if cfg.nan_check and check_every and n % check_every == 0:
            nonfinite, rmin, pmin = diagnostics.check_state(cur, cfg.gas.gamma, raise_on_error=False)
            if nonfinite or not (rmin > 0.0) or not (pmin > 0.0):
                if dump_dir is not None:
                    _dump(dump_dir, f"step{state.step + n - 1:07d}_good.pt", a)
                    _dump(dump_dir, f"step{state.step + n:07d}_bad.pt", b)
                raise FloatingPointError(f"step {state.step + n}: {nonfinite} non-finite values, "
                                         f"min rho {rmin:.3e}, min p {pmin:.3e}")
        a, b = b, a
    final = State(blocks=tuple(Block(q=q, xyz=s.xyz) for q, s in zip(a, state.blocks)), metrics=state.metrics,
                  t=state.t + nsteps * dt, step=state.step + nsteps)
    return final, log


def write_residual_log(path, log: ResidualLog) -> None:
    """Text table: step, t and the five residuals, one line per logged step."""
    lines = ["# step t res_rho res_rhou res_rhov res_rhow res_rhoE"]
    for step, t, r in log.rows:
        lines.append(f"{step:8d} {t:.10e} " + " ".join(f"{x:.10e}" for x in r))
    Path(path).write_text("\n".join(lines) + "\n")

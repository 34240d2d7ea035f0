"""The time step (famrdp_jax ``solver/step.py``) on the GPU.

``step(state, cfg, dt)`` keeps the reference's signature and semantics: halo
fill and boundary conditions once per step, then three Shu-Osher TVD-RK3
stages over all padded cells of every block, returning a new State with
t + dt and step + 1 (the input state is not modified).  The step runs through
a prepared plan (fj_plan_*: tables, FP32 metric records and scratch built
once); step() keeps the plans of the last few (block layout, metrics, cfg)
combinations it saw, so a time loop of step() calls prepares one plan.  The
metrics are constants of a plan: arrays changed in place after a step() call
need a new Metrics object (or an explicit StepPlan).
"""
from __future__ import annotations

import ctypes

import torch

from famrdp_jax_b200 import _capi, _topology
from famrdp_jax_b200.core.types import Block, Config, Metrics, State


def _params(cfg: Config):
    return _capi.params(cfg.gas, limiter=cfg.scheme.limiter, ghost=cfg.ghost,
                        precision=getattr(cfg, "precision", "f64"))


def _rhs_block(q: torch.Tensor, metrics: Metrics, cfg: Config) -> torch.Tensor:
    """Inviscid + viscous RHS of one block (solver/step.py:10-15)."""
    p = _params(cfg)
    rhs = torch.empty_like(q)
    ni, nj, nk = q.shape[1:]
    c = _capi.ctx(q.device)
    _capi.check(_capi.lib().fj_rhs_f64(c, _capi.dev_ptr(q, "q"), _capi.dev_ptr(metrics.kxyz, "kxyz"),
                                       _capi.dev_ptr(metrics.vol, "vol"), _capi.dev_ptr(rhs, "rhs"),
                                       ni, nj, nk, p, _capi.stream(q.device)), "fj_rhs_f64", c)
    return rhs


def rk_stage(q: torch.Tensor, q0: torch.Tensor | None, metrics: Metrics, cfg: Config, dt: float,
             stage: int, out: torch.Tensor | None = None) -> torch.Tensor:
    """One TVD-RK3 stage of one block, RHS and combine in one call
    (solver/step.py:45-53 without the halo fill).  ``out`` may be ``q0``."""
    p = _params(cfg)
    out = torch.empty_like(q) if out is None else out
    ni, nj, nk = q.shape[1:]
    c = _capi.ctx(q.device)
    q0p = _capi.dev_ptr(q0, "q0") if q0 is not None else None
    _capi.check(_capi.lib().fj_rk_stage_f64(c, _capi.dev_ptr(q, "q"), q0p, _capi.dev_ptr(metrics.kxyz, "kxyz"),
                                            _capi.dev_ptr(metrics.vol, "vol"), _capi.dev_ptr(out, "out"),
                                            ni, nj, nk, p, float(dt), int(stage), _capi.stream(q.device)),
                "fj_rk_stage_f64", c)
    return out


class StepPlan:
    """A prepared step (fj_plan) for one (block layout, metrics, cfg): tables
    checked and uploaded once, FP32 metric copies built once for the FP32-flux
    precision, scratch owned by the plan.  Reusable while the metrics and block
    shapes stay the same."""

    def __init__(self, state: State, cfg: Config):
        if len(state.blocks) != len(cfg.topology):
            raise ValueError("state.blocks and cfg.topology differ in length")
        self.cfg = cfg
        self.params = _params(cfg)
        self.links = _topology.links(cfg.topology)
        self.bcs = _topology.bcs(cfg.topology, cfg)
        self.metrics = state.metrics
        self.device = state.blocks[0].q.device
        self.shapes = [tuple(b.q.shape) for b in state.blocks]
        self._handle = None
        c = _capi.ctx(self.device)
        blocks = _topology.block_array([b.q for b in state.blocks], self.metrics)
        h = ctypes.c_void_p()
        _capi.check(_capi.lib().fj_plan_create(c, blocks, len(state.blocks), _topology.link_array(self.links),
                                               len(self.links), _topology.bc_array(self.bcs), len(self.bcs),
                                               self.params, ctypes.byref(h)), "fj_plan_create", c)
        self._handle = h.value
        self._lib = _capi.lib()
        self.mu0s = None
        self.dts = None

    def run(self, qs, outs, dt: float, graph: bool = False) -> None:
        """One step qs -> outs.  With graph=True the step is captured once per
        (qs, outs, dt) pointer set as a CUDA graph and replayed afterwards
        (use fixed ping-pong buffers)."""
        if [tuple(q.shape) for q in qs] != self.shapes or [tuple(o.shape) for o in outs] != self.shapes:
            raise ValueError("state shapes differ from the plan's")
        c = _capi.ctx(self.device)
        fn = self._lib.fj_plan_step_graph if graph else self._lib.fj_plan_step
        _capi.check(fn(self._handle, _topology.ptr_array(qs), _topology.ptr_array(outs), float(dt),
                       _capi.stream(self.device)), "fj_plan_step_graph" if graph else "fj_plan_step", c)

    def p_ref(self) -> float:
        """The FP32-flux pressure offset (the mean pressure over the plan's
        padded cells at creation; 0.0 on FP64 plans)."""
        out = ctypes.c_double()
        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_p_ref(self._handle, ctypes.byref(out)), "fj_plan_p_ref", c)
        return out.value

    def set_p_ref(self, value: float) -> None:
        """Sets the FP32-flux pressure offset (changes only the rounding of
        FP32-flux results; plans of the shards of one topology share one)."""
        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_set_p_ref(self._handle, float(value)), "fj_plan_set_p_ref", c)

    def set_ensemble(self, mu0=None, dt=None) -> None:
        """Per-block viscosity scale and time step (independent instances):
        block b then uses mu0[b] and dt[b], and the dt argument of run/stage is
        ignored while dt is set.  None restores the plan-wide value."""
        n = len(self.shapes)

        def arr(x):
            if x is None:
                return None
            if len(x) != n:
                raise ValueError("one value per block expected")
            return (ctypes.c_double * n)(*[float(v) for v in x])

        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_set_ensemble(self._handle, arr(mu0), arr(dt)), "fj_plan_set_ensemble", c)
        self.mu0s = None if mu0 is None else [float(v) for v in mu0]
        self.dts = None if dt is None else [float(v) for v in dt]

    def autotune(self, qs, outs, dt: float, reps: int = 3):
        """Times every launch shape of the split kernels and both stream
        counts and, on FP32-flux plans, the fused tile kernel and the
        persistent step in each of its shapes, over `reps` steps qs -> outs
        (outs is overwritten) and keeps the fastest; returns (chosen, mean step
        ms per candidate), the candidate index being shape +
        NUM_SPLIT_VARIANTS * (streams - 1), 2 * NUM_SPLIT_VARIANTS for the
        tile kernel, 2 * NUM_SPLIT_VARIANTS + 1 + k for the persistent step
        in shape k, or 2 * NUM_SPLIT_VARIANTS + 1 + NUM_PERSIST_SHAPES for the
        split kernels behind the fused ghost fill ("split_fill")."""
        n = _capi.AUTOTUNE_CANDIDATES
        ms = (ctypes.c_double * n)()
        ch = ctypes.c_int()
        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_autotune(self._handle, _topology.ptr_array(qs), _topology.ptr_array(outs),
                                               float(dt), int(reps), ctypes.byref(ch), ms, _capi.stream(self.device)),
                    "fj_plan_autotune", c)
        return ch.value, list(ms)

    def set_streams(self, n: int) -> None:
        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_set_streams(self._handle, int(n)), "fj_plan_set_streams", c)

    def set_kernel(self, kernel: str) -> None:
        """Stage kernels of an FP32-flux plan: "split" (three kernels per stage
        through scratch), "tile" (one persistent fused kernel per stage over a
        (tile, i-plane) work-list, primitive planes staged by TMA),
        "persistent" (the whole step -- halo, boundary faces and the three
        stages -- in one launch over a dependency-ordered work-list) or
        "split_fill" (the split kernels after one launch that fills the
        ghost cells -- halo and boundary faces -- and computes the stage-1
        primitives)."""
        if kernel not in _capi.KERNELS:
            raise KeyError(kernel)
        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_set_kernel(self._handle, _capi.KERNELS[kernel]), "fj_plan_set_kernel", c)

    @property
    def kernel(self) -> str:
        k = ctypes.c_int()
        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_get_kernel(self._handle, ctypes.byref(k)), "fj_plan_get_kernel", c)
        return {v: n for n, v in _capi.KERNELS.items()}[k.value]

    def set_persist_shape(self, shape: int) -> None:
        """Launch shape of the persistent step (0 .. NUM_PERSIST_SHAPES-1)."""
        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_set_persist_shape(self._handle, int(shape)), "fj_plan_set_persist_shape", c)

    def set_wait_limit(self, limit: int) -> None:
        """Tries of each bounded wait in the tile kernel and the persistent
        step (-1: the default)."""
        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_set_wait_limit(self._handle, int(limit)), "fj_plan_set_wait_limit", c)

    def check(self) -> int:
        """Waits for the plan's work on the current stream and returns the
        error words of the tile kernel (bit 0) and the persistent step (bit 1)
        (0: no bounded wait gave up), clearing them; raises RuntimeError when
        one was nonzero."""
        w = ctypes.c_int()
        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_check(self._handle, ctypes.byref(w), _capi.stream(self.device)),
                    "fj_plan_check", c)
        return w.value

    def set_variant(self, variant: int) -> None:
        c = _capi.ctx(self.device)
        _capi.check(self._lib.fj_plan_set_variant(self._handle, int(variant)), "fj_plan_set_variant", c)

    def run_save(self, qs, outs, q0s, q1s, q2s, dt: float) -> None:
        """One step that also keeps its intermediate states (the halo-filled
        start state and the first two stage values) for the step adjoint."""
        for lst in (qs, outs, q0s, q1s, q2s):
            if [tuple(q.shape) for q in lst] != self.shapes:
                raise ValueError("state shapes differ from the plan's")
        c = _capi.ctx(self.device)
        pa = _topology.ptr_array
        _capi.check(self._lib.fj_plan_step_save(self._handle, pa(qs), pa(outs), pa(q0s), pa(q1s), pa(q2s), float(dt),
                                                _capi.stream(self.device)), "fj_plan_step_save", c)

    def stage(self, qs, q0s, outs, dt: float, stage: int) -> None:
        """One TVD-RK3 stage of every block (no halo fill)."""
        c = _capi.ctx(self.device)
        q0p = _topology.ptr_array(q0s) if q0s is not None else None
        _capi.check(self._lib.fj_plan_stage(self._handle, _topology.ptr_array(qs), q0p, _topology.ptr_array(outs),
                                            float(dt), int(stage), _capi.stream(self.device)), "fj_plan_stage", c)

    def __del__(self):
        if getattr(self, "_handle", None):
            self._lib.fj_plan_destroy(self._handle)
            self._handle = None


_PLANS: list = []  # (key, cfg, metrics, plan), most recent last
_MAX_PLANS = 4


def _cached_plan(state: State, cfg: Config) -> StepPlan:
    """The plan for this block layout, these metric arrays, this cfg object
    (kept alive by the cache entry, so their ids stay unique while cached) and
    the context's current pipeline setting."""
    dev = state.blocks[0].q.device
    key = (id(cfg), id(state.metrics), tuple((tuple(b.q.shape), str(b.q.device)) for b in state.blocks),
           tuple((m.kxyz.data_ptr(), m.vol.data_ptr()) for m in state.metrics), _capi.pipeline_setting(dev))
    for n, (k, _, _, plan) in enumerate(_PLANS):
        if k == key:
            _PLANS.append(_PLANS.pop(n))
            return plan
    plan = StepPlan(state, cfg)
    _PLANS.append((key, cfg, state.metrics, plan))
    if len(_PLANS) > _MAX_PLANS:
        _PLANS.pop(0)
    return plan


def step(state: State, cfg: Config, dt: float, *, plan: StepPlan | None = None) -> State:
    """Advance by dt with TVD-RK3 (solver/step.py:18-56)."""
    plan = plan or _cached_plan(state, cfg)
    qs = [b.q for b in state.blocks]
    outs = [torch.empty_like(q) for q in qs]
    plan.run(qs, outs, dt)
    new_blocks = tuple(Block(q=o, xyz=b.xyz) for o, b in zip(outs, state.blocks))
    return State(blocks=new_blocks, metrics=state.metrics, t=state.t + dt, step=state.step + 1)

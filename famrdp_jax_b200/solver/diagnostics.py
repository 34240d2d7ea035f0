"""FP64 reductions over a State: CFL time step, kinetic-energy integral and
the state check.  The reference passes dt in (solver/step.py:18) and declares
Config.cfl / Config.nan_check without reading them (core/types.py:187-189);
these are the definitions this package adds."""
from __future__ import annotations

import ctypes

from famrdp_jax_b200 import _capi, _topology
from famrdp_jax_b200.core.types import Config, State


def cfl_dt(state: State, cfg: Config, cfl: float | None = None) -> float:
    """dt = cfl / max over interior cells of sum_a (|u . n_a| + c) |kxyz[a,:]| / vol."""
    qs = [b.q for b in state.blocks]
    dev = qs[0].device
    c = _capi.ctx(dev)
    p = _capi.params(cfg.gas, limiter=cfg.scheme.limiter, ghost=cfg.ghost)
    out = ctypes.c_double()
    _capi.check(_capi.lib().fj_cfl_dt_f64(c, _topology.block_array(qs, state.metrics), len(qs), p,
                                          float(cfg.cfl if cfl is None else cfl), ctypes.byref(out),
                                          _capi.stream(dev)), "fj_cfl_dt_f64", c)
    return out.value


def kinetic_energy(state: State, ghost: int = 2) -> float:
    """J = sum over interior cells of vol * 0.5 |rho u|^2 / rho."""
    qs = [b.q for b in state.blocks]
    dev = qs[0].device
    c = _capi.ctx(dev)
    out = ctypes.c_double()
    _capi.check(_capi.lib().fj_kinetic_energy_f64(c, _topology.block_array(qs, state.metrics), len(qs),
                                                  int(ghost), ctypes.byref(out), _capi.stream(dev)),
                "fj_kinetic_energy_f64", c)
    return out.value


def check_state(state: State, gamma: float, *, raise_on_error: bool = True):
    """(nonfinite count, min rho, min p) over all padded cells; raises
    FloatingPointError on NaN/Inf or non-positive rho/p unless told not to."""
    qs = [b.q for b in state.blocks]
    dev = qs[0].device
    c = _capi.ctx(dev)
    n = ctypes.c_int64()
    r = ctypes.c_double()
    pm = ctypes.c_double()
    s = _capi.lib().fj_check_state_f64(c, _topology.block_array(qs), len(qs), float(gamma), ctypes.byref(n),
                                       ctypes.byref(r), ctypes.byref(pm), _capi.stream(dev))
    if s != _capi.FJ_ERR_NONFINITE or raise_on_error:
        _capi.check(s, "fj_check_state_f64", c)
    return n.value, r.value, pm.value


def residual(state: State, prev, dt: float, ghost: int = 2) -> list[float]:
    """Per-component RMS over interior cells of (q - q_prev) / dt for the five
    conserved variables, over all blocks (``prev``: the previous step's q per
    block)."""
    qs = [b.q for b in state.blocks]
    dev = qs[0].device
    c = _capi.ctx(dev)
    out = (ctypes.c_double * 5)()
    _capi.check(_capi.lib().fj_residual_f64(c, _topology.block_array(qs), _topology.ptr_array(list(prev)), len(qs),
                                            int(ghost), float(dt), out, _capi.stream(dev)), "fj_residual_f64", c)
    return list(out)

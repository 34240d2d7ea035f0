"""Equation of state (famrdp_jax ``physics/eos.py``).

``prim_to_cons`` / ``cons_to_prim`` run the CUDA kernels of libfamrdp_cuda.so
on (5, ...) float64 CUDA tensors.  ``speed_of_sound`` and
``sutherland_viscosity`` are the reference's closed-form scalar helpers
(physics/eos.py:20-25) and accept floats or tensors.
"""
from __future__ import annotations

import math

import torch

from famrdp_jax_b200 import _capi


def _pointwise(fn_name: str, x: torch.Tensor, gamma: float) -> torch.Tensor:
    if x.shape[0] != 5:
        raise ValueError(f"leading dimension must be 5, got {tuple(x.shape)}")
    xc = x.contiguous()
    out = torch.empty_like(xc)
    n = xc.numel() // 5
    _capi.check(getattr(_capi.lib(), fn_name)(_capi.dev_ptr(xc, "x"), _capi.dev_ptr(out, "out"), n,
                                              float(gamma), _capi.stream(xc.device)), fn_name)
    return out


def prim_to_cons(prim: torch.Tensor, gamma: float) -> torch.Tensor:
    """[rho, u, v, w, p] -> [rho, rho u, rho v, rho w, rho E] (physics/eos.py:5-9)."""
    return _pointwise("fj_prim_to_cons_f64", prim, gamma)


def cons_to_prim(q: torch.Tensor, gamma: float) -> torch.Tensor:
    """[rho, rho u, rho v, rho w, rho E] -> [rho, u, v, w, p] (physics/eos.py:12-17)."""
    return _pointwise("fj_cons_to_prim_f64", q, gamma)


def speed_of_sound(rho, p, gamma):
    """sqrt(gamma p / rho) (physics/eos.py:20-21)."""
    if isinstance(rho, torch.Tensor) or isinstance(p, torch.Tensor):
        return torch.sqrt(gamma * p / rho)
    return math.sqrt(gamma * p / rho)


def sutherland_viscosity(T, mu0, T0, Ts):
    """mu0 (T/T0)^1.5 (T0+Ts)/(T+Ts) (physics/eos.py:24-25)."""
    return mu0 * (T / T0) ** 1.5 * (T0 + Ts) / (T + Ts)

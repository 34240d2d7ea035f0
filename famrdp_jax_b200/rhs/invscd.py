"""Inviscid RHS (famrdp_jax ``rhs/invscd.py:18-133``) on the GPU.

For each axis: MUSCL-2 on primitives, Roe flux along the normal averaged from
the two adjacent cells' kxyz rows, times |n|, differenced and divided by
vol + 1e-300 at cells [2, n-3] along that axis and at every index of the other
two axes.
"""
from __future__ import annotations

import torch

from famrdp_jax_b200 import _capi
from famrdp_jax_b200.core.types import Metrics


class _Gas:
    def __init__(self, gamma):
        self.gamma = gamma
        self.R = 1.0
        self.mu0 = 0.0
        self.T0 = 1.0
        self.Ts = 0.0
        self.Pr_lam = 1.0


def compute_invscd_rhs(q: torch.Tensor, metrics: Metrics, *, ghost: int, gamma: float,
                       reconstruct: str, flux: str, limiter: str, precision: str = "f64") -> torch.Tensor:
    """rhs (5, ni, nj, nk) of the inviscid terms (rhs/invscd.py:18-27 signature)."""
    p = _capi.params(_Gas(gamma), limiter=limiter, ghost=ghost, precision=precision)
    rhs = torch.empty_like(q)
    ni, nj, nk = q.shape[1:]
    c = _capi.ctx(q.device)
    _capi.check(_capi.lib().fj_invscd_rhs_f64(c, _capi.dev_ptr(q, "q"), _capi.dev_ptr(metrics.kxyz, "kxyz"),
                                              _capi.dev_ptr(metrics.vol, "vol"), _capi.dev_ptr(rhs, "rhs"),
                                              ni, nj, nk, p, _capi.stream(q.device)),
                "fj_invscd_rhs_f64", c)
    return rhs

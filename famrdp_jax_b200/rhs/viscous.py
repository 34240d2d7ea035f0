"""Viscous RHS (famrdp_jax ``rhs/viscous.py:19-119``) on the GPU.

Evaluated on every padded cell; central differences wrap around the padded
array (jnp.roll semantics, rhs/viscous.py:12-16) in both the gradient and the
divergence, and the divergence uses the cell's own kxyz.  No 1/vol factor.
"""
from __future__ import annotations

import torch

from famrdp_jax_b200 import _capi
from famrdp_jax_b200.core.types import GasModel, Metrics


def compute_viscous_rhs(q: torch.Tensor, metrics: Metrics, *, gas: GasModel, ghost: int,
                        precision: str = "f64") -> torch.Tensor:
    """rhs (5, ni, nj, nk) = [0, div tau_0., div tau_1., div tau_2., div(u.tau - heat)]."""
    p = _capi.params(gas, ghost=ghost, precision=precision)
    rhs = torch.empty_like(q)
    ni, nj, nk = q.shape[1:]
    c = _capi.ctx(q.device)
    _capi.check(_capi.lib().fj_viscous_rhs_f64(c, _capi.dev_ptr(q, "q"), _capi.dev_ptr(metrics.kxyz, "kxyz"),
                                               _capi.dev_ptr(rhs, "rhs"), ni, nj, nk, p,
                                               _capi.stream(q.device)),
                "fj_viscous_rhs_f64", c)
    return rhs

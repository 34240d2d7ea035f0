"""Grid metrics (famrdp_jax ``mesh/metric.py:31-70``) on the GPU.

4th-order central differences with wrap-around at the array ends (so the
outermost layers are meaningful only for periodic coordinates), per-cell
3x3 determinant and inverse: jac = det(dx/dxi), kxyz[l, m] = dxi_l/dx_m,
vol = |jac|.
"""
from __future__ import annotations

import torch

from famrdp_jax_b200 import _capi
from famrdp_jax_b200.core.types import Metrics


def compute_metrics(xyz: torch.Tensor, *, ghost: int) -> Metrics:
    if xyz.dim() != 4 or xyz.shape[0] != 3:
        raise ValueError(f"xyz must have shape (3, ni, nj, nk), got {tuple(xyz.shape)}")
    x = xyz.contiguous()
    ni, nj, nk = x.shape[1:]
    jac = torch.empty((ni, nj, nk), dtype=torch.float64, device=x.device)
    kxyz = torch.empty((3, 3, ni, nj, nk), dtype=torch.float64, device=x.device)
    vol = torch.empty_like(jac)
    _capi.check(_capi.lib().fj_metrics_f64(_capi.dev_ptr(x, "xyz"), _capi.dev_ptr(jac, "jac"),
                                           _capi.dev_ptr(kxyz, "kxyz"), _capi.dev_ptr(vol, "vol"),
                                           ni, nj, nk, _capi.stream(x.device)), "fj_metrics_f64")
    return Metrics(jac=jac, kxyz=kxyz, vol=vol)

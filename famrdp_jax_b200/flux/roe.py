"""Roe flux with Harten's entropy fix (famrdp_jax ``flux/roe.py:21-85``) on the
GPU, over any number of faces."""
from __future__ import annotations

import torch

from famrdp_jax_b200 import _capi


def roe_flux(UL: torch.Tensor, UR: torch.Tensor, nxyz: torch.Tensor, *, gamma: float,
             eps_entropy: float = 0.1) -> torch.Tensor:
    """0.5 (F(UL) + F(UR)) - 0.5 |A| (UR - UL) along the unit normal ``nxyz``.

    UL, UR: (5, ...) conserved states; nxyz: (3, ...).  Trailing dimensions
    broadcast against each other like the reference's jnp arithmetic."""
    if UL.shape[0] != 5 or UR.shape[0] != 5 or nxyz.shape[0] != 3:
        raise ValueError("UL/UR must have leading dimension 5 and nxyz 3")
    trail = torch.broadcast_shapes(UL.shape[1:], UR.shape[1:], nxyz.shape[1:])
    UL = UL.expand(5, *trail).contiguous()
    UR = UR.expand(5, *trail).contiguous()
    nx = nxyz.expand(3, *trail).contiguous()
    F = torch.empty_like(UL)
    n = F.numel() // 5
    _capi.check(_capi.lib().fj_roe_flux_f64(_capi.dev_ptr(UL, "UL"), _capi.dev_ptr(UR, "UR"),
                                            _capi.dev_ptr(nx, "nxyz"), _capi.dev_ptr(F, "F"), n,
                                            float(gamma), float(eps_entropy),
                                            _capi.stream(F.device)), "fj_roe_flux_f64")
    return F

"""TVD-RK3 (Shu-Osher) of famrdp_jax ``time/rk.py:5-20``; the stage combines run
as one CUDA kernel each."""
from __future__ import annotations

import torch

from famrdp_jax_b200 import _capi


def _combine(q0, qs, L, dt, stage):
    qs = qs.contiguous()
    L = L.contiguous()
    q0c = q0.contiguous() if q0 is not None else qs
    out = torch.empty_like(qs)
    _capi.check(_capi.lib().fj_rk3_combine_f64(_capi.dev_ptr(q0c, "q0"), _capi.dev_ptr(qs, "qs"),
                                               _capi.dev_ptr(L, "L"), _capi.dev_ptr(out, "out"), qs.numel(),
                                               float(dt), stage, _capi.stream(qs.device)), "fj_rk3_combine_f64")
    return out


def rk3_step(q: torch.Tensor, L, dt: float) -> torch.Tensor:
    """q1 = q + dt L(q); q2 = 3/4 q + 1/4 (q1 + dt L(q1)); q+ = 1/3 q + 2/3 (q2 + dt L(q2))."""
    q1 = _combine(None, q, L(q), dt, 1)
    q2 = _combine(q, q1, L(q1), dt, 2)
    return _combine(q, q2, L(q2), dt, 3)

"""MUSCL-2 reconstruction (famrdp_jax ``physics/reconstruct/muscl2.py``) on the
GPU.  Face f in [0, n-4] along ``axis`` lies between cells f+1 and f+2."""
from __future__ import annotations

import torch

from famrdp_jax_b200 import _capi

_LIMITERS = {"minmod": 0, "vanleer": 1}


def _limiter(a, b, which: int) -> torch.Tensor:
    a = torch.as_tensor(a, dtype=torch.float64)
    b = torch.as_tensor(b, dtype=torch.float64)
    dev = a.device if a.is_cuda else b.device
    a, b = torch.broadcast_tensors(a.to(dev), b.to(dev))
    a = a.contiguous()
    b = b.contiguous()
    out = torch.empty_like(a)
    _capi.check(_capi.lib().fj_limiter_f64(_capi.dev_ptr(a, "a"), _capi.dev_ptr(b, "b"),
                                           _capi.dev_ptr(out, "out"), a.numel(), which,
                                           _capi.stream(a.device)), "fj_limiter_f64")
    return out


def minmod(a, b) -> torch.Tensor:
    """sign(a) max(sign(a) sign(b), 0) min(|a|, |b|) (muscl2.py:5-7)."""
    return _limiter(a, b, 0)


def vanleer(a, b) -> torch.Tensor:
    """2ab/(a+b) where ab > 0, else 0 (muscl2.py:10-12)."""
    return _limiter(a, b, 1)


def muscl2_reconstruct(pv: torch.Tensor, *, axis: int, limiter: str = "minmod"):
    """(pv_L, pv_R) on the n-3 faces along ``axis`` (muscl2.py:18-37).

    ``pv`` is a 4-D (nv, n1, n2, n3) float64 CUDA tensor and ``axis`` in
    {1, 2, 3}.  An unknown limiter raises KeyError, as in the reference."""
    lim = _LIMITERS[limiter]
    if pv.dim() != 4 or axis not in (1, 2, 3):
        raise ValueError("pv must be 4-D and axis in {1, 2, 3}")
    n = pv.shape[axis]
    if n < 4:
        raise ValueError(f"need at least 4 cells along axis {axis}, got {n}")
    pvc = pv.contiguous()
    shape = list(pvc.shape)
    shape[axis] = n - 3
    L = torch.empty(shape, dtype=torch.float64, device=pvc.device)
    R = torch.empty_like(L)
    nv, n1, n2, n3 = pvc.shape
    _capi.check(_capi.lib().fj_muscl2_f64(_capi.dev_ptr(pvc, "pv"), _capi.dev_ptr(L, "pv_L"),
                                          _capi.dev_ptr(R, "pv_R"), nv, n1, n2, n3, axis, lim,
                                          _capi.stream(pvc.device)), "fj_muscl2_f64")
    return L, R

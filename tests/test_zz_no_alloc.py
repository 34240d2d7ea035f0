"""fj_rhs_noalloc_f64: the block RHS for callers that may not allocate device
memory (for example this library called from inside a JAX/XLA custom call,
where XLA's allocator already holds most of the GPU, or a solver loop that
forbids allocation after start-up).  The entry point keeps its intermediates
in one fixed array inside the library instead of cudaMalloc'd scratch.

Checked here through the C ABI: two calls in a row on different blocks
agree with fj_rhs_f64 (the context-scratch entry point) within the RHS
tolerance of the parity tests; a call allocates no device memory (the
device's free memory is the same before and after it); and a block too large
for the fixed array is refused before any device work.  This file is
collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from famrdp_jax_b200 import _capi
from famrdp_jax_b200.core.types import GasModel
from parity_util import dev, host, random_block, rel_l2

pytestmark = pytest.mark.gpu

GAS = GasModel(gamma=1.4, R=1.0, mu0=2e-3, T0=1 / 1.4, Ts=0.27, Pr_lam=0.72)


def _rhs_with_context(q, kxyz, vol, p):
    out = torch.empty_like(q)
    ni, nj, nk = q.shape[1:]
    c = _capi.ctx(q.device)
    _capi.check(_capi.lib().fj_rhs_f64(c, q.data_ptr(), kxyz.data_ptr(), vol.data_ptr(), out.data_ptr(),
                                       ni, nj, nk, ctypes.byref(p), _capi.stream(q.device)), "fj_rhs_f64", c)
    return out


def _rhs_no_alloc(q, kxyz, vol, p):
    out = torch.empty_like(q)
    ni, nj, nk = q.shape[1:]
    status = _capi.lib().fj_rhs_noalloc_f64(q.data_ptr(), kxyz.data_ptr(), vol.data_ptr(), out.data_ptr(),
                                            ni, nj, nk, ctypes.byref(p), _capi.stream(q.device))
    return status, out


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_noalloc_rhs_matches_context_rhs_twice(cuda_device, precision):
    p = _capi.params(GAS, limiter="minmod", ghost=2, precision=precision)
    for shape, seed in (((20, 17, 23), 31), ((12, 26, 9), 32)):
        q, kxyz, vol = random_block(shape, seed)
        qd, kd, vd = dev(q), dev(kxyz), dev(vol)
        status, got = _rhs_no_alloc(qd, kd, vd, p)
        assert status == _capi.FJ_OK, _capi.lib().fj_status_string(status)
        ref = _rhs_with_context(qd, kd, vd, p)
        torch.cuda.synchronize()
        # the RHS tolerances of the parity tests: FP64 fluxes agree to 1e-11; two
        # FP32-flux evaluations differ by FP32 rounding, bounded like FP32 vs FP64
        assert rel_l2(host(got), host(ref)) <= (1e-11 if precision == "f64" else 1e-5)


def test_noalloc_rejects_blocks_beyond_capacity(cuda_device):
    # 70^3 padded cells need ~80 MB of intermediates in FP64: above the 64 MiB array.
    shape = (70, 70, 70)
    q = torch.ones((5,) + shape, dtype=torch.float64, device=cuda_device)
    kxyz = torch.zeros((3, 3) + shape, dtype=torch.float64, device=cuda_device)
    vol = torch.ones(shape, dtype=torch.float64, device=cuda_device)
    p = _capi.params(GAS, ghost=2, precision="f64")
    status, _ = _rhs_no_alloc(q, kxyz, vol, p)
    assert status == _capi.FJ_ERR_SCRATCH_LIMIT
    assert b"fixed scratch" in _capi.lib().fj_status_string(status)


def test_noalloc_call_allocates_no_device_memory(cuda_device):
    """After a first call (which loads the library's module and looks up the
    array's address), a call on a larger block leaves the device's free
    memory unchanged: no allocation by the library, the driver or torch."""
    p = _capi.params(GAS, limiter="minmod", ghost=2, precision="f64")
    q, kxyz, vol = random_block((10, 9, 8), 40)
    status, _ = _rhs_no_alloc(dev(q), dev(kxyz), dev(vol), p)
    assert status == _capi.FJ_OK
    q, kxyz, vol = random_block((60, 58, 62), 41)
    qd, kd, vd = dev(q), dev(kxyz), dev(vol)
    out = torch.empty_like(qd)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info(cuda_device)
    ni, nj, nk = qd.shape[1:]
    status = _capi.lib().fj_rhs_noalloc_f64(qd.data_ptr(), kd.data_ptr(), vd.data_ptr(), out.data_ptr(),
                                            ni, nj, nk, ctypes.byref(p), _capi.stream(qd.device))
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info(cuda_device)
    assert status == _capi.FJ_OK
    assert free_after == free_before, (free_before, free_after)
    assert torch.isfinite(out).all()

"""ctypes binding of libfamrdp_cuda.so (the C ABI in include/famrdp_cuda.h).

This module is the only place that touches the shared library.  It loads the
in-tree build (``famrdp_jax_b200/_lib/libfamrdp_cuda.so``), declares every
entry point's argument types, owns one ``fj_ctx`` per CUDA device and turns
status codes into the Python exceptions the reference raises for the same
conditions.  There is no fallback: without the library or without a CUDA
tensor every call raises.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libfamrdp_cuda.so"

FJ_OK = 0
FJ_ERR_INVALID_ARGUMENT = 1
FJ_ERR_CUDA = 2
FJ_ERR_NOT_IMPLEMENTED = 3
FJ_ERR_SHAPE = 4
FJ_ERR_NONFINITE = 5
FJ_ERR_NO_MEMORY = 6
FJ_ERR_SCRATCH_LIMIT = 7  # block too large for fj_rhs_noalloc_f64's fixed scratch
NOALLOC_SCRATCH_BYTES = 64 << 20

VISC_LAWS = {"sutherland": 0, "constant": 1}
LIMITERS = {"minmod": 0, "vanleer": 1}
PRECISIONS = {"f64": 0, "f32": 1}


class FjParams(ctypes.Structure):
    _fields_ = [("gamma", ctypes.c_double), ("R", ctypes.c_double), ("mu0", ctypes.c_double),
                ("T0", ctypes.c_double), ("Ts", ctypes.c_double), ("Pr", ctypes.c_double),
                ("eps_entropy", ctypes.c_double), ("visc_law", ctypes.c_int),
                ("limiter", ctypes.c_int), ("ghost", ctypes.c_int), ("precision", ctypes.c_int)]


class FjBlock(ctypes.Structure):
    _fields_ = [("q", ctypes.c_void_p), ("kxyz", ctypes.c_void_p), ("vol", ctypes.c_void_p),
                ("ni", ctypes.c_int), ("nj", ctypes.c_int), ("nk", ctypes.c_int)]


class FjLink(ctypes.Structure):
    _fields_ = [("tgt_block", ctypes.c_int), ("tgt_face", ctypes.c_int),
                ("src_block", ctypes.c_int), ("src_face", ctypes.c_int), ("orient", ctypes.c_int)]


class FjBc(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int), ("face", ctypes.c_int), ("type", ctypes.c_int),
                ("isothermal", ctypes.c_int), ("T_wall", ctypes.c_double),
                ("q_inf", ctypes.c_double * 5)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "fj_abi_version": (_I, []),
    "fj_status_string": (ctypes.c_char_p, [_I]),
    "fj_ctx_create": (_I, [ctypes.POINTER(_P)]),
    "fj_ctx_destroy": (_I, [_P]),
    "fj_last_error": (ctypes.c_char_p, [_P]),
    "fj_launch_count": (_I, [_P, ctypes.POINTER(_I64)]),
    "fj_ctx_set_pipeline": (_I, [_P, _I, _I, _I]),
    "fj_ctx_set_adjoint_variant": (_I, [_P, _I]),
    "fj_plan_create": (_I, [_P, ctypes.POINTER(FjBlock), _I, ctypes.POINTER(FjLink), _I, ctypes.POINTER(FjBc), _I,
                            ctypes.POINTER(FjParams), ctypes.POINTER(_P)]),
    "fj_plan_step": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _D, _P]),
    "fj_plan_set_ensemble": (_I, [_P, _P, _P]),
    "fj_plan_set_variant": (_I, [_P, _I]),
    "fj_plan_p_ref": (_I, [_P, ctypes.POINTER(_D)]),
    "fj_plan_set_p_ref": (_I, [_P, _D]),
    "fj_plan_set_streams": (_I, [_P, _I]),
    "fj_plan_set_kernel": (_I, [_P, _I]),
    "fj_plan_set_persist_shape": (_I, [_P, _I]),
    "fj_persist_list_check": (_I, [_P, _I, _P, _I, _P, _I, _P, _I, _I, ctypes.POINTER(ctypes.c_int64)]),
    "fj_plan_get_kernel": (_I, [_P, ctypes.POINTER(_I)]),
    "fj_plan_set_wait_limit": (_I, [_P, _I]),
    "fj_plan_check": (_I, [_P, ctypes.POINTER(_I), _P]),
    "fj_plan_autotune": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _D, _I, ctypes.POINTER(_I), _P, _P]),
    "fj_plan_step_graph": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _D, _P]),
    "fj_plan_step_save": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P),
                               ctypes.POINTER(_P), _D, _P]),
    "fj_plan_destroy": (_I, [_P]),
    "fj_plan_stage": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P), _D, _I, _P]),
    "fj_rhs_vjp_f64": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _I, ctypes.POINTER(FjParams), _P]),
    "fj_step_vjp_f64": (_I, [_P, ctypes.POINTER(FjBlock), ctypes.POINTER(_P), ctypes.POINTER(_P), _I,
                             ctypes.POINTER(FjLink), _I, ctypes.POINTER(FjBc), _I, ctypes.POINTER(FjParams), _D, _P]),
    "fj_step_vjp_mu_f64": (_I, [_P, ctypes.POINTER(FjBlock), ctypes.POINTER(_P), ctypes.POINTER(_P), _I,
                                ctypes.POINTER(FjLink), _I, ctypes.POINTER(FjBc), _I, ctypes.POINTER(FjParams), _D,
                                _P, _P]),
    "fj_step_vjp_saved_f64": (_I, [_P, ctypes.POINTER(FjBlock), ctypes.POINTER(_P), ctypes.POINTER(_P),
                                   ctypes.POINTER(_P), ctypes.POINTER(_P), _I, ctypes.POINTER(FjLink), _I,
                                   ctypes.POINTER(FjBc), _I, ctypes.POINTER(FjParams), _D, _P, _P]),
    "fj_step_vjp_ensemble_f64": (_I, [_P, ctypes.POINTER(FjBlock), ctypes.POINTER(_P), ctypes.POINTER(_P),
                                      ctypes.POINTER(_P), ctypes.POINTER(_P), _I, ctypes.POINTER(FjLink), _I,
                                      ctypes.POINTER(FjBc), _I, ctypes.POINTER(FjParams), _D, _P, _P, _P, _P]),
    "fj_residual_f64": (_I, [_P, ctypes.POINTER(FjBlock), ctypes.POINTER(_P), _I, _I, _D, _P, _P]),
    "fj_kinetic_energy_grad_f64": (_I, [_P, ctypes.POINTER(FjBlock), ctypes.POINTER(_P), _I, _I, _P]),
    "fj_rk_stage_f64": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _I, ctypes.POINTER(FjParams), _D, _I, _P]),
    "fj_cons_to_prim_f64": (_I, [_P, _P, _I64, _D, _P]),
    "fj_prim_to_cons_f64": (_I, [_P, _P, _I64, _D, _P]),
    "fj_roe_flux_f64": (_I, [_P, _P, _P, _P, _I64, _D, _D, _P]),
    "fj_muscl2_f64": (_I, [_P, _P, _P, _I, _I, _I, _I, _I, _I, _P]),
    "fj_limiter_f64": (_I, [_P, _P, _P, _I64, _I, _P]),
    "fj_invscd_rhs_f64": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, ctypes.POINTER(FjParams), _P]),
    "fj_viscous_rhs_f64": (_I, [_P, _P, _P, _P, _I, _I, _I, ctypes.POINTER(FjParams), _P]),
    "fj_rhs_f64": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, ctypes.POINTER(FjParams), _P]),
    "fj_rhs_noalloc_f64": (_I, [_P, _P, _P, _P, _I, _I, _I, ctypes.POINTER(FjParams), _P]),
    "fj_halo_exchange_f64": (_I, [_P, ctypes.POINTER(FjBlock), _I, ctypes.POINTER(FjLink), _I, _I, _P]),
    "fj_halo_pack_f64": (_I, [_P, ctypes.POINTER(FjBlock), _I, ctypes.POINTER(FjLink), _I, _I,
                              ctypes.POINTER(_I), ctypes.POINTER(_I64), _I, _P, _I64, _P]),
    "fj_halo_unpack_f64": (_I, [_P, ctypes.POINTER(FjBlock), _I, ctypes.POINTER(FjLink), _I, _I,
                                ctypes.POINTER(_I), ctypes.POINTER(_I64), _I, _P, _I64, _P]),
    "fj_apply_bc_f64": (_I, [_P, ctypes.POINTER(FjBlock), _I, ctypes.POINTER(FjBc), _I,
                             ctypes.POINTER(FjParams), _P]),
    "fj_step_f64": (_I, [_P, ctypes.POINTER(FjBlock), ctypes.POINTER(_P), _I, ctypes.POINTER(FjLink), _I,
                         ctypes.POINTER(FjBc), _I, ctypes.POINTER(FjParams), _D, _P]),
    "fj_rk3_combine_f64": (_I, [_P, _P, _P, _P, _I64, _D, _I, _P]),
    "fj_metrics_f64": (_I, [_P, _P, _P, _P, _I, _I, _I, _P]),
    "fj_cfl_dt_f64": (_I, [_P, ctypes.POINTER(FjBlock), _I, ctypes.POINTER(FjParams), _D,
                           ctypes.POINTER(_D), _P]),
    "fj_kinetic_energy_f64": (_I, [_P, ctypes.POINTER(FjBlock), _I, _I, ctypes.POINTER(_D), _P]),
    "fj_check_state_f64": (_I, [_P, ctypes.POINTER(FjBlock), _I, _D, ctypes.POINTER(_I64),
                                ctypes.POINTER(_D), ctypes.POINTER(_D), _P]),
}

_lib = None
_lock = threading.Lock()
_ctxs: dict[int, int] = {}


def lib():
    """The loaded library; raises RuntimeError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m famrdp_jax_b200.build`")
            L = ctypes.CDLL(str(LIB_PATH), mode=os.RTLD_LOCAL | getattr(os, "RTLD_NOW", 2))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def ctx(device: torch.device | int | None = None) -> int:
    """The library context of a CUDA device (created on first use)."""
    if device is None:
        dev = torch.cuda.current_device()
    elif isinstance(device, torch.device):
        dev = device.index if device.index is not None else torch.cuda.current_device()
    else:
        dev = int(device)
    h = _ctxs.get(dev)
    if h is None:
        with torch.cuda.device(dev):
            p = _P()
            _raise(lib().fj_ctx_create(ctypes.byref(p)), None, "fj_ctx_create")
            h = p.value
            _ctxs[dev] = h
    return h


PIPELINES = {"fused": 0, "staged": 1, "split": 2}


NUM_SPLIT_VARIANTS = 6  # FJ_NUM_SPLIT_VARIANTS
# FJ_KERNEL_SPLIT, FJ_KERNEL_TILE, FJ_KERNEL_PERSIST, FJ_KERNEL_SPLIT_FILL
KERNELS = {"split": 0, "tile": 1, "persistent": 2, "split_fill": 3}
NUM_PERSIST_SHAPES = 4  # FJ_NUM_PERSIST_SHAPES
AUTOTUNE_CANDIDATES = 2 * NUM_SPLIT_VARIANTS + 2 + NUM_PERSIST_SHAPES  # FJ_AUTOTUNE_CANDIDATES
TILES = {"8x32": 0, "4x32": 1, "6x32": 2, "8x16": 3, "16x32": 4, "8x64": 5, "16x16": 6}


DEFAULT_PIPELINE = "split"


def set_pipeline(pipeline: str = DEFAULT_PIPELINE, seg: int = 0, tile: str | int = 0, device=None) -> None:
    """How RHS / RK stages are evaluated: "split" (default: three barrier-free
    kernels per stage over all blocks), "fused" (one shared-memory streaming
    kernel per stage and block) or "staged" (the six-kernel cross-check); for
    the fused kernel ``seg`` = planes per CTA along i (0 = automatic) and
    ``tile`` the (j, k) tile shape."""
    c = ctx(device)
    t = TILES[tile] if isinstance(tile, str) else int(tile)
    check(lib().fj_ctx_set_pipeline(c, PIPELINES[pipeline], int(seg), t), "fj_ctx_set_pipeline", c)
    _PIPELINE_SETTING[_dev_key(device)] = (pipeline, int(seg), t)


_PIPELINE_SETTING: dict = {}


def _dev_key(device):
    import torch
    d = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    return (d.type, d.index if d.index is not None else torch.cuda.current_device())


def pipeline_setting(device=None):
    """(pipeline, seg, tile) last set on the device's context."""
    return _PIPELINE_SETTING.get(_dev_key(device), (DEFAULT_PIPELINE, 0, 0))


def set_adjoint_variant(variant: int = 0, device=None) -> None:
    """Launch shape of the adjoint's face and viscous kernels: 0 = the
    default (register caps per precision; with FP32 fluxes both in one
    launch), 1 = face kernel uncapped, 2 = the other face cap, 3 / 4 = 0 / 2
    with the viscous kernel uncapped."""
    c = ctx(device)
    check(lib().fj_ctx_set_adjoint_variant(c, int(variant)), "fj_ctx_set_adjoint_variant", c)


def launch_count(device=None) -> int:
    """Kernels launched so far through the device's context."""
    n = ctypes.c_int64()
    check(lib().fj_launch_count(ctx(device), ctypes.byref(n)), "fj_launch_count")
    return n.value


def stream(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _raise(status: int, c, what: str):
    if status == FJ_OK:
        return
    detail = ""
    if c is not None:
        msg = lib().fj_last_error(c)
        detail = msg.decode(errors="replace") if msg else ""
    text = f"{what}: {lib().fj_status_string(status).decode()}" + (f" ({detail})" if detail else "")
    if status == FJ_ERR_NOT_IMPLEMENTED:
        raise NotImplementedError(detail or text)
    if status in (FJ_ERR_SHAPE, FJ_ERR_INVALID_ARGUMENT):
        raise ValueError(text)
    if status == FJ_ERR_NONFINITE:
        raise FloatingPointError(text)
    if status == FJ_ERR_NO_MEMORY:
        raise MemoryError(text)
    if status == FJ_ERR_SCRATCH_LIMIT:
        raise ValueError(text)
    raise RuntimeError(text)


def check(status: int, what: str, c=None):
    _raise(status, c, what)


def dev_ptr(t: torch.Tensor, name: str) -> int:
    """Device pointer of a contiguous float64 CUDA tensor (raises otherwise)."""
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name!r} must be a torch.Tensor, got {type(t).__name__}")
    if t.dtype != torch.float64:
        raise TypeError(f"{name!r} must be float64, got {t.dtype}.")
    if not t.is_cuda:
        raise ValueError(f"{name!r} must be a CUDA tensor (the kernels have no CPU path)")
    if not t.is_contiguous():
        raise ValueError(f"{name!r} must be contiguous")
    return t.data_ptr()


def params(gas, *, limiter: str = "minmod", ghost: int = 2, precision: str = "f64",
           eps_entropy: float = 0.1) -> FjParams:
    """fj_params from a GasModel-like object.  Unknown limiter -> KeyError
    (physics/reconstruct/muscl2.py:19)."""
    p = FjParams()
    p.gamma = float(gas.gamma)
    p.R = float(gas.R)
    p.mu0 = float(gas.mu0)
    p.T0 = float(gas.T0)
    p.Ts = float(gas.Ts)
    p.Pr = float(gas.Pr_lam)
    p.eps_entropy = float(eps_entropy)
    p.visc_law = VISC_LAWS[getattr(gas, "visc_law", "sutherland")]
    p.limiter = LIMITERS[limiter]
    p.ghost = int(ghost)
    p.precision = PRECISIONS[precision]
    return p

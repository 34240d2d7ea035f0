"""The C ABI without a GPU: the in-tree library loads, exports every entry
point declared in include/famrdp_cuda.h, the ctypes table covers them, and
argument validation answers before any device work."""
import ctypes
import re
from pathlib import Path

import pytest

from famrdp_jax_b200 import _capi

HEADER = Path(__file__).resolve().parent.parent / "include" / "famrdp_cuda.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(fj_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "fj_step_f64" in syms and "fj_rhs_f64" in syms and "fj_metrics_f64" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"not exported: {missing}"


def test_ctypes_table_covers_header():
    assert set(declared_symbols()) == set(_capi.SIGNATURES)


def test_abi_version_and_status_strings():
    lib = _capi.lib()
    assert lib.fj_abi_version() == 1
    assert lib.fj_status_string(0) == b"ok"
    assert lib.fj_status_string(3) == b"not implemented"


def test_validation_before_device_work():
    lib = _capi.lib()
    # NULL arrays and bad enums are rejected without touching a device
    assert lib.fj_roe_flux_f64(None, None, None, None, 10, 1.4, 0.1, None) == _capi.FJ_ERR_INVALID_ARGUMENT
    assert lib.fj_muscl2_f64(None, None, None, 5, 8, 8, 8, 1, 0, None) == _capi.FJ_ERR_INVALID_ARGUMENT
    assert lib.fj_rk3_combine_f64(None, None, None, None, 10, 0.1, 4, None) == _capi.FJ_ERR_INVALID_ARGUMENT
    assert lib.fj_ctx_destroy(None) == 0


def test_struct_layouts_match_header():
    # fj_params: 7 doubles + 4 ints; fj_block: 3 pointers + 3 ints (+ padding)
    assert ctypes.sizeof(_capi.FjParams) == 7 * 8 + 4 * 4
    assert ctypes.sizeof(_capi.FjBlock) == 3 * 8 + 3 * 4 + 4
    assert ctypes.sizeof(_capi.FjLink) == 5 * 4
    assert ctypes.sizeof(_capi.FjBc) == 4 * 4 + 8 + 5 * 8


def test_no_cpu_fallback():
    import torch
    with pytest.raises(ValueError, match="CUDA"):
        _capi.dev_ptr(torch.zeros(3, dtype=torch.float64), "q")
    with pytest.raises(TypeError):
        _capi.dev_ptr(torch.zeros(3, dtype=torch.float32), "q")

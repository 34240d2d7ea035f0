"""FP64 guards (famrdp_jax ``core/dtypes.py:5-17``): a state or metric array
that is not float64 raises ``TypeError`` at construction."""
import numpy as np
import torch


def assert_float64(arr, *, name: str) -> None:
    dt = getattr(arr, "dtype", None)
    if dt is None:
        return
    if dt not in (torch.float64, np.float64, np.dtype("float64")):
        raise TypeError(f"{name!r} must be float64, got {dt}.")


def check_array_f64(tree) -> None:
    """Check every array leaf of a dict/tuple/list of arrays."""
    if isinstance(tree, dict):
        leaves = list(tree.items())
    elif isinstance(tree, (list, tuple)):
        leaves = [(f"leaf[{i}]", x) for i, x in enumerate(tree)]
    else:
        leaves = [("leaf[0]", tree)]
    for name, leaf in leaves:
        assert_float64(leaf, name=name)

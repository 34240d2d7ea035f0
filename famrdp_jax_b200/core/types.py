"""Block / metric / state containers and the frozen configuration types.

The layout contract is famrdp_jax ``core/types.py:26-189``:

* ``Block.q``       (5, ni, nj, nk) float64 -- [rho, rho*u, rho*v, rho*w, rho*E],
  ghost layers embedded (``ni = interior_i + 2*ghost`` and so on), C order so
  k is the contiguous axis;
* ``Block.xyz``     (3, ni, nj, nk) float64;
* ``Metrics.jac``   (ni, nj, nk), ``Metrics.kxyz`` (3, 3, ni, nj, nk) with
  ``kxyz[l, m] = d xi_l / d x_m``, ``Metrics.vol`` (ni, nj, nk);
* ``State``         tuple of blocks, tuple of metrics, time ``t``, step index.

Here the arrays are ``torch.Tensor`` (CUDA tensors on the kernel path) instead
of ``jax.Array``; non-float64 arrays raise ``TypeError`` as in the reference
(``core/types.py:37-38,75-76``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

from famrdp_jax_b200.core.dtypes import check_array_f64


@dataclass
class Block:
    """Conservative variables and coordinates of one block (core/types.py:26-52)."""
    q: object
    xyz: object

    def __post_init__(self):
        check_array_f64({"q": self.q, "xyz": self.xyz})


@dataclass
class Metrics:
    """Grid metrics of one block (core/types.py:62-89)."""
    jac: object
    kxyz: object
    vol: object

    def __post_init__(self):
        check_array_f64({"jac": self.jac, "kxyz": self.kxyz, "vol": self.vol})


@dataclass
class State:
    """Global simulation state (core/types.py:99-136)."""
    blocks: tuple
    metrics: tuple
    t: float = 0.0
    step: int = 0


@dataclass(frozen=True)
class BlockTopology:
    """Connectivity of one block (core/types.py:146-156).

    neighbors : dict[Face -> None | (block_id, Face, orient)], in the order the
                halo fill visits the faces;
    bc_type   : dict[Face -> BCType]
    """
    block_id: int
    neighbors: dict
    bc_type: dict


@dataclass(frozen=True)
class GasModel:
    """Ideal gas + viscosity law (core/types.py:159-167).

    ``visc_law`` is an addition: "sutherland" (the reference's only law,
    physics/eos.py:24-25) or "constant" (mu = mu0 everywhere)."""
    gamma: float = 1.4
    R: float = 287.058
    mu0: float = 1.71608e-5
    T0: float = 273.15
    Ts: float = 110.4
    Pr_lam: float = 0.72
    visc_law: str = "sutherland"


@dataclass(frozen=True)
class SchemeChoice:
    """Scheme selections (core/types.py:170-176)."""
    reconstruct: str
    flux: str
    rk_order: int
    limiter: str


@dataclass(frozen=True)
class Config:
    """Top-level configuration (core/types.py:179-189).

    ``precision`` is an addition: "f64" (every flux in FP64, the drop-in path)
    or "f32" (reconstruction, Roe and viscous fluxes in FP32; state, metrics,
    RK accumulation and reductions in FP64)."""
    gas: GasModel
    scheme: SchemeChoice
    bc_params: dict
    topology: tuple
    ghost: int = 2
    nan_check: bool = True
    debug: bool = False
    cfl: float = 1.0
    precision: str = "f64"

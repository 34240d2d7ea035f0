"""Seeded synthetic workloads with the shapes of the published configurations.

No dataset or checkpoint is involved: every state is generated here from a
closed-form flow plus seeded Gaussian noise.  Nondimensionalisation: rho0 = 1,
c0 = 1, so p0 = 1/gamma, R = 1, T0 = p0/(rho0 R) = 1/gamma; a viscosity
mu = rho0 U L / Re with L = 1 and U the Mach number.

Workloads
  tgv          single block, uniform Cartesian grid on [0, 2 pi)^3, self-periodic
               CUT1TO1 on all six faces (orient 0), Taylor-Green vortex
               (32^3 at M0 = 0.1, Re = 1600, constant viscosity; or 96^3 at
               M0 = 0.3, Re = 800);
  wavy4        4 curvilinear blocks of n^3 cells in a 2 x 2 arrangement in i-j,
               periodic in i, j and k, grid x = I h + 0.05 sin(2 pi I/N) sin(2 pi J/N)
               (same displacement on y, z uniform), freestream Mach 0.5 along x,
               Re = 1e4, 1 % Gaussian noise on rho, u, v, w, p (n = 128 is the
               4 x 128^3 workload);
  tree24       24 blocks with per-axis sizes drawn from U[16, 160], joined by a
               seeded random spanning tree of same-axis opposite-face interfaces;
               each remaining face is self-periodic when its opposite face is
               also free, else farfield; Mach 0.8, Re = 5e4, 1 % noise.

``metrics_fn(xyz) -> (jac, kxyz, vol)`` computes the metrics of a curvilinear
block from coordinates extended by two extra layers on every side (the result
is cropped by two layers, so the roll wrap of the 4th-order difference never
reaches a kept cell).  Callers pass the GPU kernel; CPU tests pass the oracle.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from famrdp_jax_b200.core.constants import BCType, Face
from famrdp_jax_b200.core.types import BlockTopology, Config, GasModel, SchemeChoice

GHOST = 2


@dataclass
class Case:
    name: str
    qs: list            # numpy (5, ni, nj, nk) per block
    metrics: list       # numpy (jac, kxyz, vol) per block
    cfg: Config
    cfl: float
    steps: int
    meta: dict = field(default_factory=dict)

    @property
    def padded_cells(self) -> int:
        return int(sum(q.shape[1] * q.shape[2] * q.shape[3] for q in self.qs))

    @property
    def interior_cells(self) -> int:
        g = self.cfg.ghost
        return int(sum((q.shape[1] - 2 * g) * (q.shape[2] - 2 * g) * (q.shape[3] - 2 * g) for q in self.qs))


def to_state(case: Case, device="cuda"):
    """State (torch float64 tensors on ``device``) of a case; xyz is zero
    because the step never reads coordinates."""
    import torch

    from famrdp_jax_b200.core.types import Block, Metrics, State

    def t(x):
        return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=device)

    blocks, metrics = [], []
    for q, (jac, kxyz, vol) in zip(case.qs, case.metrics):
        blocks.append(Block(q=t(q), xyz=torch.zeros((3,) + q.shape[1:], dtype=torch.float64, device=device)))
        metrics.append(Metrics(jac=t(jac), kxyz=t(kxyz), vol=t(vol)))
    return State(blocks=tuple(blocks), metrics=tuple(metrics), t=0.0, step=0)


def prim_to_cons_np(rho, u, v, w, p, gamma):
    ke = 0.5 * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, p / (gamma - 1.0) + rho * ke], axis=0)


def _scheme(limiter="minmod"):
    return SchemeChoice(reconstruct="muscl2", flux="roe", rk_order=3, limiter=limiter)


def _self_periodic_topology(block_id=0):
    nb = {Face.IMIN: (block_id, Face.IMAX, 0), Face.IMAX: (block_id, Face.IMIN, 0),
          Face.JMIN: (block_id, Face.JMAX, 0), Face.JMAX: (block_id, Face.JMIN, 0),
          Face.KMIN: (block_id, Face.KMAX, 0), Face.KMAX: (block_id, Face.KMIN, 0)}
    return BlockTopology(block_id=block_id, neighbors=nb, bc_type={f: BCType.CUT1TO1 for f in Face})


def uniform_metrics(shape, h):
    ni, nj, nk = shape
    kxyz = np.zeros((3, 3, ni, nj, nk))
    for d in range(3):
        kxyz[d, d] = 1.0 / h
    jac = np.full((ni, nj, nk), h ** 3)
    return jac, kxyz, jac.copy()


def tgv(n=32, M0=0.1, Re=1600.0, gamma=1.4, Pr=0.72, visc_law="constant", noise=0.0, seed=0,
        limiter="minmod", cfl=0.5, steps=10, precision="f64") -> Case:
    """Taylor-Green vortex on one self-periodic block of n^3 cells."""
    g = GHOST
    h = 2.0 * math.pi / n
    x = (np.arange(n + 2 * g) - g + 0.5) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    rho0, p0 = 1.0, 1.0 / gamma
    T0 = p0 / rho0
    u = M0 * np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -M0 * np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    p = p0 + (rho0 * M0 ** 2 / 16.0) * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    rho = p / T0
    if noise > 0:
        rng = np.random.default_rng(seed)
        rho = rho * (1 + noise * rng.standard_normal(rho.shape))
        p = p * (1 + noise * rng.standard_normal(p.shape))
        u = u + noise * M0 * rng.standard_normal(u.shape)
        v = v + noise * M0 * rng.standard_normal(v.shape)
        w = w + noise * M0 * rng.standard_normal(w.shape)
    q = prim_to_cons_np(rho, u, v, w, p, gamma)
    gas = GasModel(gamma=gamma, R=1.0, mu0=rho0 * M0 / Re, T0=T0, Ts=T0 * 110.4 / 288.15, Pr_lam=Pr,
                   visc_law=visc_law)
    cfg = Config(gas=gas, scheme=_scheme(limiter), bc_params={}, topology=(_self_periodic_topology(0),),
                 ghost=g, nan_check=False, cfl=cfl, precision=precision)
    return Case(name=f"tgv{n}", qs=[q], metrics=[uniform_metrics(q.shape[1:], h)], cfg=cfg, cfl=cfl,
                steps=steps, meta={"n": n, "M0": M0, "Re": Re, "h": h})


def tgv_dq0_dM0(case: Case) -> np.ndarray:
    """d q0 / d M0 of a ``tgv`` case at its Mach number (same seed, so the
    noise draws are held fixed): u, v, w scale with M0, and rho and p carry
    M0^2 b with b = (rho0/16)(cos 2x + cos 2y)(cos 2z + 2), each times its own
    noise factor.  The case's viscosity mu0 = rho0 M0 / Re also depends on M0;
    that part is d mu0 / d M0 = rho0 / Re (see ``case.meta``)."""
    n, M0, h = case.meta["n"], case.meta["M0"], case.meta["h"]
    gamma = case.cfg.gas.gamma
    g = case.cfg.ghost
    x = (np.arange(n + 2 * g) - g + 0.5) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    rho0, p0 = 1.0, 1.0 / gamma
    b = (rho0 / 16.0) * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    q = case.qs[0]
    rho = q[0]
    u, v, w = q[1] / rho, q[2] / rho, q[3] / rho
    p = (gamma - 1.0) * (q[4] - 0.5 * rho * (u * u + v * v + w * w))
    clean = p0 + M0 ** 2 * b  # p (and rho T0) before the noise factors
    drho = 2.0 * M0 * b * rho / clean
    dp = 2.0 * M0 * b * p / clean
    du, dv, dw = u / M0, v / M0, w / M0
    out = np.empty_like(q)
    out[0] = drho
    out[1] = drho * u + rho * du
    out[2] = drho * v + rho * dv
    out[3] = drho * w + rho * dw
    out[4] = dp / (gamma - 1.0) + 0.5 * drho * (u * u + v * v + w * w) + rho * (u * du + v * dv + w * dw)
    return out


def ensemble(ninst=64, n=64, M_range=(0.1, 0.9), Re_range=(1e2, 1e4), noise=0.005, seed=0, gamma=1.4, Pr=0.72,
             visc_law="constant", limiter="minmod", cfl=0.5, steps=100, precision="f32") -> Case:
    """Independent self-periodic Taylor-Green instances of n^3 cells: Mach
    uniform in M_range and Re log-uniform in Re_range from ``seed``, each
    with its own noise seed.  Per-instance mu0 = rho0 M / Re is in
    ``meta["mu0"]``; the case's gas model carries instance 0's.  Time steps
    are per instance (``meta`` has no dt: compute it from each instance's
    initial state)."""
    rng = np.random.default_rng(seed)
    Ms = rng.uniform(M_range[0], M_range[1], ninst)
    Res = np.exp(rng.uniform(np.log(Re_range[0]), np.log(Re_range[1]), ninst))
    qs, metrics, topos, mu0 = [], [], [], []
    for b in range(ninst):
        c = tgv(n=n, M0=float(Ms[b]), Re=float(Res[b]), gamma=gamma, Pr=Pr, visc_law=visc_law, noise=noise,
                seed=seed * 1000 + b + 1, limiter=limiter, cfl=cfl, precision=precision)
        qs.append(c.qs[0])
        metrics.append(c.metrics[0])
        topos.append(_self_periodic_topology(b))
        mu0.append(c.cfg.gas.mu0)
    gas = GasModel(gamma=gamma, R=1.0, mu0=mu0[0], T0=1.0 / gamma, Ts=(1.0 / gamma) * 110.4 / 288.15, Pr_lam=Pr,
                   visc_law=visc_law)
    cfg = Config(gas=gas, scheme=_scheme(limiter), bc_params={}, topology=tuple(topos), ghost=GHOST,
                 nan_check=False, cfl=cfl, precision=precision)
    return Case(name=f"ensemble{ninst}x{n}", qs=qs, metrics=metrics, cfg=cfg, cfl=cfl, steps=steps,
                meta={"n": n, "M0": [float(m) for m in Ms], "Re": [float(r) for r in Res], "mu0": mu0,
                      "h": 2.0 * math.pi / n})


def _noisy_freestream(shape, M, gamma, rng, noise):
    rho = np.ones(shape) * (1 + noise * rng.standard_normal(shape))
    p = np.full(shape, 1.0 / gamma) * (1 + noise * rng.standard_normal(shape))
    u = M + noise * M * rng.standard_normal(shape)
    v = noise * M * rng.standard_normal(shape)
    w = noise * M * rng.standard_normal(shape)
    return prim_to_cons_np(rho, u, v, w, p, gamma)


def wavy4(n=128, M=0.5, Re=1e4, gamma=1.4, Pr=0.72, noise=0.01, seed=0, amp=0.05, limiter="minmod",
          cfl=0.5, steps=100, metrics_fn=None, precision="f64") -> Case:
    """4 curvilinear blocks of n^3 cells, 2 x 2 in i-j, periodic in i, j, k."""
    g = GHOST
    N = 2 * n
    h = 2.0 * math.pi / N
    rng = np.random.default_rng(seed)
    qs, metrics, topos = [], [], []
    for bj in range(2):
        for bi in range(2):
            b = bi + 2 * bj
            e = g + 2  # coordinates extended by two more layers for the metric stencil
            I = bi * n + np.arange(-e, n + e, dtype=np.float64)
            J = bj * n + np.arange(-e, n + e, dtype=np.float64)
            K = np.arange(-e, n + e, dtype=np.float64)
            II, JJ, KK = np.meshgrid(I, J, K, indexing="ij")
            disp = amp * np.sin(2 * math.pi * II / N) * np.sin(2 * math.pi * JJ / N)
            xyz = np.stack([II * h + disp, JJ * h + disp, KK * h], axis=0)
            if metrics_fn is None:
                raise ValueError("wavy4 needs a metrics_fn")
            jac, kxyz, vol = metrics_fn(xyz)
            crop = (slice(2, -2),) * 3
            metrics.append((np.ascontiguousarray(jac[crop]), np.ascontiguousarray(kxyz[(slice(None),) * 2 + crop]),
                            np.ascontiguousarray(vol[crop])))
            qs.append(_noisy_freestream((n + 2 * g,) * 3, M, gamma, rng, noise))
            left, right = ((bi - 1) % 2) + 2 * bj, ((bi + 1) % 2) + 2 * bj
            down, up = bi + 2 * ((bj - 1) % 2), bi + 2 * ((bj + 1) % 2)
            nb = {Face.IMIN: (left, Face.IMAX, 0), Face.IMAX: (right, Face.IMIN, 0),
                  Face.JMIN: (down, Face.JMAX, 0), Face.JMAX: (up, Face.JMIN, 0),
                  Face.KMIN: (b, Face.KMAX, 0), Face.KMAX: (b, Face.KMIN, 0)}
            topos.append(BlockTopology(block_id=b, neighbors=nb, bc_type={f: BCType.CUT1TO1 for f in Face}))
    T0 = 1.0 / gamma
    gas = GasModel(gamma=gamma, R=1.0, mu0=M / Re, T0=T0, Ts=T0 * 110.4 / 288.15, Pr_lam=Pr,
                   visc_law="sutherland")
    cfg = Config(gas=gas, scheme=_scheme(limiter), bc_params={}, topology=tuple(topos), ghost=g,
                 nan_check=False, cfl=cfl, precision=precision)
    return Case(name=f"wavy4x{n}", qs=qs, metrics=metrics, cfg=cfg, cfl=cfl, steps=steps,
                meta={"n": n, "M": M, "Re": Re, "h": h})


_OPP = {Face.IMIN: Face.IMAX, Face.IMAX: Face.IMIN, Face.JMIN: Face.JMAX, Face.JMAX: Face.JMIN,
        Face.KMIN: Face.KMAX, Face.KMAX: Face.KMIN}


def tree24(nblocks=24, lo=16, hi=160, M=0.8, Re=5e4, gamma=1.4, Pr=0.72, noise=0.01, seed=0,
           limiter="minmod", cfl=0.5, steps=200, precision="f64") -> Case:
    """Uneven blocks on a random spanning tree of opposite-face interfaces."""
    g = GHOST
    rng = np.random.default_rng(seed)
    sizes = [list(rng.integers(lo, hi + 1, size=3))]
    nbrs = [dict()]
    for b in range(1, nblocks):
        while True:
            parent = int(rng.integers(0, b))
            face = Face(int(rng.integers(0, 6)))
            if face not in nbrs[parent]:
                break
        ax = int(face) // 2
        sz = list(sizes[parent])
        sz[ax] = int(rng.integers(lo, hi + 1))
        sizes.append(sz)
        nbrs.append(dict())
        nbrs[parent][face] = (b, _OPP[face], 0)
        nbrs[b][_OPP[face]] = (parent, face, 0)
    topos = []
    for b in range(nblocks):
        nb, bct = {}, {}
        for f in Face:
            if f in nbrs[b]:
                nb[f] = nbrs[b][f]
                bct[f] = BCType.CUT1TO1
            elif _OPP[f] not in nbrs[b]:
                nb[f] = (b, _OPP[f], 0)
                bct[f] = BCType.CUT1TO1
            else:
                nb[f] = None
                bct[f] = BCType.FARFIELD
        topos.append(BlockTopology(block_id=b, neighbors=nb, bc_type=bct))
    h = 2.0 * math.pi / 128
    qs, metrics = [], []
    for b in range(nblocks):
        shape = tuple(int(s) + 2 * g for s in sizes[b])
        qs.append(_noisy_freestream(shape, M, gamma, rng, noise))
        metrics.append(uniform_metrics(shape, h))
    q_inf = prim_to_cons_np(np.array(1.0), np.array(M), np.array(0.0), np.array(0.0), np.array(1.0 / gamma), gamma)
    T0 = 1.0 / gamma
    gas = GasModel(gamma=gamma, R=1.0, mu0=M / Re, T0=T0, Ts=T0 * 110.4 / 288.15, Pr_lam=Pr,
                   visc_law="sutherland")
    cfg = Config(gas=gas, scheme=_scheme(limiter), bc_params={f: {"q_inf": [float(x) for x in q_inf]} for f in Face},
                 topology=tuple(topos), ghost=g, nan_check=False, cfl=cfl, precision=precision)
    return Case(name=f"tree{nblocks}", qs=qs, metrics=metrics, cfg=cfg, cfl=cfl, steps=steps,
                meta={"sizes": [list(map(int, s)) for s in sizes], "M": M, "Re": Re, "h": h})

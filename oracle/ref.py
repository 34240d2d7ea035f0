"""FP64 CPU restatement of famrdp_jax's RHS + TVD-RK3 step path.

TEST INFRASTRUCTURE ONLY -- the checker, never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline legs) may use it.

Every function below restates one function of the reference
(LucasLu123/famrdp-jax; paths are relative to that project) with the same
index semantics, the same operation order and the same clamps.  The code is
written once against a small array-backend adapter so that the same statement
runs on NumPy (``NP``: the parity oracle) and on PyTorch-CPU (``TORCH``: a
multithreaded twin whose autograd stands in for ``jax.grad``).

Extensions that the reference does not have (each marked "NEW" below) are the
definitions the GPU path must agree with: the constant-viscosity law, the
CFL time step, the kinetic-energy objective, the residual and the finiteness
check.

Topology conventions follow the reference exactly: ``topo.neighbors`` is an
insertion-ordered ``dict[face -> None | (block_id, src_face, orient)]`` and
``topo.bc_type`` a ``dict[face -> bc]``, with faces 0..5 = IMIN, IMAX, JMIN,
JMAX, KMIN, KMAX and bc codes CUT1TO1=-1, WALL=2, SYMMETRY=3, FARFIELD=4
(``core/constants.py:4-12,54-60``).
"""
from __future__ import annotations

import math

import numpy as np

# core/constants.py:4-12, :54-60
CUT1TO1, WALL, SYMMETRY, FARFIELD = -1, 2, 3, 4
IMIN, IMAX, JMIN, JMAX, KMIN, KMAX = 0, 1, 2, 3, 4, 5
FACES = (IMIN, IMAX, JMIN, JMAX, KMIN, KMAX)


# ---------------------------------------------------------------------------
# array-backend adapter
# ---------------------------------------------------------------------------
class _NumpyOps:
    name = "numpy"

    def asarray(self, x):
        return np.asarray(x, dtype=np.float64)

    def roll(self, a, shift, axis):
        return np.roll(a, shift, axis=axis)

    def stack(self, xs, axis=0):
        return np.stack(xs, axis=axis)

    def maximum(self, a, b):
        return np.maximum(a, b)

    def minimum(self, a, b):
        return np.minimum(a, b)

    def abs(self, a):
        return np.abs(a)

    def sign(self, a):
        return np.sign(a)

    def sqrt(self, a):
        return np.sqrt(a)

    def where(self, c, a, b):
        return np.where(c, a, b)

    def einsum(self, spec, *ops):
        return np.einsum(spec, *ops)

    def zeros_like(self, a):
        return np.zeros_like(a)

    def ones_like(self, a):
        return np.ones_like(a)

    def sum0(self, a):
        return np.sum(a, axis=0)

    def transpose(self, a, perm):
        return np.transpose(a, perm)

    def det(self, m):
        return np.linalg.det(m)

    def inv(self, m):
        return np.linalg.inv(m)

    def add_at(self, arr, idx, val):
        out = arr.copy()
        out[idx] = out[idx] + val
        return out

    def set_at(self, arr, idx, val):
        out = arr.copy()
        out[idx] = val
        return out

    def full_vec(self, vals):
        return np.asarray(vals, dtype=np.float64)

    def pow(self, a, e):
        return a ** e


class _TorchOps:
    name = "torch"

    def __init__(self):
        import torch
        self.t = torch

    def asarray(self, x):
        t = self.t
        if isinstance(x, t.Tensor):
            return x.to(t.float64)
        return t.as_tensor(np.asarray(x, dtype=np.float64))

    def roll(self, a, shift, axis):
        return self.t.roll(a, shift, dims=axis)

    def stack(self, xs, axis=0):
        t = self.t
        xs = [x if isinstance(x, t.Tensor) else t.as_tensor(x, dtype=t.float64) for x in xs]
        shape = None
        for x in xs:
            if x.dim() > 0:
                shape = x.shape
                break
        if shape is not None:
            xs = [x.expand(shape) if x.dim() == 0 else x for x in xs]
        return t.stack(xs, dim=axis)

    def _t(self, x, like):
        t = self.t
        if isinstance(x, t.Tensor):
            return x
        return t.as_tensor(x, dtype=like.dtype)

    def maximum(self, a, b):
        t = self.t
        if not isinstance(b, t.Tensor):
            return t.clamp(a, min=b)
        if not isinstance(a, t.Tensor):
            return t.clamp(b, min=a)
        return t.maximum(a, b)

    def minimum(self, a, b):
        return self.t.minimum(a, b)

    def abs(self, a):
        return self.t.abs(a)

    def sign(self, a):
        return self.t.sign(a)

    def sqrt(self, a):
        t = self.t
        return t.sqrt(a) if isinstance(a, t.Tensor) else math.sqrt(a)

    def where(self, c, a, b):
        t = self.t
        if not isinstance(a, t.Tensor):
            a = t.as_tensor(a, dtype=t.float64)
        if not isinstance(b, t.Tensor):
            b = t.as_tensor(b, dtype=t.float64)
        return t.where(c, a, b)

    def einsum(self, spec, *ops):
        return self.t.einsum(spec, *ops)

    def zeros_like(self, a):
        return self.t.zeros_like(a)

    def ones_like(self, a):
        return self.t.ones_like(a)

    def sum0(self, a):
        return self.t.sum(a, dim=0)

    def transpose(self, a, perm):
        return a.permute(*perm)

    def det(self, m):
        return self.t.linalg.det(m)

    def inv(self, m):
        return self.t.linalg.inv(m)

    def add_at(self, arr, idx, val):
        out = arr.clone()
        out[idx] = out[idx] + val
        return out

    def set_at(self, arr, idx, val):
        out = arr.clone()
        out[idx] = val
        return out

    def full_vec(self, vals):
        t = self.t
        if isinstance(vals, t.Tensor):
            return vals.to(t.float64)
        return t.as_tensor(np.asarray(vals, dtype=np.float64))

    def pow(self, a, e):
        return a ** e


# ---------------------------------------------------------------------------
# the restatement
# ---------------------------------------------------------------------------
class Ref:
    """The reference's hot path, restated over one array backend ``X``."""

    def __init__(self, ops):
        self.X = ops

    # -- physics/eos.py -----------------------------------------------------
    def prim_to_cons(self, prim, gamma):
        """physics/eos.py:5-9"""
        X = self.X
        rho = prim[0]; u = prim[1]; v = prim[2]; w = prim[3]; p = prim[4]
        ke = 0.5 * (u * u + v * v + w * w)
        rhoE = p / (gamma - 1.0) + rho * ke
        return X.stack([rho, rho * u, rho * v, rho * w, rhoE], axis=0)

    def cons_to_prim(self, q, gamma):
        """physics/eos.py:12-17 (no density clamp)."""
        X = self.X
        rho = q[0]
        u = q[1] / rho; v = q[2] / rho; w = q[3] / rho
        ke = 0.5 * (u * u + v * v + w * w)
        p = (gamma - 1.0) * (q[4] - rho * ke)
        return X.stack([rho, u, v, w, p], axis=0)

    def speed_of_sound(self, rho, p, gamma):
        """physics/eos.py:20-21"""
        return self.X.sqrt(gamma * p / rho)

    def sutherland_viscosity(self, T, mu0, T0, Ts):
        """physics/eos.py:24-25"""
        return mu0 * (T / T0) ** 1.5 * (T0 + Ts) / (T + Ts)

    # -- physics/reconstruct/muscl2.py ---------------------------------------
    def minmod(self, a, b):
        """physics/reconstruct/muscl2.py:5-7"""
        X = self.X
        s = X.sign(a) * X.maximum(X.sign(a) * X.sign(b), 0.0)
        return s * X.minimum(X.abs(a), X.abs(b))

    def vanleer(self, a, b):
        """physics/reconstruct/muscl2.py:10-12"""
        X = self.X
        safe_denom = X.where(X.abs(a + b) > 1e-30, a + b, 1.0)
        return X.where(a * b > 0.0, 2.0 * a * b / safe_denom, 0.0)

    def muscl2_reconstruct(self, pv, *, axis, limiter="minmod"):
        """physics/reconstruct/muscl2.py:18-37.  Face f in [0, n-4] lies between
        cells f+1 and f+2 along ``axis``; an unknown limiter raises KeyError."""
        lim = {"minmod": self.minmod, "vanleer": self.vanleer}[limiter]
        n = pv.shape[axis]

        def slc(start, end):
            idx = [slice(None)] * pv.ndim
            idx[axis] = slice(start, end)
            return pv[tuple(idx)]

        pmm = slc(0, n - 3)
        pc = slc(1, n - 2)
        pp1 = slc(2, n - 1)
        pp2 = slc(3, n)
        slope_L = lim(pc - pmm, pp1 - pc)
        slope_R = lim(pp1 - pc, pp2 - pp1)
        return pc + 0.5 * slope_L, pp1 - 0.5 * slope_R

    # -- flux/roe.py --------------------------------------------------------
    def physical_flux(self, U, n, gamma):
        """flux/roe.py:5-18 (density clamped at 1e-300)."""
        X = self.X
        rho = X.maximum(U[0], 1e-300)
        u = U[1] / rho; v = U[2] / rho; w = U[3] / rho
        ke = 0.5 * (u * u + v * v + w * w)
        p = (gamma - 1.0) * (U[4] - rho * ke)
        un = u * n[0] + v * n[1] + w * n[2]
        H = (U[4] + p) / rho
        return X.stack([
            rho * un,
            rho * u * un + p * n[0],
            rho * v * un + p * n[1],
            rho * w * un + p * n[2],
            rho * H * un,
        ], axis=0)

    def roe_flux(self, UL, UR, nxyz, *, gamma, eps_entropy=0.1):
        """flux/roe.py:21-85: Roe averages, Harten fix on lambda_1/lambda_5,
        the reference's shear term ``dvt`` and 0.5(FL+FR) - 0.5|A|dU."""
        X = self.X
        rhoL = X.maximum(UL[0], 1e-300)
        rhoR = X.maximum(UR[0], 1e-300)
        uL, vL, wL = UL[1] / rhoL, UL[2] / rhoL, UL[3] / rhoL
        uR, vR, wR = UR[1] / rhoR, UR[2] / rhoR, UR[3] / rhoR
        keL = 0.5 * (uL * uL + vL * vL + wL * wL); keR = 0.5 * (uR * uR + vR * vR + wR * wR)
        pL = (gamma - 1.0) * (UL[4] - rhoL * keL); pR = (gamma - 1.0) * (UR[4] - rhoR * keR)
        HL = (UL[4] + pL) / rhoL; HR = (UR[4] + pR) / rhoR

        sqL = X.sqrt(rhoL); sqR = X.sqrt(rhoR)
        ss = X.maximum(sqL + sqR, 1e-150)
        u_h = (sqL * uL + sqR * uR) / ss
        v_h = (sqL * vL + sqR * vR) / ss
        w_h = (sqL * wL + sqR * wR) / ss
        H_h = (sqL * HL + sqR * HR) / ss
        q2 = u_h ** 2 + v_h ** 2 + w_h ** 2
        c2_safe = X.maximum((gamma - 1.0) * (H_h - 0.5 * q2), 1e-30)
        c_h = X.sqrt(c2_safe)
        un_h = u_h * nxyz[0] + v_h * nxyz[1] + w_h * nxyz[2]
        rho_h = sqL * sqR

        eps = eps_entropy * (X.abs(un_h) + c_h)

        def harten(lam):
            return X.where(X.abs(lam) >= eps, X.abs(lam), 0.5 * (lam ** 2 / eps + eps))

        lam1 = un_h - c_h; lam2 = un_h; lam5 = un_h + c_h
        al1 = harten(lam1); al2 = X.abs(lam2); al5 = harten(lam5)

        dU = UR - UL
        dp = (gamma - 1.0) * (dU[4] - u_h * dU[1] - v_h * dU[2] - w_h * dU[3] + 0.5 * q2 * dU[0])
        dun = (dU[1] * nxyz[0] + dU[2] * nxyz[1] + dU[3] * nxyz[2]) - un_h * dU[0]
        a1 = (dp - rho_h * c_h * dun) / (2.0 * c2_safe)
        a5 = (dp + rho_h * c_h * dun) / (2.0 * c2_safe)
        a23 = dU[0] - dp / c2_safe

        one = X.ones_like(u_h)
        R1 = X.stack([one, u_h - c_h * nxyz[0], v_h - c_h * nxyz[1], w_h - c_h * nxyz[2], H_h - c_h * un_h])
        R5 = X.stack([one, u_h + c_h * nxyz[0], v_h + c_h * nxyz[1], w_h + c_h * nxyz[2], H_h + c_h * un_h])
        R2 = X.stack([one, u_h, v_h, w_h, 0.5 * q2])

        du_t = dU[1] / rho_h - u_h * dU[0] / rho_h
        dv_t = dU[2] / rho_h - v_h * dU[0] / rho_h
        dw_t = dU[3] / rho_h - w_h * dU[0] / rho_h
        dun_full = du_t * nxyz[0] + dv_t * nxyz[1] + dw_t * nxyz[2]
        dvt = X.stack([
            X.zeros_like(u_h),
            rho_h * (du_t - dun_full * nxyz[0]),
            rho_h * (dv_t - dun_full * nxyz[1]),
            rho_h * (dw_t - dun_full * nxyz[2]),
            rho_h * (u_h * (du_t - dun_full * nxyz[0]) + v_h * (dv_t - dun_full * nxyz[1])
                     + w_h * (dw_t - dun_full * nxyz[2])),
        ])

        absA_dU = al1 * a1 * R1 + al5 * a5 * R5 + al2 * (a23 * R2 + dvt)
        FL = self.physical_flux(UL, nxyz, gamma)
        FR = self.physical_flux(UR, nxyz, gamma)
        return 0.5 * (FL + FR) - 0.5 * absA_dU

    # -- rhs/invscd.py ------------------------------------------------------
    def compute_invscd_rhs(self, q, kxyz, vol, *, ghost, gamma, reconstruct="muscl2",
                           flux="roe", limiter="minmod"):
        """rhs/invscd.py:18-133.  For each axis: MUSCL on primitives, face normal
        = mean of the two adjacent cells' kxyz row (:87-89), unit normal and
        |n| + 1e-300 (:93-94), Roe (:97), times |n| (:100), difference and
        division by vol + 1e-300 (:119-126), added at cells [2, n-3] along the
        axis and at EVERY index of the other two axes (:129-131)."""
        X = self.X
        pv = self.cons_to_prim(q, gamma)
        rhs = X.zeros_like(q)
        for axis in (1, 2, 3):
            n = pv.shape[axis]
            d = axis - 1
            pv_L, pv_R = self.muscl2_reconstruct(pv, axis=axis, limiter=limiter)
            UL = self.prim_to_cons(pv_L, gamma)
            UR = self.prim_to_cons(pv_R, gamma)
            k_dir = kxyz[d]

            def slc4(arr, start, end, ax=axis):
                idx = [slice(None)] * arr.ndim
                idx[ax] = slice(start, end if end != 0 else None)
                return arr[tuple(idx)]

            def slc3(arr, start, end, ax=d):
                idx = [slice(None)] * arr.ndim
                idx[ax] = slice(start, end if end != 0 else None)
                return arr[tuple(idx)]

            n_face = 0.5 * (slc4(k_dir, 1, n - 2) + slc4(k_dir, 2, n - 1))
            n_mag = X.sqrt(X.sum0(n_face ** 2)) + 1e-300
            n_unit = n_face / n_mag[None]
            F_face = self.roe_flux(UL, UR, n_unit, gamma=gamma)
            F_area = F_face * n_mag[None]
            div = slc4(F_area, 1, None) - slc4(F_area, 0, -1)
            vol_cell = slc3(vol, 2, n - 2)
            rhs_dir = -div / (vol_cell[None] + 1e-300)
            idx = [slice(None)] * rhs.ndim
            idx[axis] = slice(2, n - 2)
            rhs = X.add_at(rhs, tuple(idx), rhs_dir)
        return rhs

    # -- rhs/viscous.py -----------------------------------------------------
    def _central2(self, f, axis):
        """rhs/viscous.py:12-16: periodic roll over the PADDED array."""
        return 0.5 * (self.X.roll(f, -1, axis) - self.X.roll(f, 1, axis))

    def compute_viscous_rhs(self, q, kxyz, *, gas, ghost):
        """rhs/viscous.py:19-119, evaluated on every padded cell.

        NEW: ``gas.visc_law == "constant"`` replaces Sutherland's law (:37) by
        mu = mu0 everywhere (the reference always uses Sutherland)."""
        X = self.X
        pv = self.cons_to_prim(q, gas.gamma)
        rho = pv[0]; u = pv[1]; v = pv[2]; w = pv[3]; p = pv[4]
        T = p / X.maximum(rho * gas.R, 1e-300)
        if getattr(gas, "visc_law", "sutherland") == "constant":
            mu = gas.mu0 * X.ones_like(T)
        else:
            mu = self.sutherland_viscosity(T, gas.mu0, gas.T0, gas.Ts)
        cp = gas.gamma * gas.R / (gas.gamma - 1.0)
        kappa = cp * mu / gas.Pr_lam

        def grad_xyz(phi):
            dphi_dxi = X.stack([self._central2(phi, a) for a in (0, 1, 2)], axis=0)
            return X.einsum("lijk,lmijk->mijk", dphi_dxi, kxyz)

        du = grad_xyz(u); dv = grad_xyz(v); dw = grad_xyz(w); dT = grad_xyz(T)
        div_u = du[0] + dv[1] + dw[2]
        tau = X.stack([
            X.stack([2 * mu * (du[0] - div_u / 3.0), mu * (du[1] + dv[0]), mu * (du[2] + dw[0])]),
            X.stack([mu * (du[1] + dv[0]), 2 * mu * (dv[1] - div_u / 3.0), mu * (dv[2] + dw[1])]),
            X.stack([mu * (du[2] + dw[0]), mu * (dv[2] + dw[1]), 2 * mu * (dw[2] - div_u / 3.0)]),
        ])
        heat = -kappa * dT
        vel = X.stack([u, v, w])

        def div_physical_scalar(f):
            result = X.zeros_like(f[0])
            for j in range(3):
                df = X.stack([self._central2(f[j], a) for a in (0, 1, 2)], axis=0)
                result = result + X.einsum("lijk,lijk->ijk", df, kxyz[:, j])
            return result

        rhs_mom = [div_physical_scalar(tau[i]) for i in range(3)]
        G_energy = X.stack([X.sum0(vel * tau[:, j]) - heat[j] for j in range(3)])
        rhs_energy = div_physical_scalar(G_energy)
        return X.stack([X.zeros_like(u), rhs_mom[0], rhs_mom[1], rhs_mom[2], rhs_energy], axis=0)

    # -- solver/step.py -----------------------------------------------------
    def rhs_block(self, q, kxyz, vol, cfg):
        """solver/step.py:10-15: inviscid + viscous."""
        inv = self.compute_invscd_rhs(q, kxyz, vol, ghost=cfg.ghost, gamma=cfg.gas.gamma,
                                      reconstruct=cfg.scheme.reconstruct, flux=cfg.scheme.flux,
                                      limiter=cfg.scheme.limiter)
        vis = self.compute_viscous_rhs(q, kxyz, gas=cfg.gas, ghost=cfg.ghost)
        return inv + vis

    # -- time/rk.py ---------------------------------------------------------
    def rk3_step(self, q, L, dt):
        """time/rk.py:5-20 (Shu-Osher TVD-RK3)."""
        q1 = q + dt * L(q)
        q2 = 0.75 * q + 0.25 * (q1 + dt * L(q1))
        return (1.0 / 3.0) * q + (2.0 / 3.0) * (q2 + dt * L(q2))

    # -- mesh/halo.py -------------------------------------------------------
    _FACE_AXIS = {IMIN: 1, IMAX: 1, JMIN: 2, JMAX: 2, KMIN: 3, KMAX: 3}

    def _ghost_slice(self, face, g):
        """mesh/halo.py:19-23"""
        return slice(0, g) if face in (IMIN, JMIN, KMIN) else slice(-g, None)

    def _interior_adj_slice(self, face, g):
        """mesh/halo.py:26-33"""
        return slice(g, 2 * g) if face in (IMIN, JMIN, KMIN) else slice(-2 * g, -g)

    def _copy_face(self, tgt_q, src_q, tgt_face, src_face, g):
        """mesh/halo.py:36-53"""
        idx_t = [slice(None)] * tgt_q.ndim
        idx_s = [slice(None)] * src_q.ndim
        idx_t[self._FACE_AXIS[int(tgt_face)]] = self._ghost_slice(int(tgt_face), g)
        idx_s[self._FACE_AXIS[int(src_face)]] = self._interior_adj_slice(int(src_face), g)
        src = src_q[tuple(idx_s)]
        tshape = tuple(tgt_q[tuple(idx_t)].shape)
        if tuple(src.shape) != tshape:
            raise ValueError(f"halo slab shape mismatch: target {tshape} vs source {tuple(src.shape)}")
        return self.X.set_at(tgt_q, tuple(idx_t), src)

    def halo_exchange(self, qs, topos, ghost):
        """mesh/halo.py:56-92: faces in dict insertion order, each read from the
        PRE-exchange source array (:89-90), so later faces overwrite edges and
        corners; ``orient != 0`` raises NotImplementedError (:86-87)."""
        id_to_idx = {t.block_id: i for i, t in enumerate(topos)}
        orig = list(qs)
        out = list(qs)
        for i, topo in enumerate(topos):
            for face, info in topo.neighbors.items():
                if info is None:
                    continue
                if topo.bc_type.get(face) != CUT1TO1:
                    continue
                nb_id, src_face, orient = info
                if orient != 0:
                    raise NotImplementedError(f"orient={orient} not supported in stage 1")
                out[i] = self._copy_face(out[i], orig[id_to_idx[nb_id]], face, src_face, ghost)
        return out

    # -- physics/bc ---------------------------------------------------------
    def _ghost_indices(self, face, g, n):
        """physics/bc/base.py:15-27"""
        if face in (IMIN, JMIN, KMIN):
            outer = list(range(g))
            inner = [2 * g - 1 - o for o in outer]
        else:
            outer = list(range(n - 1, n - 1 - g, -1))
            inner = [n - 2 * g + (n - 1 - o) for o in outer]
        return outer, inner

    def apply_farfield(self, q, face, g, q_inf):
        """physics/bc/farfield.py:7-21: the outer ``g`` layers := q_inf."""
        X = self.X
        ax = self._FACE_AXIS[int(face)]
        outer, _ = self._ghost_indices(int(face), g, q.shape[ax])
        qv = X.full_vec(q_inf)
        for o in outer:
            idx = [slice(None)] * q.ndim
            idx[ax] = o
            shape = [1] * (q.ndim - 1)
            shape[0] = 5
            q = X.set_at(q, tuple(idx), qv.reshape(shape) * X.ones_like(q[tuple(idx)]))
        return q

    def _mirror_ghost(self, q, face, g, sign_mask):
        """physics/bc/wall.py:7-24"""
        X = self.X
        ax = self._FACE_AXIS[int(face)]
        outer, inner = self._ghost_indices(int(face), g, q.shape[ax])
        shape = [1] * (q.ndim - 1)
        shape[0] = 5
        sgn = X.full_vec(sign_mask).reshape(shape)
        for o, n in zip(outer, inner):
            idx_o = [slice(None)] * q.ndim
            idx_n = [slice(None)] * q.ndim
            idx_o[ax] = o
            idx_n[ax] = n
            q = X.set_at(q, tuple(idx_o), q[tuple(idx_n)] * sgn)
        return q

    def apply_wall_noslip_adiabatic(self, q, face, g):
        """physics/bc/wall.py:27-29"""
        return self._mirror_ghost(q, face, g, [1.0, -1.0, -1.0, -1.0, 1.0])

    def apply_wall_noslip_isothermal(self, q, face, g, T_wall, gamma, R):
        """physics/bc/wall.py:32-55"""
        X = self.X
        ax = self._FACE_AXIS[int(face)]
        outer, inner = self._ghost_indices(int(face), g, q.shape[ax])
        for o, n in zip(outer, inner):
            idx_o = [slice(None)] * q.ndim
            idx_n = [slice(None)] * q.ndim
            idx_o[ax] = o
            idx_n[ax] = n
            qi = q[tuple(idx_n)]
            rho_i = qi[0]
            ke_i = 0.5 * (qi[1] ** 2 + qi[2] ** 2 + qi[3] ** 2) / rho_i
            p_i = (gamma - 1.0) * (qi[4] - ke_i)
            p_g = p_i
            rho_g = p_g / (R * T_wall)
            scale = rho_g / rho_i
            rhou_g = -qi[1] * scale
            rhov_g = -qi[2] * scale
            rhow_g = -qi[3] * scale
            ke_g = 0.5 * (rhou_g ** 2 + rhov_g ** 2 + rhow_g ** 2) / rho_g
            rhoE_g = p_g / (gamma - 1.0) + ke_g
            q = X.set_at(q, tuple(idx_o), X.stack([rho_g, rhou_g, rhov_g, rhow_g, rhoE_g], axis=0))
        return q

    def apply_symmetry_plane(self, q, face, g):
        """physics/bc/symmetry.py:8-11 (also wall.py:58-61 ``apply_wall_slip``)."""
        sign = [1.0] * 5
        sign[{IMIN: 1, IMAX: 1, JMIN: 2, JMAX: 2, KMIN: 3, KMAX: 3}[int(face)]] = -1.0
        return self._mirror_ghost(q, face, g, sign)

    def apply_bc(self, q, topo, cfg):
        """physics/bc/dispatch.py:11-32: faces in Face enum order, CUT1TO1 and
        absent faces skipped."""
        g = cfg.ghost
        for face in FACES:
            bct = _bc_lookup(topo.bc_type, face)
            if bct is None or bct == CUT1TO1:
                continue
            bc_p = _bc_lookup(cfg.bc_params, face) or {}
            if bct == WALL:
                if bc_p.get("wall_type", "adiabatic") == "isothermal":
                    q = self.apply_wall_noslip_isothermal(q, face, g, bc_p.get("T_wall", 300.0),
                                                          cfg.gas.gamma, cfg.gas.R)
                else:
                    q = self.apply_wall_noslip_adiabatic(q, face, g)
            elif bct == SYMMETRY:
                q = self.apply_symmetry_plane(q, face, g)
            elif bct == FARFIELD:
                q = self.apply_farfield(q, face, g, bc_p.get("q_inf", [1.0, 0.0, 0.0, 0.0, 2.5]))
        return q

    # -- solver/step.py:18-56 ----------------------------------------------
    def step(self, qs, metrics, cfg, dt, rhs_map=None):
        """solver/step.py:18-56: halo + BC once per STEP, then three RK stages
        over all padded cells.  ``metrics`` is a sequence of (kxyz, vol).
        ``rhs_map(qs) -> [rhs_block of each q]`` may evaluate the blocks'
        right-hand sides elsewhere (e.g. a process pool); the default
        evaluates them here, one after another."""
        qs = self.halo_exchange(list(qs), cfg.topology, cfg.ghost)
        qs = [self.apply_bc(q, t, cfg) for q, t in zip(qs, cfg.topology)]

        def L(qt):
            if rhs_map is not None:
                return rhs_map(qt)
            return [self.rhs_block(q, m[0], m[1], cfg) for q, m in zip(qt, metrics)]

        L0 = L(qs)
        qs1 = [q + dt * r for q, r in zip(qs, L0)]
        L1 = L(qs1)
        qs2 = [0.75 * q + 0.25 * (q1 + dt * r) for q, q1, r in zip(qs, qs1, L1)]
        L2 = L(qs2)
        return [(1.0 / 3.0) * q + (2.0 / 3.0) * (q2 + dt * r) for q, q2, r in zip(qs, qs2, L2)]

    # -- mesh/metric.py -----------------------------------------------------
    def _central4(self, f, axis):
        """mesh/metric.py:18-28 (roll wraps at the array ends)."""
        X = self.X
        fp2 = X.roll(f, -2, axis); fp1 = X.roll(f, -1, axis)
        fm1 = X.roll(f, 1, axis); fm2 = X.roll(f, 2, axis)
        return (-fp2 + 8.0 * fp1 - 8.0 * fm1 + fm2) / 12.0

    def compute_metrics(self, xyz, *, ghost):
        """mesh/metric.py:31-70: returns (jac, kxyz, vol) with
        kxyz[l, m] = d xi_l / d x_m and vol = |jac|."""
        X = self.X
        J = X.stack([X.stack([self._central4(xyz[m], l) for l in range(3)], axis=0)
                     for m in range(3)], axis=0)
        Jc = X.transpose(J, (2, 3, 4, 0, 1))
        jac = X.det(Jc)
        kxyz = X.transpose(X.inv(Jc), (3, 4, 0, 1, 2))
        return jac, kxyz, X.abs(jac)

    # -- NEW: definitions the reference does not have ------------------------
    def cfl_dt(self, qs, metrics, gamma, cfl, ghost):
        """NEW.  One global dt = CFL / max over interior cells of
        sum_a (|u . n_a| + c) |kxyz[a,:]| / vol, consistent with the
        reference's inviscid scaling (rhs/invscd.py:93-100,126)."""
        lam_max = 0.0
        g = ghost
        for q, (kxyz, vol) in zip(qs, metrics):
            sl = (slice(g, -g),) * 3
            qi = q[(slice(None),) + sl]
            k = kxyz[(slice(None), slice(None)) + sl]
            vi = vol[sl]
            rho = qi[0]
            u = qi[1] / rho; v = qi[2] / rho; w = qi[3] / rho
            p = (gamma - 1.0) * (qi[4] - rho * 0.5 * (u * u + v * v + w * w))
            c = np.sqrt(gamma * p / rho)
            lam = 0.0
            for a in range(3):
                kmag = np.sqrt(k[a, 0] ** 2 + k[a, 1] ** 2 + k[a, 2] ** 2)
                un = (u * k[a, 0] + v * k[a, 1] + w * k[a, 2]) / kmag
                lam = lam + (np.abs(un) + c) * kmag
            lam_max = max(lam_max, float(np.max(lam / vi)))
        return cfl / lam_max

    def kinetic_energy(self, qs, metrics, ghost):
        """NEW.  J = sum over interior cells of vol * 0.5 (q1^2+q2^2+q3^2)/q0."""
        X = self.X
        g = ghost
        total = 0.0
        for q, (kxyz, vol) in zip(qs, metrics):
            sl = (slice(g, q.shape[1] - g), slice(g, q.shape[2] - g), slice(g, q.shape[3] - g))
            qi = q[(slice(None),) + sl]
            e = vol[sl] * (0.5 * (qi[1] * qi[1] + qi[2] * qi[2] + qi[3] * qi[3]) / qi[0])
            total = total + e.sum()
        return total

    def residual(self, rhs, ghost):
        """NEW.  Per-variable RMS of an RHS over the interior cells."""
        g = ghost
        r = np.asarray(rhs)[:, g:-g, g:-g, g:-g]
        return np.sqrt(np.mean(r * r, axis=(1, 2, 3)))


def _bc_lookup(d, face):
    """Dict lookup by face that accepts int or IntEnum keys (the reference
    uses ``Face`` members, which hash like their int values)."""
    if d is None:
        return None
    return d.get(face)


NP = Ref(_NumpyOps())


class _LazyTorch:
    _ref = None

    def __getattr__(self, name):
        if _LazyTorch._ref is None:
            _LazyTorch._ref = Ref(_TorchOps())
        return getattr(_LazyTorch._ref, name)


TORCH = _LazyTorch()

"""The reference's own known-answer and invariance tests (famrdp_jax tests/),
restated against the CPU oracle, on both of its backends.  They pin the
oracle before it is trusted as the parity checker of the CUDA path."""
import math

import numpy as np
import pytest

from oracle.ref import CUT1TO1, FARFIELD, WALL, SYMMETRY, IMIN, IMAX, JMIN, JMAX, KMIN, KMAX, NP, TORCH

BACKENDS = [pytest.param(NP, id="numpy"), pytest.param(TORCH, id="torch")]


def A(ref, x):
    return ref.X.asarray(x)


def N(x):
    import torch
    return x.detach().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


class _Gas:
    gamma = 1.4
    R = 287.058
    mu0 = 1.71608e-5
    T0 = 273.15
    Ts = 110.4
    Pr_lam = 0.72
    visc_law = "sutherland"


class _Topo:
    def __init__(self, block_id, neighbors, bc_type):
        self.block_id, self.neighbors, self.bc_type = block_id, neighbors, bc_type


class _Scheme:
    reconstruct, flux, rk_order, limiter = "muscl2", "roe", 3, "minmod"


class _Cfg:
    def __init__(self, topology, bc_params, ghost=2):
        self.gas, self.scheme, self.topology, self.bc_params, self.ghost = _Gas(), _Scheme(), topology, bc_params, ghost


@pytest.mark.parametrize("ref", BACKENDS)
def test_roe_symmetric_states(ref):
    """tests/flux/test_roe.py:5-14"""
    g = 1.4
    rho, u, v, w, p = 1.0, 50.0, 0.0, 0.0, 101325.0
    rhoE = p / (g - 1.0) + 0.5 * rho * (u ** 2 + v ** 2 + w ** 2)
    U = A(ref, [rho, rho * u, rho * v, rho * w, rhoE])
    F = ref.roe_flux(U, U, A(ref, [1.0, 0.0, 0.0]), gamma=g)
    exp = [rho * u, rho * u * u + p, rho * u * v, rho * u * w, u * (rhoE + p)]
    np.testing.assert_allclose(N(F), exp, rtol=1e-12)


@pytest.mark.parametrize("ref", BACKENDS)
def test_roe_arbitrary_normal(ref):
    """tests/flux/test_roe.py:16-26"""
    g = 1.4
    rho, u, v, w, p = 1.0, 30.0, 20.0, 10.0, 50000.0
    rhoE = p / (g - 1.0) + 0.5 * rho * (u ** 2 + v ** 2 + w ** 2)
    U = A(ref, [rho, rho * u, rho * v, rho * w, rhoE])
    n = [0.6, 0.8, 0.0]
    F = ref.roe_flux(U, U, A(ref, n), gamma=g)
    un = u * n[0] + v * n[1] + w * n[2]
    H = (rhoE + p) / rho
    exp = [rho * un, rho * u * un + p * n[0], rho * v * un + p * n[1], rho * w * un + p * n[2], rho * H * un]
    np.testing.assert_allclose(N(F), exp, rtol=1e-12)


@pytest.mark.parametrize("ref", BACKENDS)
def test_minmod(ref):
    """tests/physics/test_muscl2.py:5-12"""
    np.testing.assert_allclose(N(ref.minmod(A(ref, [1.0, -1.0]), A(ref, [-1.0, 1.0]))), 0.0, atol=1e-15)
    assert float(ref.minmod(A(ref, 2.0), A(ref, 5.0))) == 2.0
    assert float(ref.minmod(A(ref, -3.0), A(ref, -7.0))) == -3.0


@pytest.mark.parametrize("ref", BACKENDS)
def test_muscl2_linear_profile(ref):
    """tests/physics/test_muscl2.py:14-22"""
    pv = np.stack([np.linspace(1.0, 10.0, 10)] * 5, axis=0)[:, :, None, None]
    L, R = ref.muscl2_reconstruct(A(ref, pv), axis=1, limiter="minmod")
    np.testing.assert_allclose(N(L)[0, :, 0, 0], N(R)[0, :, 0, 0], rtol=1e-12)


def test_muscl2_unknown_limiter():
    with pytest.raises(KeyError):
        NP.muscl2_reconstruct(np.zeros((5, 6, 1, 1)), axis=1, limiter="superbee")


@pytest.mark.parametrize("ref", BACKENDS)
def test_eos_roundtrip(ref):
    """tests/physics/test_eos.py:6-12"""
    prim = np.array([1.225, 50.0, 10.0, -5.0, 101325.0])[:, None, None, None]
    back = ref.cons_to_prim(ref.prim_to_cons(A(ref, prim), 1.4), 1.4)
    np.testing.assert_allclose(N(back), prim, rtol=1e-14)


def test_speed_of_sound():
    """tests/physics/test_eos.py:14-17"""
    np.testing.assert_allclose(float(NP.speed_of_sound(1.225, 101325.0, 1.4)), (1.4 * 101325.0 / 1.225) ** 0.5,
                               rtol=1e-12)


def _identity_metrics(ni, nj, nk):
    kxyz = np.zeros((3, 3, ni, nj, nk))
    for d in range(3):
        kxyz[d, d] = 1.0
    return kxyz, np.ones((ni, nj, nk))


def _uniform_q(ni, nj, nk, rho, u, v, w, p, g=1.4):
    rhoE = p / (g - 1.0) + 0.5 * rho * (u ** 2 + v ** 2 + w ** 2)
    q = np.zeros((5, ni, nj, nk))
    q[0], q[1], q[2], q[3], q[4] = rho, rho * u, rho * v, rho * w, rhoE
    return q


@pytest.mark.parametrize("ref", BACKENDS)
def test_uniform_flow_zero_invscd_rhs(ref):
    """tests/rhs/test_invscd.py:7-23"""
    q = _uniform_q(16, 12, 10, 1.225, 50.0, 0.0, 0.0, 101325.0)
    kxyz, vol = _identity_metrics(16, 12, 10)
    rhs = ref.compute_invscd_rhs(A(ref, q), A(ref, kxyz), A(ref, vol), ghost=2, gamma=1.4, limiter="minmod")
    np.testing.assert_allclose(N(rhs)[:, 4:-4, 4:-4, 4:-4], 0.0, atol=1e-8)


@pytest.mark.parametrize("ref", BACKENDS)
def test_static_isothermal_zero_viscous_rhs(ref):
    """tests/rhs/test_viscous.py:7-20"""
    q = _uniform_q(16, 12, 10, 1.225, 0.0, 0.0, 0.0, 101325.0)
    kxyz, _ = _identity_metrics(16, 12, 10)
    rhs = ref.compute_viscous_rhs(A(ref, q), A(ref, kxyz), gas=_Gas(), ghost=2)
    np.testing.assert_allclose(N(rhs)[:, 4:-4, 4:-4, 4:-4], 0.0, atol=1e-10)


def test_rk3_linear_ode():
    """tests/time/test_rk.py:6-13"""
    q1 = NP.rk3_step(np.array([1.0]), lambda q: -q, 0.1)
    assert abs(q1[0] - math.exp(-0.1)) < 1e-5


def _two_block_halo(ref):
    g, ni_in = 2, 4
    ni = ni_in + 2 * g
    q0 = np.zeros((5, ni, 6, 4))
    q0[:, g:g + ni_in] = np.arange(1.0, ni_in + 1.0)[None, :, None, None]
    q1 = np.zeros((5, ni, 6, 4))
    q1[:, g:g + ni_in] = np.arange(10.0, 10.0 + ni_in)[None, :, None, None]
    t0 = _Topo(0, {**{f: None for f in range(6)}, IMAX: (1, IMIN, 0)}, {IMAX: CUT1TO1})
    t1 = _Topo(1, {**{f: None for f in range(6)}, IMIN: (0, IMAX, 0)}, {IMIN: CUT1TO1})
    return ref.halo_exchange([A(ref, q0), A(ref, q1)], (t0, t1), g)


@pytest.mark.parametrize("ref", BACKENDS)
def test_two_blocks_imax_to_imin(ref):
    """tests/mesh/test_halo.py:10-46"""
    new = _two_block_halo(ref)
    assert float(new[0][0, -2, 0, 0]) == 10.0
    assert float(new[0][0, -1, 0, 0]) == 11.0
    assert float(new[1][0, 0, 0, 0]) == 3.0
    assert float(new[1][0, 1, 0, 0]) == 4.0


def test_halo_orient_not_implemented():
    t0 = _Topo(0, {IMAX: (0, IMIN, 1)}, {IMAX: CUT1TO1})
    with pytest.raises(NotImplementedError):
        NP.halo_exchange([np.zeros((5, 6, 6, 6))], (t0,), 2)


def _cube_xyz(ni, nj, nk):
    X, Y, Z = np.meshgrid(np.linspace(0, 1, ni), np.linspace(0, 2, nj), np.linspace(0, 3, nk), indexing="ij")
    return np.stack([X, Y, Z], axis=0)


@pytest.mark.parametrize("ref", BACKENDS)
def test_uniform_cube_metrics(ref):
    """tests/mesh/test_metric.py:15-30"""
    jac, kxyz, vol = ref.compute_metrics(A(ref, _cube_xyz(20, 20, 20)), ghost=2)
    np.testing.assert_allclose(N(jac)[4:-4, 4:-4, 4:-4], (1 / 19) * (2 / 19) * (3 / 19), rtol=1e-10)
    np.testing.assert_allclose(N(kxyz)[0, 0, 4:-4, 4:-4, 4:-4], 19.0, rtol=1e-9)
    np.testing.assert_allclose(N(kxyz)[1, 0, 4:-4, 4:-4, 4:-4], 0.0, atol=1e-9)


def _farfield_cfg(q_inf):
    topo = _Topo(0, {f: None for f in range(6)}, {f: FARFIELD for f in range(6)})
    return _Cfg((topo,), {f: {"q_inf": q_inf} for f in range(6)})


@pytest.mark.parametrize("ref", BACKENDS)
def test_uniform_flow_stays_uniform(ref):
    """tests/solver/test_step.py:7-42"""
    g = 1.4
    rho, u, v, w, p = 1.225, 50.0, 0.0, 0.0, 101325.0
    q = _uniform_q(16, 12, 10, rho, u, v, w, p)
    kxyz, vol = _identity_metrics(16, 12, 10)
    cfg = _farfield_cfg(list(q[:, 0, 0, 0]))
    qs = [A(ref, q)]
    for _ in range(3):
        qs = ref.step(qs, [(A(ref, kxyz), A(ref, vol))], cfg, 1e-6)
    np.testing.assert_allclose(N(qs[0])[:, 4:-4, 4:-4, 4:-4], q[:, 4:-4, 4:-4, 4:-4], rtol=1e-5, atol=1e-5)


def test_grad_wrt_q_nonzero_finite():
    """tests/solver/test_grad.py:10-38 (autograd of the torch twin in place of jax.grad)"""
    import torch
    q = _uniform_q(12, 10, 8, 1.225, 50.0, 0.0, 0.0, 101325.0)
    kxyz, vol = _identity_metrics(12, 10, 8)
    cfg = _farfield_cfg(list(q[:, 0, 0, 0]))
    q0 = torch.tensor(q, requires_grad=True)
    out = TORCH.step([q0], [(torch.tensor(kxyz), torch.tensor(vol))], cfg, 1e-6)
    out[0].sum().backward()
    gq = q0.grad
    assert torch.all(torch.isfinite(gq))
    assert torch.any(gq != 0.0)


@pytest.mark.parametrize("ref", BACKENDS)
def test_farfield_sets_ghost(ref):
    """tests/physics/test_bc_farfield.py:6-36"""
    q = A(ref, np.ones((5, 8, 4, 4)) * 99.0)
    qb = N(ref.apply_farfield(q, IMAX, 2, [1.0, 0.5, 0.0, 0.0, 2.5]))
    for gg in range(2):
        assert qb[0, 7 - gg, 0, 0] == 1.0 and qb[1, 7 - gg, 0, 0] == 0.5
    qb = N(ref.apply_farfield(q, IMIN, 2, [1.2, 0.3, 0.1, 0.0, 3.0]))
    assert qb[0, 0, 0, 0] == 1.2 and qb[1, 1, 0, 0] == 0.3 and qb[0, 2, 0, 0] == 99.0
    q5 = A(ref, np.ones((5, 8, 4, 4)) * 5.0)
    qb = N(ref.apply_farfield(q5, JMIN, 2, [1.0, 0.0, 0.0, 0.0, 2.5]))
    for j in range(2, 4):
        assert qb[0, 0, j, 0] == 5.0


def _bc_block():
    return _uniform_q(8, 4, 4, 1.0, 2.0, 3.0, 4.0, 1.0)


def test_dispatch_wall_symmetry_farfield_cut():
    """tests/physics/test_bc_dispatch.py:30-75"""
    q = _bc_block()
    out = NP.apply_bc(q, _Topo(0, {}, {IMIN: WALL}), _Cfg((), {}))
    for gg in range(2):
        assert out[1, gg, 0, 0] == -2.0 and out[0, gg, 0, 0] == 1.0
    out = NP.apply_bc(q, _Topo(0, {}, {JMIN: SYMMETRY}), _Cfg((), {}))
    assert out[2, 0, 0, 0] == -3.0 and out[1, 0, 0, 0] == 2.0
    qi = [1.2, 0.5, 0.1, 0.0, 3.0]
    out = NP.apply_bc(q, _Topo(0, {}, {IMAX: FARFIELD}), _Cfg((), {IMAX: {"q_inf": qi}}))
    for gg in range(2):
        assert out[0, 7 - gg, 0, 0] == qi[0] and out[1, 7 - gg, 0, 0] == qi[1]
    out = NP.apply_bc(q, _Topo(0, {}, {IMIN: CUT1TO1}), _Cfg((), {}))
    np.testing.assert_array_equal(out, q)


def test_numpy_and_torch_twins_agree():
    """The two backends of the restatement agree on a random non-uniform state."""
    import torch
    rng = np.random.default_rng(3)
    ni, nj, nk = 9, 8, 7
    q = _uniform_q(ni, nj, nk, 1.0, 0.3, -0.2, 0.1, 0.7)
    q = q * (1 + 0.02 * rng.standard_normal(q.shape))
    kxyz = np.eye(3)[:, :, None, None, None] * 3.0 + 0.1 * rng.standard_normal((3, 3, ni, nj, nk))
    vol = 0.04 + 0.001 * rng.random((ni, nj, nk))
    cfg = _Cfg((), {})
    a = NP.rhs_block(q, kxyz, vol, cfg)
    b = TORCH.rhs_block(torch.tensor(q), torch.tensor(kxyz), torch.tensor(vol), cfg).numpy()
    assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(a)

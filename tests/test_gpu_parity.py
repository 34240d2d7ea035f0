"""Parity of the CUDA path (through libfamrdp_cuda.so's C ABI, via the
Python shim that mirrors famrdp_jax's API) with the CPU oracle.

Tolerances
  * pointwise kernels (EOS, MUSCL, Roe, limiters, halo, BCs): rtol 1e-13 or
    exact -- the same expressions, at most one rounding difference where
    nvcc contracts a*b+c into an FMA;
  * RHS fields: relative L2 <= 1e-11 -- the face-flux difference F[c-1]-F[c-2]
    cancels most of |F|, so a one-ulp difference in F becomes ~|F|/|dF| ulp in
    the RHS;
  * FP64 step: relative L2 of q <= 1e-12 after every step (the drop-in bar);
  * FP32-flux step: relative L2 of q <= 1e-5 after the steps run, with the
    per-step error reported.
"""
import numpy as np
import pytest
import torch

from famrdp_jax_b200 import cases
from famrdp_jax_b200.core.constants import BCType, Face
from famrdp_jax_b200.core.types import Block, BlockTopology, Config, GasModel, Metrics, SchemeChoice, State
from famrdp_jax_b200.flux.roe import roe_flux
from famrdp_jax_b200.mesh.halo import halo_exchange
from famrdp_jax_b200.mesh.metric import compute_metrics
from famrdp_jax_b200.physics.bc.dispatch import apply_bc
from famrdp_jax_b200.physics.eos import cons_to_prim, prim_to_cons
from famrdp_jax_b200.physics.reconstruct.muscl2 import minmod, muscl2_reconstruct, vanleer
from famrdp_jax_b200.rhs.invscd import compute_invscd_rhs
from famrdp_jax_b200.rhs.viscous import compute_viscous_rhs
from famrdp_jax_b200.solver import diagnostics
from famrdp_jax_b200.solver.step import _rhs_block, step
from famrdp_jax_b200.time.rk import rk3_step
from oracle.ref import NP
from parity_util import dev, host, random_block, rel_l2, state_from_case

pytestmark = pytest.mark.gpu

GAS = GasModel(gamma=1.4, R=1.0, mu0=2e-3, T0=1 / 1.4, Ts=0.27, Pr_lam=0.72)


@pytest.fixture(params=["split", "fused", "staged"])
def pipeline(request, cuda_device):
    """Runs a test on each RHS/stage pipeline (split is the default)."""
    from famrdp_jax_b200 import _capi
    _capi.set_pipeline(request.param)
    yield request.param
    _capi.set_pipeline()


def _cfg(topology=(), bc_params=None, limiter="minmod", gas=GAS, precision="f64"):
    return Config(gas=gas, scheme=SchemeChoice("muscl2", "roe", 3, limiter), bc_params=bc_params or {},
                  topology=topology, ghost=2, nan_check=False, precision=precision)


# ---------------------------------------------------------------- pointwise
def test_roe_known_answers(cuda_device):
    """tests/flux/test_roe.py:5-26 through the CUDA kernel."""
    g = 1.4
    for (rho, u, v, w, p), n in [((1.0, 50.0, 0.0, 0.0, 101325.0), (1.0, 0.0, 0.0)),
                                 ((1.0, 30.0, 20.0, 10.0, 50000.0), (0.6, 0.8, 0.0))]:
        rhoE = p / (g - 1.0) + 0.5 * rho * (u ** 2 + v ** 2 + w ** 2)
        U = dev([rho, rho * u, rho * v, rho * w, rhoE])
        F = host(roe_flux(U, U, dev(n), gamma=g))
        un = u * n[0] + v * n[1] + w * n[2]
        H = (rhoE + p) / rho
        exp = [rho * un, rho * u * un + p * n[0], rho * v * un + p * n[1], rho * w * un + p * n[2], rho * H * un]
        np.testing.assert_allclose(F, exp, rtol=1e-12)


def test_roe_random_faces(cuda_device):
    rng = np.random.default_rng(0)
    nf = 4096
    q, _, _ = random_block((nf, 1, 1), 1, noise=0.2)
    qr, _, _ = random_block((nf, 1, 1), 2, noise=0.2)
    UL, UR = q[:, :, 0, 0], qr[:, :, 0, 0]
    nv = rng.standard_normal((3, nf))
    nv /= np.linalg.norm(nv, axis=0)
    ref = NP.roe_flux(UL, UR, nv, gamma=1.4)
    got = host(roe_flux(dev(UL), dev(UR), dev(nv), gamma=1.4))
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14)


def test_eos_roundtrip_and_parity(cuda_device):
    prim = np.array([1.225, 50.0, 10.0, -5.0, 101325.0])[:, None, None, None]
    back = host(cons_to_prim(prim_to_cons(dev(prim), 1.4), 1.4))
    np.testing.assert_allclose(back, prim, rtol=1e-14)
    q, _, _ = random_block((7, 6, 5), 3)
    np.testing.assert_allclose(host(cons_to_prim(dev(q), 1.4)), NP.cons_to_prim(q, 1.4), rtol=1e-14)


def test_limiters_and_muscl(cuda_device):
    np.testing.assert_allclose(host(minmod(dev([1.0, -1.0]), dev([-1.0, 1.0]))), 0.0, atol=1e-15)
    assert host(minmod(dev(2.0), dev(5.0))).item() == 2.0
    assert host(minmod(dev(-3.0), dev(-7.0))).item() == -3.0
    rng = np.random.default_rng(5)
    a, b = rng.standard_normal(1000), rng.standard_normal(1000)
    np.testing.assert_allclose(host(vanleer(dev(a), dev(b))), NP.vanleer(a, b), rtol=1e-14)
    pv = np.stack([np.linspace(1.0, 10.0, 10)] * 5, axis=0)[:, :, None, None]
    L, R = muscl2_reconstruct(dev(pv), axis=1, limiter="minmod")
    np.testing.assert_allclose(host(L)[0, :, 0, 0], host(R)[0, :, 0, 0], rtol=1e-12)
    pv = rng.standard_normal((5, 9, 8, 7))
    for axis in (1, 2, 3):
        for lim in ("minmod", "vanleer"):
            L, R = muscl2_reconstruct(dev(pv), axis=axis, limiter=lim)
            rL, rR = NP.muscl2_reconstruct(pv, axis=axis, limiter=lim)
            np.testing.assert_allclose(host(L), rL, rtol=1e-14, atol=1e-15)
            np.testing.assert_allclose(host(R), rR, rtol=1e-14, atol=1e-15)
    with pytest.raises(KeyError):
        muscl2_reconstruct(dev(pv), axis=1, limiter="superbee")


# ---------------------------------------------------------------- RHS
@pytest.mark.parametrize("shape,seed", [((12, 10, 9), 0), ((7, 16, 6), 1), ((9, 5, 21), 2)])
@pytest.mark.parametrize("limiter", ["minmod", "vanleer"])
def test_invscd_rhs_parity(cuda_device, pipeline, shape, seed, limiter):
    q, kxyz, vol = random_block(shape, seed)
    m = Metrics(jac=dev(vol), kxyz=dev(kxyz), vol=dev(vol))
    got = host(compute_invscd_rhs(dev(q), m, ghost=2, gamma=1.4, reconstruct="muscl2", flux="roe",
                                  limiter=limiter))
    ref = NP.compute_invscd_rhs(q, kxyz, vol, ghost=2, gamma=1.4, limiter=limiter)
    assert rel_l2(got, ref) <= 1e-11


@pytest.mark.parametrize("visc_law", ["sutherland", "constant"])
@pytest.mark.parametrize("shape,seed", [((12, 10, 9), 0), ((5, 7, 6), 4)])
def test_viscous_rhs_parity(cuda_device, pipeline, shape, seed, visc_law):
    q, kxyz, vol = random_block(shape, seed)
    gas = GasModel(gamma=1.4, R=1.0, mu0=2e-3, T0=1 / 1.4, Ts=0.27, Pr_lam=0.72, visc_law=visc_law)
    m = Metrics(jac=dev(vol), kxyz=dev(kxyz), vol=dev(vol))
    got = host(compute_viscous_rhs(dev(q), m, gas=gas, ghost=2))
    ref = NP.compute_viscous_rhs(q, kxyz, gas=gas, ghost=2)
    assert np.all(got[0] == 0.0)
    assert rel_l2(got, ref) <= 1e-11


def test_rhs_block_parity_and_reference_invariants(cuda_device, pipeline):
    q, kxyz, vol = random_block((11, 9, 13), 7)
    m = Metrics(jac=dev(vol), kxyz=dev(kxyz), vol=dev(vol))
    cfg = _cfg()
    got = host(_rhs_block(dev(q), m, cfg))
    ref = NP.rhs_block(q, kxyz, vol, cfg)
    assert rel_l2(got, ref) <= 1e-11
    # tests/rhs/test_invscd.py:7-23 and tests/rhs/test_viscous.py:7-20
    ni, nj, nk = 16, 12, 10
    k_id = np.zeros((3, 3, ni, nj, nk))
    for d in range(3):
        k_id[d, d] = 1.0
    one = np.ones((ni, nj, nk))
    mi = Metrics(jac=dev(one), kxyz=dev(k_id), vol=dev(one))
    rho, u, p = 1.225, 50.0, 101325.0
    qu = np.zeros((5, ni, nj, nk))
    qu[0], qu[1], qu[4] = rho, rho * u, p / 0.4 + 0.5 * rho * u * u
    r = host(compute_invscd_rhs(dev(qu), mi, ghost=2, gamma=1.4, reconstruct="muscl2", flux="roe",
                                limiter="minmod"))
    np.testing.assert_allclose(r[:, 4:-4, 4:-4, 4:-4], 0.0, atol=1e-8)
    qs = np.zeros((5, ni, nj, nk))
    qs[0], qs[4] = rho, p / 0.4
    r = host(compute_viscous_rhs(dev(qs), mi, gas=GasModel(), ghost=2))
    np.testing.assert_allclose(r[:, 4:-4, 4:-4, 4:-4], 0.0, atol=1e-10)


@pytest.mark.parametrize("seg", [1, 2, 5, 0])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_fused_segments_and_ragged_tiles(cuda_device, seg, precision):
    """Segment lengths along i and tiles that overhang the block in j and k."""
    from famrdp_jax_b200 import _capi
    q, kxyz, vol = random_block((13, 19, 41), 9)
    m = Metrics(jac=dev(vol), kxyz=dev(kxyz), vol=dev(vol))
    cfg = _cfg(precision=precision)
    _capi.set_pipeline("staged")
    ref = host(_rhs_block(dev(q), m, cfg))
    _capi.set_pipeline("fused", seg=seg)
    try:
        got = host(_rhs_block(dev(q), m, cfg))
    finally:
        _capi.set_pipeline()
    assert rel_l2(got, ref) <= (1e-12 if precision == "f64" else 1e-5)
    if precision == "f64":
        assert rel_l2(got, NP.rhs_block(q, kxyz, vol, cfg)) <= 1e-11


# ---------------------------------------------------------------- halo + BC
def test_two_block_halo_known_answer(cuda_device):
    """tests/mesh/test_halo.py:10-46"""
    g, ni_in = 2, 4
    shape = (5, ni_in + 2 * g, 6, 5)
    q0 = np.zeros(shape)
    q0[:, g:g + ni_in] = np.arange(1.0, ni_in + 1.0)[None, :, None, None]
    q1 = np.zeros(shape)
    q1[:, g:g + ni_in] = np.arange(10.0, 10.0 + ni_in)[None, :, None, None]
    xyz = dev(np.zeros((3,) + shape[1:]))
    t0 = BlockTopology(0, {**{f: None for f in Face}, Face.IMAX: (1, Face.IMIN, 0)}, {Face.IMAX: BCType.CUT1TO1})
    t1 = BlockTopology(1, {**{f: None for f in Face}, Face.IMIN: (0, Face.IMAX, 0)}, {Face.IMIN: BCType.CUT1TO1})
    new = halo_exchange((Block(dev(q0), xyz), Block(dev(q1), xyz)), (t0, t1), ghost=g)
    a, b = host(new[0].q), host(new[1].q)
    assert a[0, -2, 0, 0] == 10.0 and a[0, -1, 0, 0] == 11.0
    assert b[0, 0, 0, 0] == 3.0 and b[0, 1, 0, 0] == 4.0


def _rand_qs(shapes, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((5,) + tuple(s)) for s in shapes]


@pytest.mark.parametrize("name", ["wavy4", "tree", "self"])
def test_halo_exchange_matches_oracle_exactly(cuda_device, name):
    if name == "wavy4":
        c = cases.wavy4(n=6, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2))
        topos, shapes = c.cfg.topology, [q.shape[1:] for q in c.qs]
    elif name == "tree":
        c = cases.tree24(nblocks=9, lo=5, hi=11, seed=3)
        topos, shapes = c.cfg.topology, [q.shape[1:] for q in c.qs]
    else:
        c = cases.tgv(n=6)
        topos, shapes = c.cfg.topology, [q.shape[1:] for q in c.qs]
    qs = _rand_qs(shapes, 11)
    ref = NP.halo_exchange(qs, topos, 2)
    xyz = [dev(np.zeros((3,) + tuple(s))) for s in shapes]
    got = halo_exchange(tuple(Block(dev(q), x) for q, x in zip(qs, xyz)), topos, ghost=2)
    for g_, r in zip(got, ref):
        np.testing.assert_array_equal(host(g_.q), r)


@pytest.mark.parametrize("name", ["wavy4", "tree"])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_plan_step_ignores_stale_output_interior(cuda_device, name, precision):
    """A plan step uses its output array as the halo-filled start state: the
    result must not depend on what the output array held (NaN here), must
    equal the step that keeps its start state in a separate array
    (run_save), bit for bit, replayed from a graph too, and must leave the
    input unchanged."""
    import dataclasses
    from famrdp_jax_b200.solver.step import StepPlan
    if name == "wavy4":
        c = cases.wavy4(n=10, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2))
    else:
        c = cases.tree24(nblocks=6, lo=6, hi=12, seed=1)
    cfg = dataclasses.replace(c.cfg, precision=precision)
    st = state_from_case(c)
    plan = StepPlan(st, cfg)
    qin = [b.q.clone() for b in st.blocks]
    keep = [q.clone() for q in qin]
    dt = 0.5 * NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], cfg.gas.gamma, 0.5, 2)
    out = [torch.full_like(q, float("nan")) for q in qin]
    plan.run(qin, out, dt)
    ref = [torch.zeros_like(q) for q in qin]
    saved = [[torch.zeros_like(q) for q in qin] for _ in range(3)]
    plan.run_save(qin, ref, *saved, dt)
    for o, r, q, k in zip(out, ref, qin, keep):
        assert torch.equal(o, r)
        assert torch.equal(q, k)
    out2 = [torch.full_like(q, float("nan")) for q in qin]
    plan.run(qin, out2, dt, graph=True)
    for o, r in zip(out2, ref):
        assert torch.equal(o, r)


def test_halo_errors(cuda_device):
    xyz = dev(np.zeros((3, 8, 8, 8)))
    b0 = Block(dev(np.zeros((5, 8, 8, 8))), xyz)
    t = BlockTopology(0, {Face.IMAX: (0, Face.IMIN, 1)}, {Face.IMAX: BCType.CUT1TO1})
    with pytest.raises(NotImplementedError):
        halo_exchange((b0,), (t,), ghost=2)
    b1 = Block(dev(np.zeros((5, 8, 9, 8))), dev(np.zeros((3, 8, 9, 8))))
    t0 = BlockTopology(0, {Face.IMAX: (1, Face.IMIN, 0)}, {Face.IMAX: BCType.CUT1TO1})
    t1 = BlockTopology(1, {}, {})
    with pytest.raises(ValueError, match="shape"):
        halo_exchange((b0, b1), (t0, t1), ghost=2)


@pytest.mark.parametrize("bct,params", [
    (BCType.FARFIELD, {"q_inf": [1.2, 0.5, 0.1, 0.0, 3.0]}),
    (BCType.WALL, {}),
    (BCType.WALL, {"wall_type": "isothermal", "T_wall": 0.9}),
    (BCType.SYMMETRY, {}),
])
def test_bc_matches_oracle(cuda_device, bct, params):
    q, _, _ = random_block((8, 7, 9), 21)
    faces = list(Face)
    topo = BlockTopology(0, {}, {f: bct for f in faces})
    cfg = _cfg(topology=(topo,), bc_params={f: params for f in faces})
    got = host(apply_bc(Block(dev(q), dev(np.zeros((3, 8, 7, 9)))), topo, cfg).q)
    ref = NP.apply_bc(q, topo, cfg)
    np.testing.assert_allclose(got, ref, rtol=1e-15, atol=0)


# ---------------------------------------------------------------- metrics
def test_metrics_match_fortran_golden(cuda_device):
    from pathlib import Path
    data = np.load(Path(__file__).parent / "golden" / "test3_metric.npz")
    for b in (1, 2):
        m = compute_metrics(dev(data[f"xyz{b}"]), ghost=0)
        ref = data[f"jac{b}"]
        assert np.abs(host(m.jac) - ref).max() <= 1e-13
        _, kref, _ = NP.compute_metrics(data[f"xyz{b}"], ghost=0)
        assert rel_l2(host(m.kxyz), kref) <= 1e-13


def test_metrics_uniform_cube(cuda_device):
    """tests/mesh/test_metric.py:15-30"""
    X, Y, Z = np.meshgrid(np.linspace(0, 1, 20), np.linspace(0, 2, 20), np.linspace(0, 3, 20), indexing="ij")
    m = compute_metrics(dev(np.stack([X, Y, Z])), ghost=2)
    np.testing.assert_allclose(host(m.jac)[4:-4, 4:-4, 4:-4], (1 / 19) * (2 / 19) * (3 / 19), rtol=1e-10)
    np.testing.assert_allclose(host(m.kxyz)[0, 0, 4:-4, 4:-4, 4:-4], 19.0, rtol=1e-9)
    np.testing.assert_allclose(host(m.kxyz)[1, 0, 4:-4, 4:-4, 4:-4], 0.0, atol=1e-9)


# ---------------------------------------------------------------- step
def _rel_per_variable(got, ref, g=2):
    """Relative L2 per conserved variable over the full padded blocks and over
    the interiors (all blocks together)."""
    out = {}
    for part in ("full", "interior"):
        for v in range(5):
            num = den = 0.0
            for a, b in zip(got, ref):
                x, y = a[v], b[v]
                if part == "interior":
                    x, y = x[g:-g, g:-g, g:-g], y[g:-g, g:-g, g:-g]
                num += float(np.sum((x - y) ** 2))
                den += float(np.sum(y ** 2))
            out[(part, v)] = (num / den) ** 0.5 if den > 0 else num ** 0.5
    return out


def _run_steps(case, nsteps, dt, tol_fp64=1e-12):
    """nsteps GPU steps against the oracle's: returns the whole-state relative
    L2 after every step; for FP64 also checks every variable, full and interior,
    against tol_fp64 after every step."""
    st = state_from_case(case)
    qs = [q.copy() for q in case.qs]
    mets = [(m[1], m[2]) for m in case.metrics]
    errs = []
    for _ in range(nsteps):
        st = step(st, case.cfg, dt)
        qs = NP.step(qs, mets, case.cfg, dt)
        got = [host(b.q) for b in st.blocks]
        errs.append(max(rel_l2(a, r) for a, r in zip(got, qs)))
        if getattr(case.cfg, "precision", "f64") == "f64":
            per = _rel_per_variable(got, qs)
            worst = max(per.values())
            assert worst <= tol_fp64, {k: v for k, v in per.items() if v > tol_fp64}
    return errs, st


def test_step_tgv32_ten_steps_fp64(cuda_device, pipeline):
    """Config: 32^3 TGV, M0 = 0.1, Re = 1600, constant viscosity, CFL 0.5, 10 steps."""
    c = cases.tgv(n=32)
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], c.cfg.gas.gamma, c.cfl, 2)
    errs, st = _run_steps(c, 10, dt)
    assert max(errs) <= 1e-12, errs
    assert st.step == 10 and abs(st.t - 10 * dt) < 1e-15


def test_step_wavy4_fp64(cuda_device, pipeline):
    c = cases.wavy4(n=12, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2))
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], c.cfg.gas.gamma, c.cfl, 2)
    errs, _ = _run_steps(c, 3, dt)
    assert max(errs) <= 1e-12, errs


def test_step_tree_with_farfield_fp64(cuda_device, pipeline):
    c = cases.tree24(nblocks=6, lo=6, hi=12, seed=1)
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], c.cfg.gas.gamma, c.cfl, 2)
    errs, _ = _run_steps(c, 3, dt)
    assert max(errs) <= 1e-12, errs


def test_step_fp32_flux_tgv(cuda_device, pipeline):
    c = cases.tgv(n=32, precision="f32")
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], c.cfg.gas.gamma, c.cfl, 2)
    errs, _ = _run_steps(c, 10, dt)
    print("fp32-flux per-step rel L2:", ["%.2e" % e for e in errs])
    assert max(errs) <= 1e-5, errs


def test_step_input_state_unchanged(cuda_device):
    c = cases.tgv(n=8)
    st = state_from_case(c)
    before = host(st.blocks[0].q).copy()
    step(st, c.cfg, 1e-4)
    np.testing.assert_array_equal(host(st.blocks[0].q), before)


def test_rk3_linear_ode(cuda_device):
    """tests/time/test_rk.py:6-13"""
    q1 = rk3_step(dev([1.0]), lambda q: -q, 0.1)
    assert abs(float(host(q1)[0]) - np.exp(-0.1)) < 1e-5


# ---------------------------------------------------------------- reductions
def test_reductions_match_oracle(cuda_device):
    c = cases.wavy4(n=8, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2))
    st = state_from_case(c)
    mets = [(m[1], m[2]) for m in c.metrics]
    dt = diagnostics.cfl_dt(st, c.cfg, 0.5)
    assert abs(dt - NP.cfl_dt(c.qs, mets, 1.4, 0.5, 2)) <= 1e-14 * dt
    ke = diagnostics.kinetic_energy(st, 2)
    assert abs(ke - NP.kinetic_energy(c.qs, mets, 2)) <= 1e-13 * abs(ke)
    n, rmin, pmin = diagnostics.check_state(st, 1.4)
    assert n == 0 and rmin > 0 and pmin > 0


def test_check_state_reports_injected_nan(cuda_device):
    """Failure detection: a NaN and a negative density are planted on the host."""
    c = cases.tgv(n=8)
    q = c.qs[0].copy()
    q[2, 3, 4, 5] = np.nan
    q[0, 6, 6, 6] = -1.0
    c.qs[0] = q
    st = state_from_case(c)
    with pytest.raises(FloatingPointError):
        diagnostics.check_state(st, 1.4)
    n, rmin, _ = diagnostics.check_state(st, 1.4, raise_on_error=False)
    assert n == 1 and rmin == -1.0


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_graph_step_matches_plain_step(cuda_device, precision):
    """fj_plan_step_graph: ping-pong steps replayed from two captured graphs
    give bit-identical states to fj_plan_step, and each replay counts the
    graph's kernels."""
    import dataclasses
    from famrdp_jax_b200 import _capi
    from famrdp_jax_b200.solver.step import StepPlan
    c = cases.tree24(nblocks=5, lo=6, hi=12, seed=3)
    cfg = dataclasses.replace(c.cfg, precision=precision)
    st = state_from_case(c)
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], cfg.gas.gamma, c.cfl, 2)
    plan = StepPlan(st, cfg)
    a = [b.q.clone() for b in st.blocks]
    b_ = [torch.empty_like(q) for q in a]
    ga = [q.clone() for q in a]
    gb = [torch.empty_like(q) for q in a]
    for n in range(5):
        plan.run(a, b_, dt)
        a, b_ = b_, a
        before = _capi.launch_count()
        plan.run(ga, gb, dt, graph=True)
        per_step = _capi.launch_count() - before
        ga, gb = gb, ga
        for x, y in zip(a, ga):
            assert torch.equal(x, y), n
    assert per_step > 0
    # a later replay of an already captured pointer set reuses its graph
    before = _capi.launch_count()
    plan.run(ga, gb, dt, graph=True)
    assert _capi.launch_count() - before == per_step


def test_step_on_parsed_gridgen_topology(cuda_device, pipeline):
    """Two blocks joined through a parsed GridGen topology (a j-interface pair
    with orientation 0 plus wall, symmetry and farfield faces), sized as the
    file declares (5 x 5 x 3 nodes + 2 ghosts per side): FP64 steps against
    the oracle."""
    from pathlib import Path
    from famrdp_jax_b200.mesh.io_top import parse_topology
    tops = tuple(parse_topology(Path(__file__).parent / "golden" / "mini.inp"))
    blocks = [random_block((9, 9, 7), 20 + b, noise=0.02) for b in range(2)]
    qs = [b[0] for b in blocks]
    mets = [(b[1], b[2]) for b in blocks]
    q_inf = list(qs[0][:, 4, 4, 3])
    cfg = _cfg(topology=tops, bc_params={f: {"q_inf": q_inf} for f in Face})
    case = cases.Case(name="gridgen2", qs=qs, metrics=[(b[2], b[1], b[2]) for b in blocks], cfg=cfg, cfl=0.5,
                      steps=3)
    dt = 0.5 * NP.cfl_dt(qs, mets, cfg.gas.gamma, 0.5, 2)
    errs, _ = _run_steps(case, 3, dt)
    assert max(errs) <= 1e-12, errs


def test_residual_and_monitored_run(cuda_device, tmp_path):
    """fj_residual_f64 against the NumPy residual of the oracle's step, and the
    monitored loop: same states as plain steps, one log row per step, and a
    planted NaN stops it with FloatingPointError and dumps both states."""
    from famrdp_jax_b200.solver.run import run, write_residual_log
    c = cases.tgv(n=12, M0=0.3, Re=400.0, noise=0.01, seed=1)
    st = state_from_case(c)
    mets = [(m[1], m[2]) for m in c.metrics]
    dt = NP.cfl_dt(c.qs, mets, c.cfg.gas.gamma, c.cfl, 2)
    q1 = NP.step(c.qs, mets, c.cfg, dt)
    g = 2
    inner = (slice(None),) + (slice(g, -g),) * 3
    ref = np.sqrt(np.mean(((q1[0] - c.qs[0]) / dt)[inner] ** 2, axis=(1, 2, 3)))
    st1 = step(st, c.cfg, dt)
    got = diagnostics.residual(st1, [b.q for b in st.blocks], dt, g)
    np.testing.assert_allclose(got, ref, rtol=1e-9)
    final, log = run(st, c.cfg, dt, 4)
    ref_st = st
    for _ in range(4):
        ref_st = step(ref_st, c.cfg, dt)
    assert torch.equal(final.blocks[0].q, ref_st.blocks[0].q) and final.step == 4
    assert [r[0] for r in log.rows] == [1, 2, 3, 4]
    np.testing.assert_allclose(log.rows[0][2], got, rtol=1e-14)
    write_residual_log(tmp_path / "res.txt", log)
    assert len((tmp_path / "res.txt").read_text().splitlines()) == 5
    bad = st.blocks[0].q.clone()
    bad[0, 5, 5, 5] = float("nan")
    import dataclasses
    st_bad = dataclasses.replace(st, blocks=(dataclasses.replace(st.blocks[0], q=bad),))
    cfg = dataclasses.replace(c.cfg, nan_check=True)
    with pytest.raises(FloatingPointError, match="step 1"):
        run(st_bad, cfg, dt, 3, dump_dir=tmp_path / "dumps")
    assert sorted(p.name for p in (tmp_path / "dumps").iterdir()) == ["step0000000_good.pt", "step0000001_bad.pt"]


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_autotune_launch_shapes_agree(cuda_device, precision):
    """Every launch shape of the split kernels and both stream counts (block
    groups on two streams, also captured as a graph) give the same step bit for
    bit, in both precisions, and so does (FP32-flux) the persistent step in
    every launch shape; the autotuner keeps one of them (or, FP32-flux, the
    tile kernel or the persistent step)."""
    import dataclasses
    from famrdp_jax_b200 import _capi
    from famrdp_jax_b200.solver.step import StepPlan
    c = cases.tree24(nblocks=4, lo=6, hi=12, seed=2)
    cfg = dataclasses.replace(c.cfg, precision=precision)
    st = state_from_case(c)
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], cfg.gas.gamma, c.cfl, 2)
    plan = StepPlan(st, cfg)
    qs = [b.q for b in st.blocks]
    outs = []
    for streams in (1, 2):
        plan.set_streams(streams)
        for v in range(_capi.NUM_SPLIT_VARIANTS):
            plan.set_variant(v)
            for graph in (False, True):
                o = [torch.empty_like(q) for q in qs]
                plan.run(qs, o, dt, graph=graph)
                outs.append(o)
    if precision == "f32":
        # the persistent step in every launch shape, plain and as a graph
        plan.set_streams(1)
        plan.set_kernel("persistent")
        for shape in range(_capi.NUM_PERSIST_SHAPES):
            plan.set_persist_shape(shape)
            for graph in (False, True):
                o = [torch.empty_like(q) for q in qs]
                plan.run(qs, o, dt, graph=graph)
                outs.append(o)
        # the split kernels behind the fused ghost fill, every shape and stream count
        plan.set_kernel("split_fill")
        for streams in (1, 2):
            plan.set_streams(streams)
            for v in range(_capi.NUM_SPLIT_VARIANTS):
                plan.set_variant(v)
                o = [torch.empty_like(q) for q in qs]
                plan.run(qs, o, dt, graph=v % 2 == 1)
                outs.append(o)
        assert plan.check() == 0
        plan.set_kernel("split")
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert torch.equal(a, b)
    chosen, ms = plan.autotune(qs, [torch.empty_like(q) for q in qs], dt, reps=2)
    n = _capi.NUM_SPLIT_VARIANTS
    # candidates: every split shape at one and two streams, then (FP32-flux) the
    # tile kernel and the persistent step's shapes
    timed = ms if precision == "f32" else ms[:2 * n]
    assert 0 <= chosen < _capi.AUTOTUNE_CANDIDATES and len(ms) == _capi.AUTOTUNE_CANDIDATES and min(timed) > 0
    if precision == "f64":
        assert chosen < 2 * n and not any(ms[2 * n:])
    fill = 2 * n + 1 + _capi.NUM_PERSIST_SHAPES
    assert plan.kernel == ("tile" if chosen == 2 * n else "split_fill" if chosen == fill
                           else "persistent" if chosen > 2 * n else "split")


def test_plan_argument_errors(cuda_device):
    """The plan entry points reject bad arguments with the mapped exceptions
    and leave the plan usable."""
    import ctypes
    import dataclasses
    from famrdp_jax_b200 import _capi
    from famrdp_jax_b200.solver import adjoint
    from famrdp_jax_b200.solver.step import StepPlan
    c = cases.tree24(nblocks=2, lo=6, hi=9, seed=4)
    cfg = dataclasses.replace(c.cfg, precision="f32")
    st = state_from_case(c)
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], cfg.gas.gamma, c.cfl, 2)
    plan = StepPlan(st, cfg)
    qs = [b.q for b in st.blocks]
    with pytest.raises(ValueError):
        plan.set_variant(_capi.NUM_SPLIT_VARIANTS)
    with pytest.raises(ValueError):
        plan.set_variant(-1)
    with pytest.raises(ValueError):
        plan.set_streams(3)
    with pytest.raises(ValueError):
        plan.set_ensemble([1e-3])  # one value for two blocks
    with pytest.raises(ValueError):
        plan.set_ensemble(None, [1e-3, -1.0])
    with pytest.raises(ValueError):
        plan.run(qs, [torch.empty((5, 3, 3, 3), dtype=torch.float64, device="cuda")] * 2, dt)
    lib = _capi.lib()
    ch = ctypes.c_int()
    assert lib.fj_plan_autotune(plan._handle, _topology_ptrs(qs), _topology_ptrs(qs), dt, 0, ctypes.byref(ch),
                                None, None) == _capi.FJ_ERR_INVALID_ARGUMENT
    # still usable
    out = [torch.empty_like(q) for q in qs]
    plan.run(qs, out, dt)
    assert all(torch.isfinite(o).all() for o in out)
    # the ensemble adjoint wants one dJ/dmu0 slot per block
    saved = tuple([torch.empty_like(q) for q in qs] for _ in range(3))
    plan.run_save(qs, out, *saved, dt)
    with pytest.raises(ValueError):
        adjoint.step_vjp_saved(saved, st.metrics, cfg, dt, [torch.ones_like(q) for q in qs],
                               dmu=torch.zeros(1, dtype=torch.float64, device="cuda"), mu0s=[1e-3, 1e-3])


def _topology_ptrs(qs):
    from famrdp_jax_b200 import _topology
    return _topology.ptr_array(qs)


def test_host_stepper_matches_step(cuda_device):
    """HostStepper (pipelined host->device copy, step, device->host copy over
    three streams and two buffer sets) gives every step's result exactly as
    step() does, for different inputs per step."""
    from famrdp_jax_b200.solver.step import StepPlan
    from famrdp_jax_b200.solver.stream import HostStepper
    c = cases.tree24(nblocks=3, lo=6, hi=10, seed=6)
    st = state_from_case(c)
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], c.cfg.gas.gamma, c.cfl, 2)
    plan = StepPlan(st, c.cfg)
    n = 5
    ins = [[(b.q * (1.0 + 1e-3 * i)).cpu().pin_memory() for b in st.blocks] for i in range(n)]
    outs = [[torch.empty_like(h).pin_memory() for h in row] for row in ins]
    HostStepper(plan).run(ins, outs, dt)
    torch.cuda.current_stream().synchronize()
    for i in range(n):
        s_i = State(blocks=tuple(Block(q=h.cuda(), xyz=b.xyz) for h, b in zip(ins[i], st.blocks)), metrics=st.metrics)
        ref = step(s_i, c.cfg, dt, plan=plan)
        for h, b in zip(outs[i], ref.blocks):
            assert torch.equal(h, b.q.cpu()), i


def test_plans_are_reproducible(cuda_device):
    """Two plans made from the same state give bit-identical FP32-flux steps
    (the plan's pressure offset comes from a fixed-order reduction)."""
    import dataclasses
    from famrdp_jax_b200.solver.step import StepPlan
    c = cases.tree24(nblocks=5, lo=8, hi=14, seed=7)
    cfg = dataclasses.replace(c.cfg, precision="f32")
    st = state_from_case(c)
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], cfg.gas.gamma, c.cfl, 2)
    outs = []
    for _ in range(2):
        plan = StepPlan(st, cfg)
        o = [torch.empty_like(b.q) for b in st.blocks]
        plan.run([b.q for b in st.blocks], o, dt)
        outs.append(o)
    for a, b in zip(*outs):
        assert torch.equal(a, b)

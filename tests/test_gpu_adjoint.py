"""The hand-written adjoint (fj_rhs_vjp_f64, fj_step_vjp_f64 and the
checkpointed trajectory) against (a) torch.autograd of the CPU oracle's
PyTorch twin -- standing in for jax.grad of the reference, which is not
installable here -- and (b) central finite differences of the GPU forward.

Tolerances: VJPs relative L2 <= 1e-10 against autograd (FP64; the two sides
evaluate algebraically equal expressions in different orders); directional
derivatives against central differences (eps = 1e-6) to <= 1e-6 relative.
"""
import numpy as np
import pytest
import torch

from famrdp_jax_b200 import cases
from famrdp_jax_b200.core.constants import BCType, Face
from famrdp_jax_b200.core.types import Block, BlockTopology, Config, GasModel, Metrics, SchemeChoice, State
from famrdp_jax_b200.solver import adjoint, diagnostics
from famrdp_jax_b200.solver.step import StepPlan, step
from oracle.ref import NP, TORCH
from parity_util import dev, host, random_block, rel_l2

pytestmark = pytest.mark.gpu


def _cfg(topology=(), bc_params=None, limiter="minmod", visc_law="sutherland", precision="f64"):
    gas = GasModel(gamma=1.4, R=1.0, mu0=2e-3, T0=1 / 1.4, Ts=0.27, Pr_lam=0.72, visc_law=visc_law)
    return Config(gas=gas, scheme=SchemeChoice("muscl2", "roe", 3, limiter), bc_params=bc_params or {},
                  topology=topology, ghost=2, nan_check=False, precision=precision)


@pytest.mark.parametrize("limiter", ["minmod", "vanleer"])
@pytest.mark.parametrize("visc_law", ["sutherland", "constant"])
def test_rhs_vjp_matches_autograd(cuda_device, limiter, visc_law):
    q, kxyz, vol = random_block((9, 8, 10), 5)
    cfg = _cfg(limiter=limiter, visc_law=visc_law)
    lam = np.random.default_rng(6).standard_normal(q.shape)
    qt = torch.tensor(q, requires_grad=True)
    L = TORCH.rhs_block(qt, torch.tensor(kxyz), torch.tensor(vol), cfg)
    (ref,) = torch.autograd.grad(L, qt, grad_outputs=torch.tensor(lam))
    m = Metrics(jac=dev(vol), kxyz=dev(kxyz), vol=dev(vol))
    got = host(adjoint.rhs_vjp(dev(q), m, cfg, dev(lam)))
    assert rel_l2(got, ref.numpy()) <= 1e-10


@pytest.mark.parametrize("limiter", ["minmod", "vanleer"])
@pytest.mark.parametrize("visc_law", ["sutherland", "constant"])
@pytest.mark.parametrize("shape", [(9, 8, 10), (13, 19, 41)])
def test_f32_rhs_vjp_close_to_autograd(cuda_device, limiter, visc_law, shape):
    """The FP32-flux RHS VJP (face and viscous VJPs in one launch of
    interleaved CTAs, FP32 face arithmetic, FP64 lam/vol and final
    accumulation) against torch.autograd of the FP64 twin, on a block whose k
    rows do not align with warps.  Bound: relative L2 <= 2e-6 (measured
    1.4e-7 with minmod, 5.7e-7 with van Leer)."""
    q, kxyz, vol = random_block(shape, 5)
    cfg = _cfg(limiter=limiter, visc_law=visc_law, precision="f32")
    lam = np.random.default_rng(6).standard_normal(q.shape)
    qt = torch.tensor(q, requires_grad=True)
    L = TORCH.rhs_block(qt, torch.tensor(kxyz), torch.tensor(vol), cfg)
    (ref,) = torch.autograd.grad(L, qt, grad_outputs=torch.tensor(lam))
    m = Metrics(jac=dev(vol), kxyz=dev(kxyz), vol=dev(vol))
    got = host(adjoint.rhs_vjp(dev(q), m, cfg, dev(lam)))
    err = rel_l2(got, ref.numpy())
    assert err <= 2e-6


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_rhs_vjp_every_launch_variant(cuda_device, variant, precision):
    """Every launch shape of the face and viscous VJPs (fj_ctx_set_adjoint_variant;
    variant 0 runs FP32 as one combined launch, the others as two) against
    torch.autograd of the FP64 twin: FP64 <= 1e-10, FP32 <= 2e-6 relative L2."""
    from famrdp_jax_b200 import _capi
    q, kxyz, vol = random_block((13, 19, 41), 7)
    cfg = _cfg(limiter="vanleer", precision=precision)
    lam = np.random.default_rng(8).standard_normal(q.shape)
    qt = torch.tensor(q, requires_grad=True)
    L = TORCH.rhs_block(qt, torch.tensor(kxyz), torch.tensor(vol), cfg)
    (ref,) = torch.autograd.grad(L, qt, grad_outputs=torch.tensor(lam))
    m = Metrics(jac=dev(vol), kxyz=dev(kxyz), vol=dev(vol))
    qd = dev(q)
    _capi.set_adjoint_variant(variant, qd.device)
    try:
        got = host(adjoint.rhs_vjp(qd, m, cfg, dev(lam)))
    finally:
        _capi.set_adjoint_variant(0, qd.device)
    assert rel_l2(got, ref.numpy()) <= (1e-10 if precision == "f64" else 2e-6)


def _mirror_case():
    """One block with farfield, symmetry and adiabatic-wall faces and one
    self-periodic pair."""
    q, kxyz, vol = random_block((10, 9, 11), 8, noise=0.03)
    faces = {Face.IMIN: BCType.FARFIELD, Face.IMAX: BCType.SYMMETRY, Face.JMIN: BCType.WALL,
             Face.JMAX: BCType.FARFIELD, Face.KMIN: BCType.CUT1TO1, Face.KMAX: BCType.CUT1TO1}
    nb = {f: None for f in Face}
    nb[Face.KMIN] = (0, Face.KMAX, 0)
    nb[Face.KMAX] = (0, Face.KMIN, 0)
    topo = BlockTopology(0, nb, faces)
    q_inf = list(q[:, 4, 4, 4])
    cfg = _cfg(topology=(topo,), bc_params={f: {"q_inf": q_inf} for f in Face})
    return [q], [(kxyz, vol)], cfg


def _periodic_case():
    c = cases.tgv(n=8, M0=0.3, Re=100.0, noise=0.02, seed=4)
    return c.qs, [(m[1], m[2]) for m in c.metrics], c.cfg


@pytest.mark.parametrize("which", ["periodic", "mirror"])
def test_step_vjp_matches_autograd(cuda_device, which):
    qs, mets, cfg = _periodic_case() if which == "periodic" else _mirror_case()
    dt = 0.5 * NP.cfl_dt(qs, mets, cfg.gas.gamma, 0.5, 2)
    lam = [np.random.default_rng(9).standard_normal(q.shape) for q in qs]
    qt = [torch.tensor(q, requires_grad=True) for q in qs]
    out = TORCH.step(qt, [(torch.tensor(k), torch.tensor(v)) for k, v in mets], cfg, dt)
    ref = torch.autograd.grad(out, qt, grad_outputs=[torch.tensor(l) for l in lam])
    metrics = tuple(Metrics(jac=dev(v), kxyz=dev(k), vol=dev(v)) for k, v in mets)
    got = adjoint.step_vjp([dev(q) for q in qs], metrics, cfg, dt, [dev(l) for l in lam])
    for g, r in zip(got, ref):
        assert rel_l2(host(g), r.numpy()) <= 1e-10


def _tgv_state(n=12, M0=0.3, Re=800.0):
    c = cases.tgv(n=n, M0=M0, Re=Re, noise=0.01, seed=2)
    return c, cases.to_state(c, "cuda:0")


def _J(c, q0, nsteps, dt, cfg=None):
    cfg = cfg or c.cfg
    st = cases.to_state(c, "cuda:0")
    st = State(blocks=(Block(q=q0.clone(), xyz=st.blocks[0].xyz),), metrics=st.metrics)
    plan = StepPlan(st, cfg)
    for _ in range(nsteps):
        st = step(st, cfg, dt, plan=plan)
    return diagnostics.kinetic_energy(st, 2)


def test_trajectory_gradient_matches_finite_differences(cuda_device):
    """Config-4-style objective (kinetic energy after N steps, checkpointed
    reverse sweep) on a small Taylor-Green block with 1 % noise.

    The noise matters: the exact Taylor-Green state (w = 0, mirror-symmetric
    slopes) sits on the limiters' non-differentiable points (zero and equal
    slopes), where central differences average the one-sided derivatives and
    agree with no gradient.  Directions are random with unit L2 norm over the
    whole state; eps = 1e-7: J is only piecewise smooth (minmod switches where
    two slopes have equal magnitude or a slope changes sign), and a +-eps
    perturbation that crosses one of the ~1e4 limiter switching points of a
    stage biases the central difference; at 1e-6 that happened for one of six
    directions on this state, at 1e-7 the crossing probability is ten times
    lower while FP64 rounding of J stays below 1e-7 |grad J|.  The error of each directional derivative is
    measured relative to |grad J| (its bound for a unit direction): a
    direction nearly orthogonal to the gradient has a tiny derivative that the
    central difference resolves only to FP64 rounding of J (~1e-15 J / eps)."""
    c, st = _tgv_state()
    mets = [(m[1], m[2]) for m in c.metrics]
    dt = NP.cfl_dt(c.qs, mets, 1.4, 0.5, 2)
    nsteps = 6
    J, grads, dmu = adjoint.adjoint_kinetic_energy(st, c.cfg, dt, nsteps, checkpoint_every=4)
    g = grads[0]
    q0 = st.blocks[0].q
    rng = np.random.default_rng(11)
    eps = 1e-7
    gnorm = float(torch.linalg.vector_norm(g))
    for _ in range(16):
        d = torch.tensor(rng.standard_normal(tuple(q0.shape)), dtype=torch.float64, device="cuda")
        d = d / torch.linalg.vector_norm(d)
        fd = (_J(c, q0 + eps * d, nsteps, dt) - _J(c, q0 - eps * d, nsteps, dt)) / (2 * eps)
        ad = float(torch.sum(g * d))
        assert abs(fd - ad) <= 1e-6 * gnorm, (fd, ad, gnorm)
    # the gradient direction itself: the derivative is |g| and fully resolved
    d = g / gnorm
    fd = (_J(c, q0 + eps * d, nsteps, dt) - _J(c, q0 - eps * d, nsteps, dt)) / (2 * eps)
    assert abs(fd - gnorm) <= 1e-6 * gnorm, (fd, gnorm)
    # dJ/dmu0 (the viscous RHS is linear in mu0)
    h = 1e-6 * c.cfg.gas.mu0
    import dataclasses
    cp = dataclasses.replace(c.cfg, gas=dataclasses.replace(c.cfg.gas, mu0=c.cfg.gas.mu0 + h))
    cm = dataclasses.replace(c.cfg, gas=dataclasses.replace(c.cfg.gas, mu0=c.cfg.gas.mu0 - h))
    fd_mu = (_J(c, q0, nsteps, dt, cp) - _J(c, q0, nsteps, dt, cm)) / (2 * h)
    assert abs(fd_mu - dmu) <= 1e-6 * abs(dmu), (fd_mu, dmu)
    assert abs(J - _J(c, q0, nsteps, dt)) <= 1e-12 * abs(J)


def test_integrate_autograd_matches_adjoint_driver(cuda_device):
    c, st = _tgv_state(n=8)
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], 1.4, 0.5, 2)
    q0 = st.blocks[0].q.clone().requires_grad_(True)
    s0 = State(blocks=(Block(q=q0, xyz=st.blocks[0].xyz),), metrics=st.metrics)
    sN = adjoint.integrate(s0, c.cfg, dt, 5, checkpoint_every=2)
    qN = sN.blocks[0].q
    vol = st.metrics[0].vol
    inner = (slice(2, -2),) * 3
    J = torch.sum(vol[inner] * 0.5 * (qN[1][inner] ** 2 + qN[2][inner] ** 2 + qN[3][inner] ** 2) / qN[0][inner])
    J.backward()
    _, grads, _ = adjoint.adjoint_kinetic_energy(st, c.cfg, dt, 5, checkpoint_every=3)
    assert rel_l2(host(q0.grad), host(grads[0])) <= 1e-12


def test_reference_gradient_is_finite_and_nonzero(cuda_device):
    """tests/solver/test_grad.py:10-38: d(sum q after one step)/dq0 with
    farfield faces is finite and not all zero."""
    ni, nj, nk = 12, 10, 8
    rho, u, p = 1.225, 50.0, 101325.0
    q = np.zeros((5, ni, nj, nk))
    q[0], q[1], q[4] = rho, rho * u, p / 0.4 + 0.5 * rho * u * u
    kxyz = np.zeros((3, 3, ni, nj, nk))
    for d in range(3):
        kxyz[d, d] = 1.0
    one = np.ones((ni, nj, nk))
    topo = BlockTopology(0, {f: None for f in Face}, {f: BCType.FARFIELD for f in Face})
    cfg = Config(gas=GasModel(), scheme=SchemeChoice("muscl2", "roe", 3, "minmod"),
                 bc_params={f: {"q_inf": list(q[:, 0, 0, 0])} for f in Face}, topology=(topo,), ghost=2,
                 nan_check=False)
    metrics = (Metrics(jac=dev(one), kxyz=dev(kxyz), vol=dev(one)),)
    g = adjoint.step_vjp([dev(q)], metrics, cfg, 1e-6, [torch.ones((5, ni, nj, nk), dtype=torch.float64,
                                                                    device="cuda")])[0]
    assert torch.all(torch.isfinite(g)) and torch.any(g != 0)


@pytest.mark.parametrize("which", ["periodic", "mirror"])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_saved_step_vjp_matches_recomputing_vjp(cuda_device, which, precision):
    """fj_plan_step_save + fj_step_vjp_saved_f64 against fj_plan_step and the
    recomputing fj_step_vjp_mu_f64: same new state, same adjoint, same dJ/dmu0."""
    import dataclasses
    qs, mets, cfg = _periodic_case() if which == "periodic" else _mirror_case()
    cfg = dataclasses.replace(cfg, precision=precision)
    dt = 0.5 * NP.cfl_dt(qs, mets, cfg.gas.gamma, 0.5, 2)
    metrics = tuple(Metrics(jac=dev(v), kxyz=dev(k), vol=dev(v)) for k, v in mets)
    st = State(blocks=tuple(Block(q=dev(q), xyz=None) for q in qs), metrics=metrics)
    plan = StepPlan(st, cfg)
    qd = [b.q for b in st.blocks]
    ref_out = [torch.empty_like(q) for q in qd]
    plan.run(qd, ref_out, dt)
    out = [torch.empty_like(q) for q in qd]
    saved = tuple([torch.empty_like(q) for q in qd] for _ in range(3))
    plan.run_save(qd, out, *saved, dt)
    for a, b in zip(out, ref_out):
        assert torch.equal(a, b)
    lam = [dev(np.random.default_rng(3).standard_normal(q.shape)) for q in qs]
    dmu_a = torch.zeros(1, dtype=torch.float64, device="cuda")
    dmu_b = torch.zeros(1, dtype=torch.float64, device="cuda")
    ga = adjoint.step_vjp(qd, metrics, cfg, dt, lam, dmu=dmu_a)
    gb = adjoint.step_vjp_saved(saved, metrics, cfg, dt, lam, dmu=dmu_b)
    # the face adjoints are accumulated with atomics, whose order varies from
    # run to run: FP64 rounding in the FP64 path, FP32 rounding in the FP32 one
    tol = 1e-13 if precision == "f64" else 1e-6
    for a, b in zip(ga, gb):
        assert rel_l2(host(b), host(a)) <= tol
    assert abs(float(dmu_a) - float(dmu_b)) <= tol * abs(float(dmu_a))


@pytest.mark.parametrize("which", ["periodic", "mirror"])
def test_step_vjp_into_separate_or_same_buffers(cuda_device, which):
    """The step adjoint accumulates straight into ``out`` when it overlaps no
    input, and in scratch followed by a copy when ``out`` is the incoming
    adjoint itself: both give the same result (to the atomics' FP64 rounding)."""
    qs, mets, cfg = _periodic_case() if which == "periodic" else _mirror_case()
    dt = 0.5 * NP.cfl_dt(qs, mets, cfg.gas.gamma, 0.5, 2)
    metrics = tuple(Metrics(jac=dev(v), kxyz=dev(k), vol=dev(v)) for k, v in mets)
    st = State(blocks=tuple(Block(q=dev(q), xyz=None) for q in qs), metrics=metrics)
    plan = StepPlan(st, cfg)
    qd = [b.q for b in st.blocks]
    saved = tuple([torch.empty_like(q) for q in qd] for _ in range(3))
    plan.run_save(qd, [torch.empty_like(q) for q in qd], *saved, dt)
    lam = [dev(np.random.default_rng(4).standard_normal(q.shape)) for q in qs]
    separate = adjoint.step_vjp_saved(saved, metrics, cfg, dt, lam, out=[torch.empty_like(q) for q in qd])
    same = [l.clone() for l in lam]
    adjoint.step_vjp_saved(saved, metrics, cfg, dt, same, out=same)
    for a, b in zip(separate, same):
        assert rel_l2(host(b), host(a)) <= 1e-13


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_checkpoint_spacing_leaves_the_gradient_unchanged(cuda_device, precision):
    """The reverse sweep recomputes segment s-1 on a second stream into the
    second saved-state pool while the adjoints of segment s run: with a
    checkpoint every 2 or 3 steps (several overlapped segments, a short last
    one), none (one segment, nothing recomputed) or without the overlap (one
    pool, recompute between the adjoints) the 7-step gradient and dJ/dmu0 are
    the same to the atomics' rounding."""
    import dataclasses
    c, st = _tgv_state(n=10)
    cfg = dataclasses.replace(c.cfg, precision=precision)
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], 1.4, 0.5, 2)
    runs = [adjoint.adjoint_kinetic_energy(st, cfg, dt, 7, checkpoint_every=k) for k in (7, 2, 3)]
    runs.append(adjoint.adjoint_kinetic_energy(st, cfg, dt, 7, checkpoint_every=2, overlap=False))
    tol = 1e-13 if precision == "f64" else 1e-6
    J0, g0, m0 = runs[0]
    for J, g, m in runs[1:]:
        assert J == J0
        assert rel_l2(host(g[0]), host(g0[0])) <= tol
        assert abs(m - m0) <= tol * abs(m0)


def test_mu_gradient_matches_autograd(cuda_device):
    """dJ/dmu0 of one step (J = lam . q_new) against torch.autograd of the
    oracle's twin with mu0 as a leaf."""
    import dataclasses
    qs, mets, cfg = _periodic_case()
    dt = 0.5 * NP.cfl_dt(qs, mets, cfg.gas.gamma, 0.5, 2)
    lam = [np.random.default_rng(5).standard_normal(q.shape) for q in qs]
    h = 1e-2 * cfg.gas.mu0

    def J(mu):
        c2 = dataclasses.replace(cfg, gas=dataclasses.replace(cfg.gas, mu0=mu))
        out = TORCH.step([torch.tensor(q) for q in qs], [(torch.tensor(k), torch.tensor(v)) for k, v in mets], c2, dt)
        return sum(float(torch.sum(o * torch.tensor(l))) for o, l in zip(out, lam))
    # J is nearly linear in mu0 (exactly linear within one stage): central
    # differences of the FP64 oracle agree to ~1e-8 between h = 1e-2 mu0 and
    # 1e-3 mu0; the larger h keeps the cancellation error smallest
    ref = (J(cfg.gas.mu0 + h) - J(cfg.gas.mu0 - h)) / (2 * h)
    metrics = tuple(Metrics(jac=dev(v), kxyz=dev(k), vol=dev(v)) for k, v in mets)
    dmu = torch.zeros(1, dtype=torch.float64, device="cuda")
    adjoint.step_vjp([dev(q) for q in qs], metrics, cfg, dt, [dev(l) for l in lam], dmu=dmu)
    assert abs(float(dmu) - ref) <= 1e-7 * abs(ref), (float(dmu), ref)


def test_f32_mu_gradient_close_to_f64(cuda_device):
    """dJ/dmu0 of one step accumulated by the FP32-flux viscous VJP (inside
    the combined face + viscous launch) against the FP64 path's, and the
    step's input adjoint likewise.  Bounds: 1e-6 relative (measured 5.7e-8
    and 1.7e-8)."""
    import dataclasses
    qs, mets, cfg = _periodic_case()
    dt = 0.5 * NP.cfl_dt(qs, mets, cfg.gas.gamma, 0.5, 2)
    lam = [np.random.default_rng(5).standard_normal(q.shape) for q in qs]
    metrics = tuple(Metrics(jac=dev(v), kxyz=dev(k), vol=dev(v)) for k, v in mets)
    vals, grads = {}, {}
    for prec in ("f64", "f32"):
        c2 = dataclasses.replace(cfg, precision=prec)
        dmu = torch.zeros(1, dtype=torch.float64, device="cuda")
        grads[prec] = host(adjoint.step_vjp([dev(q) for q in qs], metrics, c2, dt, [dev(l) for l in lam],
                                            dmu=dmu)[0])
        vals[prec] = float(dmu)
    assert abs(vals["f32"] - vals["f64"]) <= 1e-6 * abs(vals["f64"])
    assert rel_l2(grads["f32"], grads["f64"]) <= 1e-6


def test_mach_gradient_matches_finite_differences(cuda_device):
    """dJ/dM0 of the kinetic-energy objective: M0 enters the Taylor-Green
    initial state and the viscosity mu0 = rho0 M0 / Re, so
    dJ/dM0 = dJ/dq0 . dq0/dM0 + dJ/dmu0 * rho0 / Re, with dt held fixed (it is
    computed once from the initial state).  Central differences regenerate
    the case at M0 +- h with the same seed (the same noise draws); h keeps the
    state perturbation near 1e-7 in L2, as in the trajectory test."""
    n, M0, Re, nsteps = 12, 0.3, 800.0, 4

    def case(m):
        return cases.tgv(n=n, M0=m, Re=Re, noise=0.01, seed=2)

    c = case(M0)
    st = cases.to_state(c, "cuda:0")
    dt = NP.cfl_dt(c.qs, [(m[1], m[2]) for m in c.metrics], 1.4, 0.5, 2)
    J, grads, dmu = adjoint.adjoint_kinetic_energy(st, c.cfg, dt, nsteps, checkpoint_every=2)
    dq = torch.tensor(cases.tgv_dq0_dM0(c), device="cuda")
    dJ = float(torch.sum(grads[0] * dq)) + dmu * 1.0 / Re
    h = 1e-8 * M0

    def J_of(m):
        cm = case(m)
        s = cases.to_state(cm, "cuda:0")
        plan = StepPlan(s, cm.cfg)
        for _ in range(nsteps):
            s = step(s, cm.cfg, dt, plan=plan)
        return diagnostics.kinetic_energy(s, 2)

    fd = (J_of(M0 + h) - J_of(M0 - h)) / (2 * h)
    assert abs(fd - dJ) <= 1e-6 * abs(dJ), (fd, dJ)


def test_ensemble_matches_separate_instances(cuda_device):
    """An ensemble plan (per-block mu0 and dt, all blocks per launch) steps each
    instance exactly like a plan of that instance alone, and matches the
    oracle; the per-instance adjoint (J_b, dJ_b/dq0_b, dJ_b/dmu0_b) matches the
    single-instance adjoint."""
    import dataclasses
    ens = cases.ensemble(ninst=3, n=8, seed=5, precision="f64")
    st = cases.to_state(ens, "cuda:0")
    mets = [(m[1], m[2]) for m in ens.metrics]
    dts = [NP.cfl_dt([q], [mt], 1.4, 0.5, 2) for q, mt in zip(ens.qs, mets)]
    mu0s = ens.meta["mu0"]
    plan = StepPlan(st, ens.cfg)
    plan.set_ensemble(mu0s, dts)
    qa = [b.q.clone() for b in st.blocks]
    qb = [torch.empty_like(q) for q in qa]
    nsteps = 3
    for _ in range(nsteps):
        plan.run(qa, qb, 123.0)  # the dt argument is ignored while per-block dt is set
        qa, qb = qb, qa
    for b in range(3):
        cfg_b = dataclasses.replace(ens.cfg, gas=dataclasses.replace(ens.cfg.gas, mu0=mu0s[b]),
                                    topology=(cases._self_periodic_topology(0),))
        s_b = State(blocks=(st.blocks[b],), metrics=(st.metrics[b],))
        p_b = StepPlan(s_b, cfg_b)
        x = [st.blocks[b].q.clone()]
        y = [torch.empty_like(x[0])]
        ref = [ens.qs[b]]
        for _ in range(nsteps):
            p_b.run(x, y, dts[b])
            x, y = y, x
            ref = NP.step(ref, [mets[b]], cfg_b, dts[b])
        assert torch.equal(x[0], qa[b]), b
        assert rel_l2(host(qa[b]), ref[0]) <= 1e-12
    Js, grads, dmus = adjoint.adjoint_kinetic_energy_ensemble(st, ens.cfg, nsteps, mu0s=mu0s, dts=dts,
                                                              checkpoint_every=2)
    for b in range(3):
        cfg_b = dataclasses.replace(ens.cfg, gas=dataclasses.replace(ens.cfg.gas, mu0=mu0s[b]),
                                    topology=(cases._self_periodic_topology(0),))
        s_b = State(blocks=(st.blocks[b],), metrics=(st.metrics[b],))
        J, g, dmu = adjoint.adjoint_kinetic_energy(s_b, cfg_b, dts[b], nsteps, checkpoint_every=2)
        assert abs(J - Js[b]) <= 1e-14 * abs(J)
        assert rel_l2(host(grads[b]), host(g[0])) <= 1e-13
        assert abs(dmu - dmus[b]) <= 1e-12 * abs(dmu)

"""The persistent step kernel (FP32 fluxes / FP64 state) through the C ABI.

The persistent step runs the split kernels' arithmetic in one launch over a
dependency-ordered work-list (halo gathers and scatters, boundary faces,
primitives, and the flux and assembly chunks of the three stages), so:
  * persistent vs split: bit-identical states after every step (halo links,
    farfield / wall / symmetry faces, uneven and ragged blocks, ensembles,
    every launch shape, graph replays, the adjoint's saving step), and so is
    the split path behind the fused ghost fill (the list's head alone);
  * persistent vs the FP64 oracle: relative L2 of q <= 1e-5 after the steps
    run (the FP32-flux bound of the other parity tests);
  * a bounded wait that runs out is reported by fj_plan_check and leaves the
    plan usable.
"""
import dataclasses

import numpy as np
import pytest
import torch

from famrdp_jax_b200 import _capi, cases
from famrdp_jax_b200.solver.step import StepPlan
from oracle.ref import NP
from parity_util import host, state_from_case

pytestmark = pytest.mark.gpu


def _plan(case, kernel, precision="f32"):
    cfg = dataclasses.replace(case.cfg, precision=precision)
    st = state_from_case(case)
    plan = StepPlan(st, cfg)
    plan.set_kernel(kernel)
    assert plan.kernel == kernel
    return plan, st


def _steps(plan, st, n, dt, graph=False):
    a = [b.q.clone() for b in st.blocks]
    b = [torch.empty_like(x) for x in a]
    out = []
    for _ in range(n):
        plan.run(a, b, dt, graph=graph)
        a, b = b, a
        out.append([x.clone() for x in a])
    assert plan.check() == 0
    return out


def _dt(case):
    return NP.cfl_dt(case.qs, [(m[1], m[2]) for m in case.metrics], case.cfg.gas.gamma, case.cfl, 2)


def _rel(got, ref):
    num = sum(float(np.sum((host(a) - b) ** 2)) for a, b in zip(got, ref))
    den = sum(float(np.sum(b ** 2)) for b in ref)
    return (num / den) ** 0.5


def _mirror_case(limiter="minmod", visc_law="sutherland", iso=False):
    """One block with farfield, symmetry and wall faces and a self-periodic k
    pair, a perturbed non-diagonal metric field."""
    from types import SimpleNamespace
    from famrdp_jax_b200.core.constants import BCType, Face
    from famrdp_jax_b200.core.types import BlockTopology, Config, GasModel, SchemeChoice
    from parity_util import random_block
    q, kxyz, vol = random_block((14, 19, 37), 8, noise=0.03)
    faces = {Face.IMIN: BCType.FARFIELD, Face.IMAX: BCType.SYMMETRY, Face.JMIN: BCType.WALL,
             Face.JMAX: BCType.FARFIELD, Face.KMIN: BCType.CUT1TO1, Face.KMAX: BCType.CUT1TO1}
    nb = {f: None for f in Face}
    nb[Face.KMIN] = (0, Face.KMAX, 0)
    nb[Face.KMAX] = (0, Face.KMIN, 0)
    topo = BlockTopology(0, nb, faces)
    q_inf = [float(x) for x in q[:, 4, 4, 4]]
    gas = GasModel(gamma=1.4, R=1.0, mu0=2e-3, T0=1 / 1.4, Ts=0.27, Pr_lam=0.72, visc_law=visc_law)
    params = {f: {"q_inf": q_inf} for f in Face}
    if iso:
        params[Face.JMIN] = {"q_inf": q_inf, "wall_type": "isothermal", "T_wall": 0.8}
    cfg = Config(gas=gas, scheme=SchemeChoice("muscl2", "roe", 3, limiter), bc_params=params, topology=(topo,),
                 ghost=2, nan_check=False, precision="f32")
    return SimpleNamespace(qs=[q], metrics=[(vol, kxyz, vol)], cfg=cfg, cfl=0.3)


def _case(name):
    if name == "tgv32":
        return cases.tgv(n=32, noise=0.01, seed=1), 4
    if name == "wavy4":
        return cases.wavy4(n=12, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2)), 3
    if name == "tree24":
        return cases.tree24(nblocks=24, lo=6, hi=14, seed=3), 3
    if name == "ragged":
        # tiny i extents (planes smaller than a chunk), partial chunks everywhere
        return cases.tree24(nblocks=5, lo=3, hi=23, seed=7), 3
    if name == "mirror":
        return _mirror_case(), 3
    if name == "isothermal":
        return _mirror_case(limiter="vanleer", visc_law="constant", iso=True), 3
    raise KeyError(name)


@pytest.mark.parametrize("kernel", ["persistent", "split_fill"])
@pytest.mark.parametrize("name", ["tgv32", "wavy4", "tree24", "ragged", "mirror", "isothermal"])
def test_persistent_step_is_bit_identical_to_split(cuda_device, name, kernel):
    """The persistent step, and the split kernels behind the fused ghost fill
    (the work-list's head: halo, boundary faces, primitives in one launch)."""
    c, n = _case(name)
    dt = _dt(c)
    res = {}
    for k in ("split", kernel):
        plan, st = _plan(c, k)
        res[k] = _steps(plan, st, n, dt)
    for s in range(n):
        for a, b in zip(res[kernel][s], res["split"][s]):
            assert torch.equal(a, b), (name, kernel, s)


@pytest.mark.parametrize("name", ["wavy4", "tree24", "mirror"])
def test_persistent_steps_match_oracle(cuda_device, name):
    c, n = _case(name)
    dt = _dt(c)
    plan, st = _plan(c, "persistent")
    got = _steps(plan, st, n, dt, graph=True)
    qs = [q.copy() for q in c.qs]
    mets = [(m[1], m[2]) for m in c.metrics]
    cfg64 = dataclasses.replace(c.cfg, precision="f64")
    errs = []
    for s in range(n):
        qs = NP.step(qs, mets, cfg64, dt)
        errs.append(_rel(got[s], qs))
    print(name, ["%.2e" % e for e in errs])
    assert max(errs) <= 1e-5, errs


def test_persistent_graph_replay_and_shapes(cuda_device):
    c = cases.tree24(nblocks=6, lo=8, hi=36, seed=5)
    dt = _dt(c)
    plan, st = _plan(c, "persistent")
    ref = _steps(plan, st, 2, dt)
    for shape in range(_capi.NUM_PERSIST_SHAPES):
        plan.set_persist_shape(shape)
        for graph in (False, True):
            got = _steps(plan, st, 2, dt, graph=graph)
            for x, y in zip(got, ref):
                for a, b in zip(x, y):
                    assert torch.equal(a, b), shape


def test_persistent_shapes_on_large_blocks(cuda_device):
    """Blocks large enough that every launch shape's ordering interleaves
    flux and assembly chunks of one block (the lag shapes) or of two blocks
    (the mixing shapes): every shape bit-identical to the split kernels."""
    for c in (cases.tgv(n=60, noise=0.01, seed=4), cases.tree24(nblocks=3, lo=40, hi=64, seed=8)):
        dt = _dt(c)
        ref_plan, ref_st = _plan(c, "split")
        ref = _steps(ref_plan, ref_st, 1, dt)[0]
        plan, st = _plan(c, "persistent")
        for shape in range(_capi.NUM_PERSIST_SHAPES):
            plan.set_persist_shape(shape)
            got = _steps(plan, st, 1, dt)[0]
            for a, b in zip(got, ref):
                assert torch.equal(a, b), shape


def test_persistent_ensemble_matches_split(cuda_device):
    from famrdp_jax_b200.core.types import State
    from famrdp_jax_b200.solver import diagnostics
    c = cases.ensemble(ninst=5, n=12, seed=2)
    st0 = state_from_case(c)
    mu0 = c.meta["mu0"]
    dts = [diagnostics.cfl_dt(State(blocks=(b,), metrics=(m,)), c.cfg, c.cfl) for b, m in zip(st0.blocks, st0.metrics)]
    dt = _dt(c)
    res = {}
    for kernel in ("split", "persistent"):
        plan, st = _plan(c, kernel)
        plan.set_ensemble(mu0, dts)
        res[kernel] = _steps(plan, st, 2, dt)
    for x, y in zip(res["persistent"], res["split"]):
        for a, b in zip(x, y):
            assert torch.equal(a, b)


def test_persistent_saving_step_matches_split(cuda_device):
    """The adjoint's saving step (stage values into caller buffers)."""
    c = cases.tree24(nblocks=4, lo=6, hi=12, seed=9)
    dt = _dt(c)
    res = {}
    for kernel in ("split", "persistent"):
        plan, st = _plan(c, kernel)
        qs = [b.q for b in st.blocks]
        out = [torch.empty_like(q) for q in qs]
        saved = tuple([torch.empty_like(q) for q in qs] for _ in range(3))
        plan.run_save(qs, out, *saved, dt)
        assert plan.check() == 0
        res[kernel] = [out] + list(saved)
    for x, y in zip(res["persistent"], res["split"]):
        for a, b in zip(x, y):
            assert torch.equal(a, b)


def test_persistent_bounded_wait_gives_up_and_recovers(cuda_device):
    """Failure detection without a fault: with a wait limit of 0 every wait
    on a completion counter gives up at once; the CTA records it in the
    plan's error word and raises the abort flag, every CTA stops taking items
    and the launch ends; fj_plan_check reports it.  With the default limit the
    next step is bit-identical to the split kernels' again."""
    c = cases.tree24(nblocks=3, lo=8, hi=16, seed=11)
    dt = _dt(c)
    ref_plan, ref_st = _plan(c, "split")
    ref = _steps(ref_plan, ref_st, 1, dt)[0]
    plan, st = _plan(c, "persistent")
    a = [b.q.clone() for b in st.blocks]
    b = [torch.empty_like(x) for x in a]
    plan.set_wait_limit(0)
    plan.run(a, b, dt)
    with pytest.raises(RuntimeError, match="bounded wait of the persistent step"):
        plan.check()
    assert plan.check() == 0  # the word was cleared
    plan.set_wait_limit(-1)
    a = [x.q.clone() for x in st.blocks]
    plan.run(a, b, dt)
    assert plan.check() == 0
    for x, y in zip(b, ref):
        assert torch.equal(x, y)


def test_persistent_refused_where_it_does_not_apply(cuda_device):
    c = cases.tgv(n=8)
    plan = StepPlan(state_from_case(c), dataclasses.replace(c.cfg, precision="f64"))
    with pytest.raises(Exception):
        plan.set_kernel("persistent")
    assert plan.kernel == "split"
    # more blocks than one launch's table holds
    c = cases.tree24(nblocks=65, lo=4, hi=5, seed=1)
    plan = StepPlan(state_from_case(c), dataclasses.replace(c.cfg, precision="f32"))
    with pytest.raises(Exception):
        plan.set_kernel("persistent")
    assert plan.kernel == "split"


@pytest.mark.parametrize("kernel", ["persistent", "split_fill"])
def test_adjoint_through_persistent_forward(cuda_device, kernel):
    """The checkpointed adjoint with its forward sweeps (plain, saving and
    recomputing steps, some on a second stream) run by the persistent step or
    the fused ghost fill: J bit-identical to the split kernels' (the forward
    is); dJ/dq0 and dJ/dmu0 within 1e-6 relative, because the reverse sweep
    accumulates face and viscosity adjoints with atomics, whose order (and so
    rounding) differs from run to run even with the same forward."""
    from famrdp_jax_b200.solver import adjoint
    c = cases.tree24(nblocks=3, lo=8, hi=14, seed=13)
    dt = _dt(c)
    res = {}
    for k in ("split", kernel):
        plan, st = _plan(c, k)
        J, g, dmu = adjoint.adjoint_kinetic_energy(st, dataclasses.replace(c.cfg, precision="f32"), dt, 6,
                                                   checkpoint_every=2, plan=plan)
        assert plan.check() == 0
        res[k] = (float(J), [x.clone() for x in g], float(dmu))
    assert res[kernel][0] == res["split"][0]
    assert abs(res[kernel][2] - res["split"][2]) <= 1e-6 * abs(res["split"][2])
    num = sum(float(torch.sum((a - b) ** 2)) for a, b in zip(res[kernel][1], res["split"][1]))
    den = sum(float(torch.sum(b ** 2)) for b in res["split"][1])
    assert (num / den) ** 0.5 <= 1e-6


def test_persist_shape_argument_errors(cuda_device):
    c = cases.tgv(n=8)
    plan, st = _plan(c, "persistent")
    for bad in (-1, _capi.NUM_PERSIST_SHAPES):
        with pytest.raises(ValueError):
            plan.set_persist_shape(bad)
    plan.set_persist_shape(_capi.NUM_PERSIST_SHAPES - 1)
    assert plan.kernel == "persistent"

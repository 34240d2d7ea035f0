"""The fused TMA-tile stage kernel (FP32 fluxes / FP64 state) through the C ABI.

Tolerances: the tile kernel evaluates the same face, viscous and combine
arithmetic as the split kernels in FP32 (the temperature is formed in FP32
from the stored pressure, the split kernels store it from FP64), so
  * tile vs the FP64 oracle: relative L2 of q <= 1e-5 after the steps run
    (the FP32-flux bound of the other parity tests);
  * tile vs split (both FP32-flux): relative L2 <= 1e-7 after one step;
  * graph replays of the tile step: bit-identical to plain tile steps.
"""
import dataclasses

import numpy as np
import pytest
import torch

from famrdp_jax_b200 import cases
from famrdp_jax_b200.solver.step import StepPlan
from oracle.ref import NP
from parity_util import host, rel_l2, state_from_case

pytestmark = pytest.mark.gpu


def _plan(case, kernel, precision="f32"):
    cfg = dataclasses.replace(case.cfg, precision=precision)
    st = state_from_case(case)
    plan = StepPlan(st, cfg)
    plan.set_kernel(kernel)
    assert plan.kernel == kernel
    return plan, st, cfg


def _steps(plan, st, n, dt, graph=False):
    a = [b.q.clone() for b in st.blocks]
    b = [torch.empty_like(x) for x in a]
    out = []
    for _ in range(n):
        plan.run(a, b, dt, graph=graph)
        a, b = b, a
        out.append([host(x).copy() for x in a])
    assert plan.check() == 0
    return out


def _dt(case):
    return NP.cfl_dt(case.qs, [(m[1], m[2]) for m in case.metrics], case.cfg.gas.gamma, case.cfl, 2)


def _rel(got, ref):
    num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(got, ref))
    den = sum(float(np.sum(b ** 2)) for b in ref)
    return (num / den) ** 0.5


@pytest.mark.parametrize("name", ["tgv32", "wavy4", "tree", "ragged"])
def test_tile_steps_match_oracle(cuda_device, name):
    if name == "tgv32":
        c, n = cases.tgv(n=32), 10
    elif name == "wavy4":
        c, n = cases.wavy4(n=12, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2)), 3
    elif name == "tree":
        c, n = cases.tree24(nblocks=6, lo=6, hi=12, seed=1), 3
    else:
        # extents that leave partial tiles in j (not a multiple of 8) and k (not
        # a multiple of 30), k wider than one tile, tiny i
        c, n = cases.tree24(nblocks=3, lo=3, hi=40, seed=7), 3
    dt = _dt(c)
    plan, st, _ = _plan(c, "tile")
    got = _steps(plan, st, n, dt)
    qs = [q.copy() for q in c.qs]
    mets = [(m[1], m[2]) for m in c.metrics]
    errs = []
    for s in range(n):
        qs = NP.step(qs, mets, c.cfg, dt)
        errs.append(_rel(got[s], qs))
    print(name, [q.shape for q in c.qs], ["%.2e" % e for e in errs])
    assert max(errs) <= 1e-5, errs


@pytest.mark.parametrize("name", ["wavy4", "tree", "ensemble"])
def test_tile_matches_split_kernels(cuda_device, name):
    if name == "wavy4":
        c = cases.wavy4(n=20, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2))
        ens = None
    elif name == "tree":
        c = cases.tree24(nblocks=8, lo=8, hi=40, seed=3)
        ens = None
    else:
        c = cases.ensemble(ninst=5, n=12, seed=2)
        st0 = state_from_case(c)
        from famrdp_jax_b200.core.types import State
        from famrdp_jax_b200.solver import diagnostics
        ens = (c.meta["mu0"], [diagnostics.cfl_dt(State(blocks=(b,), metrics=(m,)), c.cfg, c.cfl)
                               for b, m in zip(st0.blocks, st0.metrics)])
    dt = _dt(c)
    res = {}
    for kernel in ("split", "tile"):
        plan, st, _ = _plan(c, kernel)
        if ens:
            plan.set_ensemble(*ens)
        res[kernel] = _steps(plan, st, 2, dt)
    e1 = _rel(res["tile"][0], res["split"][0])
    e2 = _rel(res["tile"][1], res["split"][1])
    print(name, "tile vs split after 1 / 2 steps: %.2e %.2e" % (e1, e2))
    assert e1 <= 1e-7 and e2 <= 2e-7, (e1, e2)


def test_tile_graph_replay_is_bit_identical(cuda_device):
    c = cases.tree24(nblocks=4, lo=8, hi=36, seed=5)
    dt = _dt(c)
    plan, st, _ = _plan(c, "tile")
    plain = _steps(plan, st, 3, dt)
    graphed = _steps(plan, st, 3, dt, graph=True)
    for a, b in zip(plain, graphed):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_tile_stage_matches_split_stage(cuda_device):
    """fj_plan_stage (one stage-2 evaluation, the bench's roofline group)."""
    c = cases.wavy4(n=16, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2))
    dt = _dt(c)
    outs = {}
    for kernel in ("split", "tile"):
        plan, st, _ = _plan(c, kernel)
        q0 = [b.q for b in st.blocks]
        qin = [q * (1.0 + 1e-3 * torch.sin(torch.arange(q.numel(), device=q.device, dtype=q.dtype)).reshape(q.shape))
               for q in q0]
        out = [torch.empty_like(q) for q in q0]
        plan.stage(qin, q0, out, dt, 2)
        assert plan.check() == 0
        outs[kernel] = [host(x) for x in out]
    e = _rel(outs["tile"], outs["split"])
    assert e <= 1e-7, e


def test_tile_bounded_wait_gives_up_and_recovers(cuda_device):
    """Failure detection without a fault: with a wait limit of 0 every wait for
    a TMA copy gives up at once; the kernel records it in the plan's error
    word, waits for its copies in flight and exits; fj_plan_check reports it.
    With the default limit the next step is correct again."""
    c = cases.tgv(n=16, noise=0.01, seed=3)
    dt = _dt(c)
    plan, st, _ = _plan(c, "tile")
    a = [b.q.clone() for b in st.blocks]
    b = [torch.empty_like(x) for x in a]
    plan.set_wait_limit(0)
    plan.run(a, b, dt)
    with pytest.raises(RuntimeError, match="bounded wait"):
        plan.check()
    assert plan.check() == 0  # the word was cleared
    plan.set_wait_limit(-1)
    plan.run(a, b, dt)
    assert plan.check() == 0
    ref = NP.step([q.copy() for q in c.qs], [(m[1], m[2]) for m in c.metrics], c.cfg, dt)
    assert rel_l2(host(b[0]), ref[0]) <= 1e-5


def test_tile_kernel_refused_for_fp64(cuda_device):
    c = cases.tgv(n=8)
    cfg = dataclasses.replace(c.cfg, precision="f64")
    plan = StepPlan(state_from_case(c), cfg)
    with pytest.raises(Exception):
        plan.set_kernel("tile")
    assert plan.kernel == "split"


@pytest.mark.parametrize("limiter", ["minmod", "vanleer"])
@pytest.mark.parametrize("visc_law", ["sutherland", "constant"])
def test_tile_mirror_bcs_limiters_and_viscosity_laws(cuda_device, limiter, visc_law):
    """One block with farfield, symmetry and adiabatic-wall faces and a
    self-periodic pair, a non-diagonal perturbed metric field, both limiters
    and both viscosity laws: tile kernel vs the FP64 oracle after 3 steps."""
    from famrdp_jax_b200.core.constants import BCType, Face
    from famrdp_jax_b200.core.types import BlockTopology, Config, GasModel, SchemeChoice
    from parity_util import random_block
    from types import SimpleNamespace
    q, kxyz, vol = random_block((14, 19, 37), 8, noise=0.03)
    faces = {Face.IMIN: BCType.FARFIELD, Face.IMAX: BCType.SYMMETRY, Face.JMIN: BCType.WALL,
             Face.JMAX: BCType.FARFIELD, Face.KMIN: BCType.CUT1TO1, Face.KMAX: BCType.CUT1TO1}
    nb = {f: None for f in Face}
    nb[Face.KMIN] = (0, Face.KMAX, 0)
    nb[Face.KMAX] = (0, Face.KMIN, 0)
    topo = BlockTopology(0, nb, faces)
    q_inf = [float(x) for x in q[:, 4, 4, 4]]
    gas = GasModel(gamma=1.4, R=1.0, mu0=2e-3, T0=1 / 1.4, Ts=0.27, Pr_lam=0.72, visc_law=visc_law)
    cfg = Config(gas=gas, scheme=SchemeChoice("muscl2", "roe", 3, limiter),
                 bc_params={f: {"q_inf": q_inf} for f in Face}, topology=(topo,), ghost=2, nan_check=False,
                 precision="f32")
    c = SimpleNamespace(qs=[q], metrics=[(vol, kxyz, vol)], cfg=cfg, cfl=0.3)
    dt = _dt(c)
    plan, st, _ = _plan(c, "tile")
    got = _steps(plan, st, 3, dt)
    qs = [q.copy()]
    mets = [(kxyz, vol)]
    cfg64 = dataclasses.replace(cfg, precision="f64")
    for s in range(3):
        qs = NP.step(qs, mets, cfg64, dt)
        e = _rel(got[s], qs)
        assert e <= 1e-5, (s, e)

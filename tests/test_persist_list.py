"""The persistent step's work-list on the host (no GPU): for several block
layouts, link sets and boundary faces, every launch shape and several grid
sizes, the list the plan would run has the expected number of items and every
item waits only for items ahead of it (fj_persist_list_check), which is what
makes the one-launch step deadlock-free."""
import ctypes
import math

import pytest

from famrdp_jax_b200 import _capi, _topology, cases
from oracle.ref import NP

FLUX_CELLS, ASM_CELLS, HALO_CHUNK = 224, 217, 2048  # per flux / assembly chunk, per halo or BC item


def _arrays(case, precision="f32"):
    cfg = case.cfg
    shapes = [tuple(q.shape[1:]) for q in case.qs]
    blocks = (_capi.FjBlock * len(shapes))()
    for b, (ni, nj, nk) in enumerate(shapes):
        blocks[b].ni, blocks[b].nj, blocks[b].nk = ni, nj, nk
    links = _topology.links(cfg.topology)
    bcs = _topology.bcs(cfg.topology, cfg)
    p = _capi.params(cfg.gas, limiter=cfg.scheme.limiter, ghost=cfg.ghost, precision=precision)
    return shapes, links, bcs, blocks, _topology.link_array(links), _topology.bc_array(bcs), p


def _expected_items(shapes, links, bcs, g):
    n = 0
    for (t, tf, s, sf, o) in links:
        ext = list(shapes[t])
        ext[tf // 2] = g
        V = ext[0] * ext[1] * ext[2]
        n += math.ceil(5 * V / HALO_CHUNK) + math.ceil(V / HALO_CHUNK)
    for (b, f, ty, iso, tw, qi) in bcs:
        area = shapes[b][0] * shapes[b][1] * shapes[b][2] // shapes[b][f // 2]
        n += math.ceil(g * area / HALO_CHUNK)
    for (ni, nj, nk) in shapes:
        N = ni * nj * nk
        n += math.ceil(N / FLUX_CELLS) + 3 * (math.ceil(N / FLUX_CELLS) + math.ceil(N / ASM_CELLS))
    return n


def _check(case, grid, shape):
    shapes, links, bcs, blocks, la, ba, p = _arrays(case)
    n = ctypes.c_int64(-1)
    st = _capi.lib().fj_persist_list_check(blocks, len(shapes), la, len(links), ba, len(bcs), ctypes.byref(p),
                                           grid, shape, ctypes.byref(n))
    return st, n.value, _expected_items(shapes, links, bcs, case.cfg.ghost)


def _mirror():
    from types import SimpleNamespace
    from famrdp_jax_b200.core.constants import BCType, Face
    from famrdp_jax_b200.core.types import BlockTopology, Config, GasModel, SchemeChoice
    import numpy as np
    faces = {Face.IMIN: BCType.FARFIELD, Face.IMAX: BCType.SYMMETRY, Face.JMIN: BCType.WALL,
             Face.JMAX: BCType.FARFIELD, Face.KMIN: BCType.CUT1TO1, Face.KMAX: BCType.CUT1TO1}
    nb = {f: None for f in Face}
    nb[Face.KMIN] = (0, Face.KMAX, 0)
    nb[Face.KMAX] = (0, Face.KMIN, 0)
    gas = GasModel(gamma=1.4, R=1.0, mu0=2e-3, T0=1 / 1.4, Ts=0.27, Pr_lam=0.72)
    cfg = Config(gas=gas, scheme=SchemeChoice("muscl2", "roe", 3, "minmod"),
                 bc_params={f: {"q_inf": [1.0, 0.1, 0.0, 0.0, 2.5]} for f in Face},
                 topology=(BlockTopology(0, nb, faces),), ghost=2, nan_check=False, precision="f32")
    return SimpleNamespace(qs=[np.zeros((5, 14, 19, 37))], cfg=cfg)


CASES = {
    "tgv32": lambda: cases.tgv(n=32),
    "tgv60": lambda: cases.tgv(n=60),
    "wavy4": lambda: cases.wavy4(n=12, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2)),
    "tree24": lambda: cases.tree24(nblocks=24, lo=6, hi=40, seed=3),
    "ragged": lambda: cases.tree24(nblocks=5, lo=3, hi=23, seed=7),
    "mirror": _mirror,
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("shape", range(_capi.NUM_PERSIST_SHAPES))
def test_work_list_is_ordered_and_complete(name, shape):
    case = CASES[name]()
    for grid in (1, 7, 444, 592):
        st, n, expected = _check(case, grid, shape)
        assert st == _capi.FJ_OK, (name, shape, grid, st)
        assert n == expected, (name, shape, grid, n, expected)


def test_work_list_refused_where_the_step_does_not_apply():
    case = cases.tree24(nblocks=65, lo=4, hi=5, seed=1)  # more blocks than one launch's table holds
    st, n, _ = _check(case, 592, 0)
    assert st == _capi.FJ_ERR_NOT_IMPLEMENTED
    shapes, links, bcs, blocks, la, ba, p = _arrays(cases.tgv(n=8), precision="f64")
    assert _capi.lib().fj_persist_list_check(blocks, len(shapes), la, len(links), ba, len(bcs), ctypes.byref(p),
                                             592, 0, None) == _capi.FJ_ERR_NOT_IMPLEMENTED
    shapes, links, bcs, blocks, la, ba, p = _arrays(cases.tgv(n=8))
    for grid, shape in ((0, 0), (592, -1), (592, _capi.NUM_PERSIST_SHAPES)):
        assert _capi.lib().fj_persist_list_check(blocks, len(shapes), la, len(links), ba, len(bcs),
                                                 ctypes.byref(p), grid, shape, None) == _capi.FJ_ERR_INVALID_ARGUMENT


def test_work_list_with_mapped_and_overlapping_links():
    """Links between faces of different axes in every mapped orientation,
    target slabs that overlap at edges, a block linked to itself, and no
    boundary faces."""
    from famrdp_jax_b200.core.constants import Face, mapped_orientation as m
    shapes = [(8, 9, 10), (9, 10, 7), (6, 10, 8)]
    spec = [
        [(Face.IMAX, 1, Face.KMIN, m(reverse_a=True)), (Face.JMIN, 2, Face.IMAX, m(swap=True, reverse_b=True)),
         (Face.KMAX, 0, Face.KMIN, m(reverse_a=True, reverse_b=True)), (Face.KMIN, 0, Face.KMAX, 0)],
        [(Face.KMIN, 0, Face.IMAX, m(reverse_a=True)), (Face.IMIN, 1, Face.IMAX, 0), (Face.IMAX, 1, Face.IMIN, m())],
        [(Face.IMAX, 0, Face.JMIN, m(swap=True)), (Face.JMAX, 2, Face.JMIN, m(reverse_a=True, reverse_b=True))],
    ]
    links = [(b, int(f), sb, int(sf), o) for b, s in enumerate(spec) for f, sb, sf, o in s]
    blocks = (_capi.FjBlock * 3)()
    for b, (ni, nj, nk) in enumerate(shapes):
        blocks[b].ni, blocks[b].nj, blocks[b].nk = ni, nj, nk
    gas = cases.tgv(n=8).cfg.gas
    p = _capi.params(gas, limiter="minmod", ghost=2, precision="f32")
    expected = _expected_items(shapes, links, [], 2)
    for shape in range(_capi.NUM_PERSIST_SHAPES):
        for grid in (1, 5, 592):
            n = ctypes.c_int64(-1)
            st = _capi.lib().fj_persist_list_check(blocks, 3, _topology.link_array(links), len(links),
                                                   _topology.bc_array([]), 0, ctypes.byref(p), grid, shape,
                                                   ctypes.byref(n))
            assert st == _capi.FJ_OK and n.value == expected, (shape, grid, st, n.value, expected)

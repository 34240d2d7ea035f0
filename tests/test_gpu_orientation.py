"""Mapped interface orientations on the GPU (an extension: the reference's
halo fill rejects every orientation but 0, mesh/halo.py:86-87).

* The halo fill through the C ABI against the NumPy statement of the mapping
  (tests/orientation_util.py), bit for bit, on three blocks joined by links
  between faces of different axes with every swap/reversal bit, mixed with
  the reference's orientation-0 copy, overlapping ghost slabs included.
* Physical equivalence: a periodic box of two blocks stepped once as built
  and once with the second block stored with its j and k axes swapped and/or
  reversed (its metrics relabelled to match, its interfaces described by
  mapped orientations): after several steps the two runs hold the same
  solution (relative L2 <= 1e-12 in FP64, the difference being the order of
  the per-axis sums), and so do their step adjoints (which run the
  transposed mapped halo fill).
"""
import numpy as np
import pytest
import torch

from famrdp_jax_b200.core.constants import BCType, Face, mapped_orientation
from famrdp_jax_b200.core.types import Block, BlockTopology, Config, GasModel, Metrics, SchemeChoice, State
from famrdp_jax_b200.mesh.halo import halo_exchange
from famrdp_jax_b200.solver import adjoint
from famrdp_jax_b200.solver.step import step
from oracle.ref import NP
from orientation_util import mapped_halo, relabel, relabel_kxyz, unrelabel
from parity_util import dev, host, random_block, rel_l2

pytestmark = pytest.mark.gpu

G = 2


def _cfg(topology, precision="f64"):
    gas = GasModel(gamma=1.4, R=1.0, mu0=2e-3, T0=1 / 1.4, Ts=0.27, Pr_lam=0.72)
    return Config(gas=gas, scheme=SchemeChoice("muscl2", "roe", 3, "minmod"), bc_params={}, topology=topology,
                  ghost=G, nan_check=False, precision=precision)


def _topo(bid, links):
    nb, bc = {}, {}
    for face, src_block, src_face, orient in links:
        nb[face] = (src_block, src_face, orient)
        bc[face] = BCType.CUT1TO1
    return BlockTopology(bid, nb, bc)


def _blocks(qs):
    return tuple(Block(q=dev(q), xyz=torch.zeros((3,) + q.shape[1:], dtype=torch.float64, device="cuda"))
                 for q in qs)


def test_mapped_halo_matches_numpy(cuda_device):
    rng = np.random.default_rng(11)
    shapes = [(8, 9, 10), (9, 10, 7), (6, 10, 8)]
    qs = [rng.standard_normal((5,) + s) for s in shapes]
    m = mapped_orientation
    # (target face, source block, source face, orient) per block, in dict order
    spec = [
        [(Face.IMAX, 1, Face.KMIN, m(reverse_a=True)),
         (Face.JMIN, 2, Face.IMAX, m(swap=True, reverse_b=True)),
         (Face.KMAX, 0, Face.KMIN, m(reverse_a=True, reverse_b=True)),
         (Face.KMIN, 0, Face.KMAX, 0)],
        [(Face.KMIN, 0, Face.IMAX, m(reverse_a=True)),
         (Face.IMIN, 1, Face.IMAX, 0),
         (Face.IMAX, 1, Face.IMIN, m())],
        [(Face.IMAX, 0, Face.JMIN, m(swap=True)),
         (Face.JMAX, 2, Face.JMIN, m(swap=False, reverse_a=True, reverse_b=True))],
    ]
    topos = tuple(_topo(b, s) for b, s in enumerate(spec))
    links = [(b, int(f), sb, int(sf), o) for b, s in enumerate(spec) for f, sb, sf, o in s]
    ref = mapped_halo(qs, links, G)
    got = halo_exchange(_blocks(qs), topos, G)
    for b in range(3):
        assert np.array_equal(host(got[b].q), ref[b]), f"block {b}"


def test_mapped_halo_rejects_mismatched_extents(cuda_device):
    rng = np.random.default_rng(12)
    qs = [rng.standard_normal((5, 8, 9, 10)), rng.standard_normal((5, 8, 9, 10))]
    topos = (_topo(0, [(Face.IMAX, 1, Face.IMIN, mapped_orientation(swap=True))]), _topo(1, []))
    with pytest.raises(ValueError):
        halo_exchange(_blocks(qs), topos, G)


# (perm, flip) of the second block's axes: new axis a is old axis perm[a],
# reversed where flip[a]; the interface axis (i) stays as it is
RELABELS = [((0, 2, 1), (False, False, False)),
            ((0, 1, 2), (False, False, True)),
            ((0, 2, 1), (False, True, False)),
            ((0, 2, 1), (False, True, True))]

_FACES = [(Face.IMIN, Face.IMAX), (Face.JMIN, Face.JMAX), (Face.KMIN, Face.KMAX)]


def _new_face(face, perm, flip):
    """The relabelled block's name for one of the old block's faces."""
    old_axis, old_max = int(face) // 2, int(face) % 2
    a = perm.index(old_axis)
    return _FACES[a][old_max ^ int(flip[a])]


def _box(perm, flip, seed=21):
    """Two blocks side by side along i in a periodic box (uniform anisotropic
    spacing, non-uniform seeded state), the second one relabelled by
    (perm, flip); returns (qs, metrics, topos)."""
    na, nb = (10, 12, 11), (9, 12, 11)
    hx, hy, hz = 0.3, 0.25, 0.2
    qa, _, _ = random_block(na, seed)
    qb, _, _ = random_block(nb, seed + 1)

    def metrics(shape):
        k = np.zeros((3, 3) + shape)
        k[0, 0], k[1, 1], k[2, 2] = 1 / hx, 1 / hy, 1 / hz
        return k, np.full(shape, hx * hy * hz)

    ka, va = metrics(na)
    kb, vb = metrics(nb)
    inv = [perm.index(a) for a in range(3)]
    identity = (perm, flip) == ((0, 1, 2), (False, False, False))
    # A's links to B: A's tangential axes (j, k) are B's axes inv[1], inv[2]
    a_from_b = 0 if identity else mapped_orientation(swap=inv[1] > inv[2], reverse_a=flip[inv[1]],
                                                     reverse_b=flip[inv[2]])
    # B's links to A: B's tangential axes (1, 2) are A's axes perm[1], perm[2]
    b_from_a = 0 if identity else mapped_orientation(swap=perm[1] > perm[2], reverse_a=flip[1], reverse_b=flip[2])
    topo_a = _topo(0, [(Face.IMIN, 1, _new_face(Face.IMAX, perm, flip), a_from_b),
                       (Face.IMAX, 1, _new_face(Face.IMIN, perm, flip), a_from_b),
                       (Face.JMIN, 0, Face.JMAX, 0), (Face.JMAX, 0, Face.JMIN, 0),
                       (Face.KMIN, 0, Face.KMAX, 0), (Face.KMAX, 0, Face.KMIN, 0)])
    # B's faces in the physical order of the unrelabelled block, so that the
    # last writer of every edge cell is the same physical link in both runs
    nf = lambda f: _new_face(f, perm, flip)  # noqa: E731
    topo_b = _topo(1, [(nf(Face.IMIN), 0, Face.IMAX, b_from_a), (nf(Face.IMAX), 0, Face.IMIN, b_from_a),
                       (nf(Face.JMIN), 1, nf(Face.JMAX), 0), (nf(Face.JMAX), 1, nf(Face.JMIN), 0),
                       (nf(Face.KMIN), 1, nf(Face.KMAX), 0), (nf(Face.KMAX), 1, nf(Face.KMIN), 0)])
    qs = [qa, relabel(qb, perm, flip)]
    mets = [(ka, va), (relabel_kxyz(kb, perm, flip), relabel(vb, perm, flip, lead=0))]
    return qs, mets, (topo_a, topo_b)


def _state(qs, mets):
    return State(blocks=_blocks(qs), metrics=tuple(Metrics(jac=dev(v), kxyz=dev(k), vol=dev(v)) for k, v in mets))


@pytest.mark.parametrize("perm,flip,precision", [r + ("f64",) for r in RELABELS] + [RELABELS[3] + ("f32",)])
def test_relabelled_block_steps_like_the_original(cuda_device, perm, flip, precision):
    qs0, mets0, topos0 = _box((0, 1, 2), (False, False, False))
    qs1, mets1, topos1 = _box(perm, flip)
    cfg0, cfg1 = _cfg(topos0, precision), _cfg(topos1, precision)
    dt = 0.5 * NP.cfl_dt(qs0, mets0, 1.4, 0.5, G)
    s0, s1 = _state(qs0, mets0), _state(qs1, mets1)
    for _ in range(4):
        s0, s1 = step(s0, cfg0, dt), step(s1, cfg1, dt)
    # FP64: the runs differ only in the order of the per-axis sums; FP32-flux:
    # by FP32 rounding of those sums (and of the mean-pressure offset)
    tol = 1e-12 if precision == "f64" else 1e-6
    assert rel_l2(host(s1.blocks[0].q), host(s0.blocks[0].q)) <= tol
    assert rel_l2(unrelabel(host(s1.blocks[1].q), perm, flip), host(s0.blocks[1].q)) <= tol
    assert rel_l2(host(s0.blocks[1].q), qs0[1]) > 1e-6  # the state did evolve


@pytest.mark.parametrize("perm,flip", RELABELS)
def test_relabelled_block_adjoint_like_the_original(cuda_device, perm, flip):
    qs0, mets0, topos0 = _box((0, 1, 2), (False, False, False), seed=31)
    qs1, mets1, topos1 = _box(perm, flip, seed=31)
    dt = 0.5 * NP.cfl_dt(qs0, mets0, 1.4, 0.5, G)
    rng = np.random.default_rng(32)
    lam0 = [rng.standard_normal(q.shape) for q in qs0]
    lam1 = [lam0[0], relabel(lam0[1], perm, flip)]
    m0 = tuple(Metrics(jac=dev(v), kxyz=dev(k), vol=dev(v)) for k, v in mets0)
    m1 = tuple(Metrics(jac=dev(v), kxyz=dev(k), vol=dev(v)) for k, v in mets1)
    g0 = adjoint.step_vjp([dev(q) for q in qs0], m0, _cfg(topos0), dt, [dev(l) for l in lam0])
    g1 = adjoint.step_vjp([dev(q) for q in qs1], m1, _cfg(topos1), dt, [dev(l) for l in lam1])
    assert rel_l2(host(g1[0]), host(g0[0])) <= 1e-12
    assert rel_l2(unrelabel(host(g1[1]), perm, flip), host(g0[1])) <= 1e-12


@pytest.mark.parametrize("kernel", ["persistent", "split_fill"])
def test_relabelled_box_persistent_matches_split(cuda_device, kernel):
    """The persistent step's halo items (and the fused ghost fill) with mapped
    orientations: bit-identical to the split kernels after 3 steps."""
    from famrdp_jax_b200.solver.step import StepPlan
    perm, flip = RELABELS[3]
    qs, mets, topos = _box(perm, flip)
    cfg = _cfg(topos, "f32")
    dt = 0.5 * NP.cfl_dt(qs, mets, 1.4, 0.5, G)
    res = {}
    for k in ("split", kernel):
        st = _state(qs, mets)
        plan = StepPlan(st, cfg)
        plan.set_kernel(k)
        a = [b.q.clone() for b in st.blocks]
        b = [torch.empty_like(x) for x in a]
        for _ in range(3):
            plan.run(a, b, dt)
            a, b = b, a
        assert plan.check() == 0
        res[k] = a
    for x, y in zip(res[kernel], res["split"]):
        assert torch.equal(x, y)

"""Mapped interface orientations on the CPU: the NumPy statement of the
mapping against the reference's copy where the two coincide, the
relabelling used by the GPU equivalence tests against the oracle's metrics,
and the topology marshalling of the orientation codes."""
import numpy as np
import pytest

from famrdp_jax_b200 import _topology
from famrdp_jax_b200.core.constants import (BCType, Face, ORIENT_MAPPED, ORIENT_REV_A, ORIENT_REV_B, ORIENT_SWAP,
                                            mapped_orientation, orientation_supported)
from famrdp_jax_b200.core.types import BlockTopology
from oracle.ref import NP
from orientation_util import mapped_copy, relabel, relabel_kxyz, unrelabel

G = 2


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("tgt_min", [True, False])
def test_mapped_identity_equals_reference_copy_on_opposite_faces(axis, tgt_min):
    # a MIN face fed from the partner's MAX face (and vice versa) is the
    # reference's aligned copy: the mapping must reproduce it exactly
    rng = np.random.default_rng(axis + 3 * tgt_min)
    shape = [7, 8, 9]
    tgt = rng.standard_normal([5] + shape)
    sshape = list(shape)
    sshape[axis] = 6
    src = rng.standard_normal([5] + sshape)
    tf = Face(2 * axis + (0 if tgt_min else 1))
    sf = Face(2 * axis + (1 if tgt_min else 0))
    ref = NP._copy_face(tgt.copy(), src, tf, sf, G)
    got = mapped_copy(tgt, src, tf, sf, mapped_orientation(), G)
    assert np.array_equal(np.asarray(ref), got)


def test_same_side_faces_pair_layers_by_distance():
    # IMIN fed from another block's IMIN (a mirrored connection): the ghost
    # layer next to the interface takes the first interior layer
    rng = np.random.default_rng(1)
    tgt, src = rng.standard_normal((5, 6, 4, 5)), rng.standard_normal((5, 7, 4, 5))
    got = mapped_copy(tgt, src, Face.IMIN, Face.IMIN, mapped_orientation(), G)
    assert np.array_equal(got[:, G - 1], src[:, G])
    assert np.array_equal(got[:, G - 2], src[:, G + 1])
    assert np.array_equal(got[:, G:], tgt[:, G:])


def test_swap_and_reversal_bits():
    rng = np.random.default_rng(2)
    tgt = rng.standard_normal((5, 6, 7, 7))
    src = rng.standard_normal((5, 6, 7, 7))
    plain = mapped_copy(tgt, src, Face.IMIN, Face.IMAX, mapped_orientation(), G)
    sw = mapped_copy(tgt, src, Face.IMIN, Face.IMAX, mapped_orientation(swap=True), G)
    ra = mapped_copy(tgt, src, Face.IMIN, Face.IMAX, mapped_orientation(reverse_a=True), G)
    rb = mapped_copy(tgt, src, Face.IMIN, Face.IMAX, mapped_orientation(reverse_b=True), G)
    gs = slice(0, G)
    assert np.array_equal(sw[:, gs], np.swapaxes(plain[:, gs], 2, 3))
    assert np.array_equal(ra[:, gs], plain[:, gs, ::-1, :])
    assert np.array_equal(rb[:, gs], plain[:, gs, :, ::-1])


def test_tangential_extent_mismatch_raises():
    tgt, src = np.zeros((5, 6, 7, 8)), np.zeros((5, 6, 7, 8))
    with pytest.raises(ValueError):
        mapped_copy(tgt, src, Face.IMIN, Face.IMAX, mapped_orientation(swap=True), G)


def test_orientation_codes():
    assert (ORIENT_MAPPED, ORIENT_SWAP, ORIENT_REV_A, ORIENT_REV_B) == (8, 1, 2, 4)
    assert sorted(mapped_orientation(s, a, b) for s in (0, 1) for a in (0, 1) for b in (0, 1)) == list(range(8, 16))
    assert orientation_supported(0)
    assert all(orientation_supported(o) for o in range(8, 16))
    assert not any(orientation_supported(o) for o in (1, 2, 7, 16, -1))


def test_topology_accepts_mapped_and_rejects_the_rest():
    for o in range(8, 16):
        t0 = BlockTopology(0, {Face.IMAX: (0, Face.IMIN, o)}, {Face.IMAX: BCType.CUT1TO1})
        assert _topology.links((t0,)) == [(0, int(Face.IMAX), 0, int(Face.IMIN), o)]
    for o in (1, 5, 16):
        t0 = BlockTopology(0, {Face.IMAX: (0, Face.IMIN, o)}, {Face.IMAX: BCType.CUT1TO1})
        with pytest.raises(NotImplementedError):
            _topology.links((t0,))


@pytest.mark.parametrize("perm,flip", [((0, 2, 1), (False, False, False)),
                                       ((0, 1, 2), (False, False, True)),
                                       ((0, 2, 1), (False, True, False))])
def test_relabelled_metrics_match_the_oracle(perm, flip):
    # the metrics of a relabelled block (rows permuted and negated) are what
    # compute_metrics gives on the relabelled coordinates (interior cells; the
    # roll wrap spoils the outer two layers of both)
    n = (10, 11, 12)
    i, j, k = np.meshgrid(*[np.arange(m, dtype=np.float64) for m in n], indexing="ij")
    x = 0.3 * i + 0.02 * np.sin(0.5 * j) + 0.01 * k
    y = 0.25 * j + 0.03 * np.cos(0.4 * i) + 0.02 * np.sin(0.3 * k)
    z = 0.2 * k + 0.015 * i * 0.1 + 0.01 * np.sin(0.6 * j)
    xyz = np.stack([x, y, z])
    _, kxyz, vol = NP.compute_metrics(xyz, ghost=G)
    _, kxyz2, vol2 = NP.compute_metrics(relabel(xyz, perm, flip), ghost=G)
    s = (slice(None), slice(None)) + (slice(2, -2),) * 3
    assert np.allclose(np.asarray(kxyz2)[s], relabel_kxyz(np.asarray(kxyz), perm, flip)[s], rtol=0, atol=1e-12)
    assert np.allclose(np.asarray(vol2)[2:-2, 2:-2, 2:-2],
                       relabel(np.asarray(vol), perm, flip, lead=0)[2:-2, 2:-2, 2:-2], rtol=1e-12, atol=0)
    q = np.random.default_rng(0).standard_normal((5,) + n)
    assert np.array_equal(unrelabel(relabel(q, perm, flip), perm, flip), q)

"""Grid and topology input (famrdp_jax mesh/io_grd.py, mesh/io_top.py,
mesh/build_state.py), after tests/mesh/test_io_grd.py, test_io_top.py and
test_build_state.py.  The fixtures under tests/golden are written by
tests/golden/make_mesh_fixtures.py; when the reference tree is present its own
fixtures are parsed too (set FAMRDP_JAX_REFERENCE to the root of a
famrdp_jax checkout)."""
import os
from pathlib import Path

import numpy as np
import pytest
import torch

from famrdp_jax_b200 import _topology
from famrdp_jax_b200.core.constants import BCType, Face
from famrdp_jax_b200.core.types import BlockTopology
from famrdp_jax_b200.mesh.build_state import build_initial_state
from famrdp_jax_b200.mesh.io_grd import read_grd, write_grd
from famrdp_jax_b200.mesh.io_top import _face, parse_topology

GOLD = Path(__file__).parent / "golden"
# the reference project's own fixtures, when a checkout is named by
# FAMRDP_JAX_REFERENCE (its root directory); skipped otherwise
_REF_ROOT = os.environ.get("FAMRDP_JAX_REFERENCE")
REF_FIX = Path(_REF_ROOT) / "tests" / "fixtures" if _REF_ROOT else Path("/nonexistent")


def test_read_grd_shapes_and_values():
    blocks = read_grd(GOLD / "mini.grd")
    assert [b.shape for b in blocks] == [(3, 4, 3, 2), (3, 3, 3, 2)]
    assert all(b.dtype == np.float64 for b in blocks)
    x = blocks[0][0]
    np.testing.assert_allclose(x[0], 0.0, atol=1e-14)
    np.testing.assert_allclose(x[-1], 1.0, atol=1e-14)
    np.testing.assert_allclose(blocks[0][1][:, 1, :], 0.5, atol=1e-14)  # y at j = 1 of 3 nodes


def test_grd_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    blocks = [rng.standard_normal((3, 5, 2, 3)), rng.standard_normal((3, 1, 4, 2))]
    write_grd(tmp_path / "r.grd", blocks)
    back = read_grd(tmp_path / "r.grd")
    for a, b in zip(blocks, back):
        np.testing.assert_array_equal(a, b)


def test_read_grd_rejects_truncated(tmp_path):
    data = (GOLD / "mini.grd").read_bytes()
    (tmp_path / "t.grd").write_bytes(data[:-8])
    with pytest.raises(ValueError):
        read_grd(tmp_path / "t.grd")


def test_parse_topology():
    tops = parse_topology(GOLD / "mini.inp")
    assert [t.block_id for t in tops] == [0, 1]
    for t in tops:
        assert len(t.bc_type) == 6 and all(isinstance(v, BCType) for v in t.bc_type.values())
        assert t.bc_type[Face.KMIN] == BCType.WALL and t.bc_type[Face.KMAX] == BCType.WALL
        assert t.bc_type[Face.IMIN] == BCType.SYMMETRY and t.bc_type[Face.IMAX] == BCType.FARFIELD
        for f in (Face.IMIN, Face.IMAX, Face.KMIN, Face.KMAX):
            assert t.neighbors[f] is None
    assert tops[0].neighbors[Face.JMAX] == (1, Face.JMIN, 0)
    assert tops[0].neighbors[Face.JMIN] == (1, Face.JMAX, 0)
    assert tops[1].neighbors[Face.JMAX] == (0, Face.JMIN, 0)


def test_face_rules_follow_the_reference():
    dims = (5, 5, 3)
    assert _face([1, 1, 1, 5, 1, 3], dims) == Face.IMIN
    assert _face([5, 5, 1, 5, 1, 3], dims) == Face.IMAX
    assert _face([1, 5, -1, -1, 1, 3], dims) == Face.JMIN  # absolute value 1
    assert _face([1, 5, 5, 5, -3, -1], dims) == Face.JMAX
    assert _face([1, 5, 1, 5, 0, 0], dims) == Face.KMIN
    assert _face([1, 5, 1, 5, -3, -3], dims) == Face.KMAX
    assert _face([1, 2, 1, 5, 1, 3], dims) == Face.IMIN  # no degenerate axis: smallest extent


def test_misaligned_interface_keeps_orientation_marker(tmp_path):
    txt = (GOLD / "mini.inp").read_text().splitlines()
    # reverse the i range of block A's first interface's neighbour line
    for n, ln in enumerate(txt):
        if ln.split()[:7] == ["1", "5", "1", "1", "-3", "-1", "2"]:
            txt[n] = "      5       1       1       1      -3      -1       2"
            break
    (tmp_path / "m.inp").write_text("\n".join(txt) + "\n")
    tops = parse_topology(tmp_path / "m.inp")
    assert tops[0].neighbors[Face.JMAX] == (1, Face.JMIN, 1)
    with pytest.raises(NotImplementedError):
        _topology.links(tuple(tops))


def test_build_initial_state():
    st, tops = build_initial_state(GOLD / "mini.grd", GOLD / "mini.inp", ghost=2,
                                   q_init_fn=lambda shape: np.zeros(shape))
    assert len(st.blocks) == 2 and len(tops) == 2
    assert st.blocks[0].xyz.shape == (3, 8, 7, 6) and st.blocks[0].q.shape == (5, 8, 7, 6)
    assert st.blocks[0].q.dtype == torch.float64 and st.blocks[0].xyz.dtype == torch.float64
    x = st.blocks[0].xyz.numpy()
    np.testing.assert_array_equal(x[:, 0], x[:, 2])  # edge replication
    assert torch.all(st.metrics[0].kxyz == 0) and torch.all(st.metrics[0].vol == 1)


@pytest.mark.skipif(not REF_FIX.exists(), reason="reference fixtures not present")
def test_reference_fixtures():
    blocks = read_grd(REF_FIX / "mini.grd")
    assert [b.shape for b in blocks] == [(3, 4, 3, 2), (3, 3, 3, 2)]
    np.testing.assert_allclose(blocks[0][0, 0], 0.0, atol=1e-14)
    np.testing.assert_allclose(blocks[0][0, -1], 1.0, atol=1e-14)
    tops = parse_topology(REF_FIX / "mini.inp")
    assert len(tops) == 2
    for t in tops:
        assert len(t.bc_type) == 6
        cut = [f for f, b in t.bc_type.items() if b == BCType.CUT1TO1]
        assert cut
        for f in cut:
            nb, nf, orient = t.neighbors[f]
            assert 0 <= nb < 2 and isinstance(nf, Face) and orient == 0
        for f, b in t.bc_type.items():
            if b != BCType.CUT1TO1:
                assert t.neighbors[f] is None

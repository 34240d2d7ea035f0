"""Host-side marshalling of topology and boundary conditions: table order
carries the reference's overwrite semantics."""
import pytest

from famrdp_jax_b200 import _topology, cases
from famrdp_jax_b200.core.constants import BCType, Face
from famrdp_jax_b200.core.types import BlockTopology, Config, GasModel, SchemeChoice


def test_links_follow_block_then_dict_order():
    t0 = BlockTopology(0, {Face.JMAX: (7, Face.JMIN, 0), Face.IMIN: (0, Face.IMAX, 0), Face.KMIN: None},
                       {Face.JMAX: BCType.CUT1TO1, Face.IMIN: BCType.CUT1TO1})
    t1 = BlockTopology(7, {Face.JMIN: (0, Face.JMAX, 0)}, {Face.JMIN: BCType.CUT1TO1})
    ls = _topology.links((t0, t1))
    assert ls == [(0, int(Face.JMAX), 1, int(Face.JMIN), 0), (0, int(Face.IMIN), 0, int(Face.IMAX), 0),
                  (1, int(Face.JMIN), 0, int(Face.JMAX), 0)]


def test_links_skip_non_cut_faces():
    t0 = BlockTopology(0, {Face.IMAX: (0, Face.IMIN, 0)}, {Face.IMAX: BCType.FARFIELD})
    assert _topology.links((t0,)) == []


def test_orient_raises_not_implemented():
    t0 = BlockTopology(0, {Face.IMAX: (0, Face.IMIN, 1)}, {Face.IMAX: BCType.CUT1TO1})
    with pytest.raises(NotImplementedError):
        _topology.links((t0,))


def test_bcs_in_face_order_and_defaults():
    t0 = BlockTopology(0, {}, {Face.KMAX: BCType.FARFIELD, Face.IMIN: BCType.WALL, Face.JMIN: BCType.SYMMETRY,
                               Face.JMAX: BCType.CUT1TO1, Face.IMAX: BCType.OUTFLOW})
    cfg = Config(gas=GasModel(), scheme=SchemeChoice("muscl2", "roe", 3, "minmod"),
                 bc_params={Face.IMIN: {"wall_type": "isothermal", "T_wall": 250.0}}, topology=(t0,))
    bs = _topology.bcs((t0,), cfg)
    assert [b[1] for b in bs] == [int(Face.IMIN), int(Face.JMIN), int(Face.KMAX)]
    assert bs[0][2] == int(BCType.WALL) and bs[0][3] == 1 and bs[0][4] == 250.0
    assert bs[2][5] == (1.0, 0.0, 0.0, 0.0, 2.5)  # dispatch.py:27 default q_inf


def test_tree24_interfaces_have_matching_slabs():
    c = cases.tree24(seed=0)
    assert len(c.qs) == 24
    shapes = [q.shape[1:] for q in c.qs]
    for (t, tf, s, sf, o) in _topology.links(c.cfg.topology):
        ax_t, ax_s = tf // 2, sf // 2
        assert ax_t == ax_s
        others = [a for a in range(3) if a != ax_t]
        assert all(shapes[t][a] == shapes[s][a] for a in others)


def test_wavy4_topology_is_a_torus():
    from oracle import NP
    c = cases.wavy4(n=8, metrics_fn=lambda xyz: NP.compute_metrics(xyz, ghost=2))
    ls = _topology.links(c.cfg.topology)
    assert len(ls) == 24
    assert all(l[4] == 0 for l in ls)
    assert c.interior_cells == 4 * 8 ** 3

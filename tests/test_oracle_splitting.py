"""Body bonds, brick removal and body splitting (finalize_brick, src/lib.rs:668-696; remove_brick, src/lib.rs:705-718;
rebuild_body, src/lib.rs:930-1002) in the CPU oracle, against answers that follow from the reference's rules:

  * two face-adjacent bricks of one body are bonded with the weaker brick's capacity on that axis (CAPH across, CAPV
    up), except across an infill gap (glass against another material sideways, or glass below);
  * removing the middle brick of a row splits the body in two; the first piece (seeded at the body's first brick)
    keeps the body, the other takes the next body; each piece is set up about the parent's pose, so at rest with the
    identity rotation the pieces' centres are their bricks' cell centres, and a spinning parent's pieces move with
    v = v_parent + w x (centre - parent centre), w = w_parent;
  * without room for new bodies the body stays whole; a body with no brick left dies.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S

CAPV = [0.0, 140000.0, 50000.0, 150000.0, 1500.0, 9000.0]
CAPH = [0.0, 12000.0, 12000.0, 90000.0, 400.0, 5000.0]


def body_scene(cells_per_body, mats_per_body, poses):
    first = [0]
    xyz, mat = [], []
    for cells, mats in zip(cells_per_body, mats_per_body):
        for c, m in zip(cells, mats):
            xyz.append([S.ORIGIN[0] + c[0], S.ORIGIN[1] + c[1], S.ORIGIN[2] + c[2]])
            mat.append(m)
        first.append(len(xyz))
    return S.Scene(body_first=np.array(first, np.uint32), body_brick_xyz=np.array(xyz, np.int32),
                   body_brick_mat=np.array(mat, np.uint8),
                   body_pose=np.asarray(poses, np.float32).reshape(-1, 13)).contiguous()


def pose(p, v=(0, 0, 0), w=(0, 0, 0)):
    return [*p, 0, 0, 0, 1, *v, *w]


def lat(c):
    return np.array([c[0] * 0.5 + 0.25, c[1] * 0.5 + 0.25, c[2] * 0.5 + 0.25])


def test_body_bonds_follow_finalize_rule(oracle):
    C, G = S.CONC, S.GLASS
    sc = body_scene([[(0, 10, 0), (1, 10, 0)], [(0, 20, 0), (1, 20, 0)], [(5, 20, 0), (5, 21, 0)], [(8, 20, 0), (8, 21, 0)]],
                    [[C, S.STEEL], [C, G], [G, C], [C, G]], [pose((0, 0, 0))] * 4)
    ow = oracle.OracleWorld(sc)
    b, nb = ow.body_bonds()
    assert b[0, 0] == min(CAPH[C], CAPH[S.STEEL]) and nb[0, 0] == 1 and nb[1, 1] == 0
    assert b[2, 0] == 0.0                      # concrete | glass sideways: an infill gap
    assert b[4, 1] == 0.0                      # glass below concrete: a gap
    assert b[6, 1] == min(CAPV[C], CAPV[G])    # concrete below glass: bonded
    assert (b[:, 3] == 0).all()                # no foundation bond on a body


def test_removing_the_middle_brick_splits_a_row(oracle):
    sc = body_scene([[(0, 20, 0), (1, 20, 0), (2, 20, 0)]], [[S.CONC] * 3], [pose((0, 0, 0))])
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(4, 16)
    ow.remove_bricks(body_bricks=[1])
    assert ow.rebuild_bodies() == (1, 1, 1, 0, 0)
    st, _, fl = ow.bodies()
    assert st.shape[0] == 2 and (fl & 1).all()
    np.testing.assert_allclose(st[0, :3], lat((0, 20, 0)), atol=2e-6)
    np.testing.assert_allclose(st[1, :3], lat((2, 20, 0)), atol=2e-6)
    b12, _ = ow.setup()
    assert b12[0, 0] == 300.0 and b12[1, 0] == 300.0
    # the body's first brick stays at the front of its range; the other piece took the next brick id
    b, nb = ow.body_bonds()
    assert (nb[0] == 0xFFFFFFFF).all() and (nb[3] == 0xFFFFFFFF).all()


def test_pieces_inherit_the_parent_motion(oracle):
    v, w = np.array([1.0, -2.0, 0.5]), np.array([0.0, 3.0, 0.0])
    sc = body_scene([[(0, 20, 0), (1, 20, 0), (2, 20, 0), (3, 20, 0)]], [[S.CONC] * 4], [pose((0, 0, 0), v, w)])
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(4, 16)
    st0, _, _ = ow.bodies()
    ow.remove_bricks(body_bricks=[2])
    ow.rebuild_bodies()
    st, _, _ = ow.bodies()
    for k in range(2):
        off = st[k, :3].astype(np.float64) - st0[0, :3]
        np.testing.assert_allclose(st[k, 7:10], st0[0, 7:10] + np.cross(w, off), atol=1e-5)
        np.testing.assert_allclose(st[k, 10:13], w, atol=0)


def test_no_room_keeps_the_body_whole_and_empty_bodies_die(oracle):
    sc = body_scene([[(0, 20, 0), (1, 20, 0), (2, 20, 0)], [(9, 20, 0)]], [[S.CONC] * 3, [S.CONC]],
                    [pose((0, 0, 0))] * 2)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(0, 0)
    ow.remove_bricks(body_bricks=[1, 3])
    assert ow.rebuild_bodies() == (2, 0, 2, 1, 0)
    st, _, fl = ow.bodies()
    assert fl[0] & 1 and not fl[1] & 1
    np.testing.assert_allclose(st[0, :3], (lat((0, 20, 0)) + lat((2, 20, 0))) / 2, atol=2e-6)


def test_detached_piece_keeps_its_bonds_and_splits_later(oracle):
    """A floating 3-brick row of a structure detaches with its bonds; removing its middle brick then splits it."""
    col = [(0, y, 0) for y in range(4)]
    row = [(4, 6, 0), (5, 6, 0), (6, 6, 0)]
    xyz = np.array([[S.ORIGIN[0] + x, y, S.ORIGIN[2] + z] for x, y, z in col + row], np.int32)
    n = len(xyz)
    sc = S.Scene(xyz, np.full(n, S.CONC, np.uint8), np.zeros(n, np.int32), np.zeros(n, np.uint8)).contiguous()
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(4, 16)
    (pieces, detached, _), _, _ = ow.connect([0])
    assert (pieces, detached) == (1, 3)
    b, nb = ow.body_bonds()
    assert b[0, 0] == CAPH[S.CONC] and nb[0, 0] == 1 and nb[1, 0] == 2
    ow.remove_bricks(body_bricks=[1])
    assert ow.rebuild_bodies()[:2] == (1, 1)
    assert ow.counts()["n_bodies"] == 2

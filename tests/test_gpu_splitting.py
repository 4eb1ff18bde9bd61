"""Brick removal and body splitting on the GPU (sf_world_remove_bricks / sf_world_rebuild_bodies: remove_brick and
rebuild_body, src/lib.rs:705-718, 930-1002) against the oracle's restatement, bit for bit: body bricks' bonds, which
bricks leave, the pieces and their brick order, their set-up about the parent's pose and cached rotation, the
lone-brick rule, and the rigid step of the world afterwards.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S
from test_gpu_connectivity import DT, IT, compare_world, hand_built, join

pytestmark = pytest.mark.gpu


def compare_bonds(w, ow, scene=0):
    r = w.scene_ranges(scene)
    k0, nk = r[4], r[7]
    b, nb = w.body_bonds()
    ob, onb = ow.body_bonds()
    np.testing.assert_array_equal(b[k0:k0 + nk], ob)
    g = nb[k0:k0 + nk].astype(np.int64)
    g[g != 0xFFFFFFFF] -= k0
    np.testing.assert_array_equal(g.astype(np.uint32), onb)


def test_split_compound_debris_against_oracle(sf, oracle):
    """300 compound bodies (1-256 bricks) fall for 30 steps; a brick of every third multi-brick body is removed
    (some bodies split in two or more, some only lose the brick); after the rebuild and 60 more steps the world is
    bit-exact against the oracle."""
    sc = S.debris_scene(300, seed=11, kmax=64)
    w = sf.World(sc, iterations=IT, detach_bodies=600, detach_bricks=4000)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(600, 4000)
    compare_bonds(w, ow)
    for _ in range(30):
        w.step(DT)
        ow.step(DT, iterations=IT)
    first = sc.body_first.astype(np.int64)
    picks = []
    for b in range(0, sc.n_bodies, 3):
        n = first[b + 1] - first[b]
        if n >= 3:
            picks.append(first[b] + n // 2)
    assert len(picks) > 20
    w.remove_bricks(body_bricks=picks)
    ow.remove_bricks(body_bricks=picks)
    rep = w.rebuild_bodies()
    orep = ow.rebuild_bodies()
    assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == orep
    assert rep.pieces > 0
    compare_world(w, ow)
    compare_bonds(w, ow)
    for k in range(60):
        w.step(DT)
        ow.step(DT, iterations=IT)
    compare_world(w, ow)


def test_lone_bricks_turn_to_debris_when_many_bodies_are_awake(sf, oracle):
    """1,700 single bricks in the air keep more than 1,500 bodies awake; two rows of bricks then lose every second
    brick, leaving lone-brick pieces, of which the rule (drawn from h01 of the rebuild count and brick) removes about
    (awake - 1500) / 2000 of the non-steel ones. GPU and oracle agree on every draw."""
    bf, bxyz, bmat, pose = S.loose_debris(1700, seed=5, box_lo=(-30.0, 20.0, -30.0), box_hi=(30.0, 60.0, 30.0))
    rows = []
    for k in range(2):
        cells = [(x, 40 + 2 * k, 40) for x in range(21)]
        rows.append(cells)
    xyz = [bxyz]
    first = list(bf)
    mats = [bmat]
    poses = [pose]
    for cells in rows:
        xyz.append(np.array([[S.ORIGIN[0] + c[0], c[1], S.ORIGIN[2] + c[2]] for c in cells], np.int32))
        mats.append(np.full(len(cells), S.CONC, np.uint8))
        first.append(first[-1] + len(cells))
        p = np.zeros((1, 13), np.float32)
        p[0, 6] = 1.0
        poses.append(p)
    sc = S.Scene(body_first=np.array(first, np.uint32), body_brick_xyz=np.concatenate(xyz),
                 body_brick_mat=np.concatenate(mats), body_pose=np.concatenate(poses)).contiguous()
    w = sf.World(sc, iterations=IT, detach_bodies=64, detach_bricks=64)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(64, 64)
    w.step(DT)
    ow.step(DT, iterations=IT)
    base = int(bf[-1])
    picks = [base + 21 * k + x for k in range(2) for x in range(1, 21, 2)]
    w.remove_bricks(body_bricks=picks)
    ow.remove_bricks(body_bricks=picks)
    rep = w.rebuild_bodies()
    orep = ow.rebuild_bodies()
    assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == orep
    assert rep.lone > 0 and rep.pieces > 0
    compare_world(w, ow)
    for _ in range(20):
        w.step(DT)
        ow.step(DT, iterations=IT)
    compare_world(w, ow)


def test_detached_piece_splits_after_removal(sf, oracle):
    """The hand-built structure's floating L detaches with its bonds (the body-brick bonds equal the oracle's); a
    static brick removed from the column's middle cuts the beam and the upper column loose at the next walk; a brick
    removed from the L splits it; all of it then falls for 60 steps, bit-exact."""
    sc = join(*hand_built())
    w = sf.World(sc, iterations=IT, detach_bodies=8, detach_bricks=64)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(8, 64)
    w.structure_connect([0])
    ow.connect([0])
    compare_bonds(w, ow)
    w.remove_bricks(statics=[4])
    ow.remove_bricks(statics=[4])
    rep, now, top = w.connectivity()
    (op, od, _), onow, otop = ow.connectivity()
    assert (rep.pieces, rep.detached) == (op, od) and rep.pieces == 1 and now[0] == onow[0] == 4
    compare_bonds(w, ow)
    w.remove_bricks(body_bricks=[1])          # the L's middle brick (list order: x=10, x=11, (10,6), x=12)
    ow.remove_bricks(body_bricks=[1])
    rep = w.rebuild_bodies()
    assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == ow.rebuild_bodies()
    compare_world(w, ow)
    compare_bonds(w, ow)
    for _ in range(60):
        w.step(DT)
        ow.step(DT, iterations=IT)
    compare_world(w, ow)

"""Connectivity and detachment on the GPU (sf_structure_connect / sf_world_connectivity, conn_struct and connectivity,
src/lib.rs:1085-1141) against the oracle's restatement, bit for bit: which static bricks leave, the new bodies' set-up
(mass, inertia, radius, brick offsets, pose), the woken neighbours, the pending flags, st_now / st_top, and the rigid
step of the world afterwards.

The GPU labels the structure's bricks by union-find over intact bonds and walks only the unsupported pieces in the
reference's breadth-first order; the oracle walks every brick as conn_struct does. New bodies take the scene's next
spare body and bricks on both sides.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
IT = 8


def cells(cs, mat=S.CONC, sid=0, dx=0):
    xyz = np.array([[S.ORIGIN[0] + x + dx, y, S.ORIGIN[2] + z] for x, y, z in cs], np.int32)
    n = len(cs)
    return xyz, np.full(n, mat, np.uint8), np.full(n, sid, np.int32), np.zeros(n, np.uint8)


def join(*parts, bodies=None):
    xyz, mat, sid, inf = (np.concatenate([p[k] for p in parts]) for k in range(4))
    sc = S.Scene(xyz, mat, sid, inf)
    if bodies is not None:
        sc.body_first, sc.body_brick_xyz, sc.body_brick_mat, sc.body_pose = bodies
    return sc.contiguous()


def hand_built(sid=0, dx=0, mat=S.CONC):
    """A grounded column with a beam, a floating L (given out of brick order), a floating 2x2 block of another
    material, and a glass pane hanging from nothing."""
    column = cells([(0, y, 0) for y in range(8)] + [(1, 7, 0), (2, 7, 0)], mat, sid, dx)
    l_piece = cells([(10, 5, 0), (12, 5, 0), (11, 5, 0), (10, 6, 0)], mat, sid, dx)
    block = cells([(3, 9, 2), (4, 9, 2), (3, 9, 3), (4, 9, 3)], S.WOOD, sid, dx)
    pane = cells([(6, 3, 4), (6, 4, 4)], S.GLASS, sid, dx)
    return [column, l_piece, block, pane]


def compare_world(w, ow, scene=0):
    r = w.scene_ranges(scene)
    b0, nb_used, k0, nk_used = r[2], r[6], r[4], r[7]
    st, sl, fl = w.bodies()
    ost, osl, ofl = ow.bodies()
    assert nb_used == ost.shape[0]
    np.testing.assert_array_equal(st[b0:b0 + nb_used], ost)
    np.testing.assert_array_equal(sl[b0:b0 + nb_used], osl)
    np.testing.assert_array_equal(fl[b0:b0 + nb_used], ofl)
    assert not (fl[b0 + nb_used:b0 + r[3]] & 1).any()      # the spare bodies stay dead
    b12, l3 = w.body_setup()
    ob12, ol3 = ow.setup()
    np.testing.assert_array_equal(b12[b0:b0 + nb_used], ob12)
    np.testing.assert_array_equal(l3[k0:k0 + nk_used], ol3)
    np.testing.assert_array_equal(w.brick_positions()[k0:k0 + nk_used], ow.brick_positions())
    s0, n_s = r[0], r[1]
    np.testing.assert_array_equal(w.phi64()[s0:s0 + n_s], ow.phi64())
    b, _, _ = w.bonds()
    ob, _ = ow.bonds()
    np.testing.assert_array_equal(b[s0:s0 + n_s], ob)


def test_connect_pieces_against_oracle(sf, oracle):
    """Three unsupported pieces (an L given out of order, a timber block, a glass pane) and a grounded column: the
    GPU's pieces, their brick order and set-up, st_now / st_top and the removed static bricks equal the oracle's;
    then 90 steps of the world (the pieces fall past and onto the column and the ground) stay bit-exact."""
    sc = join(*hand_built())
    w = sf.World(sc, iterations=IT, detach_bodies=8, detach_bricks=64)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(8, 64)
    rep, now, top = w.structure_connect([0])
    (op, od, opend), onow, otop = ow.connect([0])
    assert (rep.pieces, rep.detached, rep.retry) == (op, od, opend) == (3, 10, 0)
    assert rep.listed == 10
    assert now[0] == onow[0] == 10 and top[0] == otop[0] == 8
    compare_world(w, ow)
    for k in range(90):
        w.step(DT)
        ow.step(DT, iterations=IT)
        if k % 10 == 9:
            compare_world(w, ow)


def test_pieces_wait_for_room_and_wake_sleepers(sf, oracle):
    """Room for one new body: the piece seeded first detaches and the structure stays pending; sf_world_connectivity
    walks it again (pending from the last call) and, with the spare body used, leaves it pending once more. A
    sleeping body beside the new piece wakes (wake_near); one far away sleeps on."""
    bf = np.array([0, 1, 2], np.uint32)
    bxyz = np.array([[S.ORIGIN[0] + 12, 0, S.ORIGIN[2]], [S.ORIGIN[0] + 60, 0, S.ORIGIN[2]]], np.int32)
    bmat = np.array([S.CONC, S.CONC], np.uint8)
    pose = np.zeros((2, 13), np.float32)
    pose[:, 6] = 1.0
    sc = join(*hand_built(), bodies=(bf, bxyz, bmat, pose))
    w = sf.World(sc, iterations=IT, detach_bodies=1, detach_bricks=64)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(1, 64)
    # let the two resting bodies fall asleep first (the rest timer runs out after 0.45 s)
    for _ in range(40):
        w.step(DT)
        ow.step(DT, iterations=IT)
    _, _, fl = w.bodies()
    assert (fl[:2] & 2).all()
    rep, now, top = w.structure_connect([0])
    (op, od, opend), onow, otop = ow.connect([0])
    assert (rep.pieces, rep.detached, rep.retry) == (op, od, opend) == (1, 4, 1)
    assert now[0] == onow[0] and top[0] == otop[0]
    compare_world(w, ow)
    _, _, fl = w.bodies()
    assert not fl[0] & 2 and fl[1] & 2          # the near sleeper woke, the far one did not
    rep, _, _ = w.connectivity()
    (op, od, opend), _, _ = ow.connectivity()
    assert (rep.structures, rep.pieces, rep.retry) == (1, 0, 1) and (op, opend) == (0, 1)
    for _ in range(30):
        w.step(DT)
        ow.step(DT, iterations=IT)
    compare_world(w, ow)


def test_connect_per_scene(sf, oracle):
    """Two scenes, each with its own structure and spare capacity: each scene's pieces take that scene's spare
    bodies and bricks, and each scene matches its own oracle."""
    sc0 = join(*hand_built(sid=0))
    sc1 = join(*hand_built(sid=1, mat=S.MASON))
    w = sf.World([sc0, sc1], iterations=IT, detach_bodies=4, detach_bricks=32)
    ows = []
    for k, sc in enumerate([sc0, sc1]):
        ow = oracle.OracleWorld(sc)
        ow.set_capacity(4, 32)
        ows.append(ow)
    rep, now, top = w.structure_connect([1, 0])
    assert rep.pieces == 6 and rep.detached == 20
    ows[0].connect([0])
    ows[1].connect([1])
    for _ in range(30):
        w.step(DT)
        for ow in ows:
            ow.step(DT, iterations=IT)
    for k in range(2):
        compare_world(w, ows[k], scene=k)


def test_collapse_frames_against_oracle(sf, oracle):
    """The 5-storey frame with two ground columns removed, run frame by frame in the reference's order (step's
    substeps, connectivity, the resting loads and the load-path frame, connectivity again; src/lib.rs:3650-3659):
    joints fail once the structure's joints are live, the pieces they cut loose become bodies and land on what is
    left. Every frame's reports match; every 20 frames, and at the end, the whole world state is bit-exact."""
    fr, rm = S.frame5_structure()
    sc = fr.without_static(rm)
    ids = sc.structure_ids()
    w = sf.World(sc, iterations=IT, detach_bodies=64, detach_bricks=20000)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(64, 20000)
    for s in ids:
        w.structure_warm(s)
        ow.structure_warm(s)
    pieces = 0
    for f in range(1, 241):
        w.step(DT)
        ow.step(DT, iterations=IT)
        rep1, _, _ = w.connectivity()
        (op1, od1, _), _, _ = ow.connectivity()
        w.structure_loads(ids)
        ow.structure_loads(ids)
        fr_ = w.structure_frame(f, ids, dt=DT)
        osw, ows, olive, oj, oover, ofail, ocrush, omr = ow.structure_frame(f, DT, ids)
        assert (fr_.sweeps, fr_.warm_sweeps, fr_.live, fr_.joints, fr_.failed, fr_.crushed) == \
            (osw, ows, olive, oj, ofail, ocrush), f
        rep2, now, top = w.connectivity()
        (op2, od2, _), onow, otop = ow.connectivity()
        assert (rep1.pieces, rep1.detached, rep2.pieces, rep2.detached) == (op1, od1, op2, od2), f
        pieces += rep1.pieces + rep2.pieces
        if f % 20 == 0 or f == 240:
            compare_world(w, ow)
    assert pieces >= 2


def test_tower_footings_fail_and_the_tower_detaches(sf, oracle):
    """The 16-storey tower (47,760 bricks) with eight ground columns removed, frame by frame through the load-path
    schedule and connectivity only (no rigid steps): once its joints are live, footings and joints fail, pieces break
    off, and when the last footings go the whole tower becomes one 46,818-brick body. The GPU labels all 47,760 bricks
    each walk and reads back only the pieces; every frame's reports and the final bodies' set-up match the oracle."""
    tw, rm = S.tower16_structure()
    sc = tw.without_static(rm)
    ids = sc.structure_ids()
    w = sf.World(sc, iterations=IT, detach_bodies=256, detach_bricks=48000)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(256, 48000)
    for s in ids:
        w.structure_warm(s)
        ow.structure_warm(s)
    pieces = detached = 0
    for f in range(1, 261):
        fr_ = w.structure_frame(f, ids, dt=DT)
        osw, ows, olive, oj, oover, ofail, ocrush, omr = ow.structure_frame(f, DT, ids)
        assert (fr_.sweeps, fr_.warm_sweeps, fr_.joints, fr_.failed, fr_.crushed) == (osw, ows, oj, ofail, ocrush), f
        rep, now, top = w.connectivity()
        (op, od, _), onow, otop = ow.connectivity()
        assert (rep.pieces, rep.detached) == (op, od), f
        if rep.structures:
            assert now[0] == onow[0] and top[0] == otop[0], f
        pieces += rep.pieces
        detached += rep.detached
    assert pieces > 10 and detached > 45000
    compare_world(w, ow)

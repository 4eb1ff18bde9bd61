"""Connectivity and detachment (conn_struct, src/lib.rs:1085-1134; connectivity, src/lib.rs:1137-1141) in the CPU
oracle, pinned by answers that follow from the reference's rules on hand-built structures:

  * a piece is a set of static bricks of one structure that no intact bond path joins to a footing (a bottom-row
    brick with an intact foundation bond); each piece becomes one body, pieces seeded in brick order;
  * a body's bricks are listed in breadth-first order from the seed, neighbours in direction order +x, -x, +y, -y,
    +z, -z (DIRS, src/lib.rs:196), so a row of bricks given out of order is listed along the row;
  * the body is set up at rest, identity rotation, its centre the mass-weighted mean of the bricks' lattice centres
    (setup_body, src/lib.rs:844-891), and the detached static bricks leave the static set;
  * a piece that finds no room stays static and its structure stays pending (src/lib.rs:1111-1125);
  * a joint pass that fails a joint leaves its structure pending (src/lib.rs:1202, 1223).
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S

MASS = [0.0, 300.0, 230.0, 250.0, 60.0, 70.0, 2000.0, 8.0, 44.0]


def cells_scene(cells, mat=S.CONC, sid=0):
    xyz = np.array([[S.ORIGIN[0] + x, y, S.ORIGIN[2] + z] for x, y, z in cells], np.int32)
    n = len(cells)
    return S.Scene(xyz, np.full(n, mat, np.uint8), np.full(n, sid, np.int32), np.zeros(n, np.uint8)).contiguous()


def lat(x, y, z):
    return np.array([x * 0.5 + 0.25, y * 0.5 + 0.25, z * 0.5 + 0.25])


COLUMN = [(0, y, 0) for y in range(6)]


def test_floating_block_becomes_one_body(oracle):
    """A grounded column and a 2x1x2 block floating beside it: one piece of 4 bricks; its mass 4 x 300, its centre
    the mean of the four cell centres, at rest, identity rotation; the column stays (6 bricks, 6 cells high)."""
    block = [(3, 4, 0), (4, 4, 0), (3, 4, 1), (4, 4, 1)]
    sc = cells_scene(COLUMN + block)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(4, 64)
    (pieces, detached, pending), now, top = ow.connect([0])
    assert (pieces, detached, pending) == (1, 4, 0)
    assert now[0] == 6 and top[0] == 6
    st, sl, fl = ow.bodies()
    assert st.shape[0] == 1 and fl[0] & 1 and not fl[0] & 2
    centre = np.mean([lat(*c) for c in block], axis=0)
    np.testing.assert_allclose(st[0, :3], centre, rtol=0, atol=1e-6)       # f32 sums of 4 equal masses: exact to 1 ulp
    np.testing.assert_array_equal(st[0, 3:7], [0, 0, 0, 1])
    np.testing.assert_array_equal(st[0, 7:], np.zeros(6))
    b12, _ = ow.setup()
    assert b12[0, 0] == 4 * MASS[S.CONC]
    # the static bricks of the block are gone: their potentials read 0 and a second walk finds nothing
    (p2, d2, _), _, _ = ow.connect([0])
    assert (p2, d2) == (0, 0)


def test_piece_lists_bricks_breadth_first(oracle):
    """A floating row given out of order (x = 0, 2, 1 at y = 5): seeded at the first given brick, the walk goes +x
    first, so the body lists x = 0, 1, 2. An L adds a brick above x = 0, reached from the seed after +x (+y comes
    after +x and -x in direction order) but before x = 2 (breadth first)."""
    row = [(10, 5, 0), (12, 5, 0), (11, 5, 0), (10, 6, 0)]
    sc = cells_scene(COLUMN + row)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(1, 16)
    (pieces, detached, _), _, _ = ow.connect([0])
    assert (pieces, detached) == (1, 4)
    # brick world positions of the new body (at rest, identity rotation: the lattice centres) in list order
    wp = ow.brick_positions()
    expect = [lat(10, 5, 0), lat(11, 5, 0), lat(10, 6, 0), lat(12, 5, 0)]
    np.testing.assert_allclose(wp[-4:], expect, rtol=0, atol=1e-4)


def test_pieces_seed_in_brick_order_and_wait_for_room(oracle):
    """Two floating pieces with room for one body: the piece holding the lower brick index detaches, the other stays
    static and its structure pending; with room added, connectivity() detaches it."""
    a = [(20, 3, 0), (21, 3, 0)]           # indices 6, 7
    b = [(30, 3, 0), (30, 4, 0), (30, 5, 0)]   # indices 8..10
    sc = cells_scene(COLUMN + a + b)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(1, 64)
    (pieces, detached, pending), now, _ = ow.connect([0])
    assert (pieces, detached, pending) == (1, 2, 1)
    assert now[0] == 6 + 3
    assert ow.pending()[0] == 1
    ow.set_capacity(1, 64)                 # one more body beyond the current count
    (pieces, detached, pending), now, top = ow.connectivity()
    assert (pieces, detached, pending) == (1, 3, 0)
    assert now[0] == 6 and top[0] == 6 and ow.pending()[0] == 0
    st, _, _ = ow.bodies()
    np.testing.assert_allclose(st[0, 0], lat(20.5, 3, 0)[0], atol=1e-6)
    np.testing.assert_allclose(st[1, 1], lat(30, 4, 0)[1], atol=1e-6)


def test_bricks_of_other_structures_and_ground_stay(oracle):
    """Walking structure 0 leaves structure 1 alone, even an ungrounded piece of it; a piece touching the ground row
    without a foundation bond is still a footing only if its bottom brick has the bond (every bottom-row brick of a
    fresh structure does)."""
    s0 = cells_scene(COLUMN + [(5, 2, 0)], sid=0)
    s1 = cells_scene([(8, y, 0) for y in range(3)] + [(12, 7, 0)], sid=1)
    sc = S.Scene(np.concatenate([s0.static_xyz, s1.static_xyz]), np.concatenate([s0.static_mat, s1.static_mat]),
                 np.concatenate([s0.static_sid, s1.static_sid]), np.concatenate([s0.static_infill, s1.static_infill])).contiguous()
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(8, 64)
    (pieces, detached, _), now, top = ow.connect([0])
    assert (pieces, detached) == (1, 1)
    assert now[0] == 6 and top[0] == 6
    (pieces, detached, _), now, top = ow.connect([1])
    assert (pieces, detached) == (1, 1)
    assert now[1] == 3 and top[1] == 3


def test_failed_joints_leave_the_structure_pending_and_pieces_fall(oracle):
    """The 5-storey frame with two ground columns removed: once its joints go live, overloaded joints fail, the
    structure is pending, and connectivity() turns the pieces cut loose into bodies, which the rigid step then moves
    (they settle onto what is left of the frame: the contacts hold them up once the bonds are gone)."""
    fr, rm = S.frame5_structure()
    sc = fr.without_static(rm)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(64, 20000)
    ids = sc.structure_ids()
    for s in ids:
        ow.structure_warm(s)
    detached = 0
    for f in range(1, 200):
        r = ow.structure_frame(f, 1.0 / 60.0, ids)
        failed, crushed = r[5], r[6]
        if failed or crushed:
            assert ow.pending()[0] == 1
        (pieces, d, pending), now, _ = ow.connectivity()
        assert ow.pending()[0] == 0 and pending == 0
        detached += d
        if pieces:
            break
    assert detached > 0
    st0, _, _ = ow.bodies()
    for _ in range(10):
        ow.step(1.0 / 60.0, iterations=8)
    st1, _, fl = ow.bodies()
    assert (fl & 1).all() and np.isfinite(st1).all()
    assert ow.counts()["contacts"] > 0
    assert (st1[:, :3] != st0[:, :3]).any()

"""The CPU oracle against the known answers the reference offers for this path.

The reference holds no numeric golden vectors for the load path or the sphere solve (its tests are Node scripts
over the wasm build). What it does pin:
  * intact structures hold under their own weight: tests/stab.mjs runs every structure awake for 20 s and expects
    no brick lost — every joint ratio below 1 on a settled field;
  * the load-path equations themselves (src/lib.rs:1005-1026, 1153-1227), which give closed forms on simple
    shapes: a free-standing column carries the weight above each bond, and the foundation term sets the base.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S


def column(n, mat=S.CONC):
    xyz = np.array([[S.ORIGIN[0], y, S.ORIGIN[2]] for y in range(n)], np.int32)
    return S.Scene(xyz, np.full(n, mat, np.uint8), np.zeros(n, np.int32), np.zeros(n, np.uint8)).contiguous()


@pytest.mark.parametrize("n", [1, 3, 10])
def test_column_potential_closed_form(oracle, n):
    # brick y: (k_up + k_down + ground) phi_y - sum k phi_j = MASS. With k = 1 (concrete, vertical) and the
    # ground term GROUNDK * STIFF = 4 at y = 0: phi_{y+1} - phi_y = 300 (n - 1 - y) and 4 phi_0 = 300 n.
    w = oracle.OracleWorld(column(n))
    w.sor(0, omega=1.0, tol=1e-15, max_sweeps=200000, mode=oracle.MODE_LEX_F64)
    phi = w.phi64()
    expect = np.zeros(n)
    expect[0] = 75.0 * n
    for y in range(1, n):
        expect[y] = expect[y - 1] + 300.0 * (n - y)
    np.testing.assert_allclose(phi, expect, rtol=1e-12)


def test_column_joint_ratios_closed_form(oracle):
    n = 10
    w = oracle.OracleWorld(column(n))
    w.sor(0, omega=1.0, tol=1e-15, max_sweeps=200000, mode=oracle.MODE_LEX_F64)
    ids, vals, mr = w.stress(0, live=False)
    vert = {int(i): float(v[0]) for (i, ax, j, d, k), v in zip(ids, vals) if ax == 1}
    found = [float(v[0]) for (i, ax, j, d, k), v in zip(ids, vals) if ax == 3]
    for y in range(n - 1):
        # compression through the bond above y: 300 (n - 1 - y) over CAPV[concrete] = 140000
        assert vert[y] == pytest.approx(300.0 * (n - 1 - y) / 140000.0, rel=1e-6)
    assert found[0] == pytest.approx(4.0 * 75.0 * n / 280000.0, rel=1e-6)
    assert ids[:, 3].max() == 0


def test_intact_frame_holds(oracle):
    """tests/stab.mjs: an intact structure loses nothing under its own weight."""
    sc, _ = S.frame5_structure()
    w = oracle.OracleWorld(sc)
    w.sor(0, omega=1.7, tol=1e-9, max_sweeps=100000, mode=oracle.MODE_REDBLACK_F64)
    ids, vals, mr = w.stress(0, live=True)
    assert len(ids) > 5000
    assert mr < 1.0
    assert (ids[:, 3] == 0).all()


def test_frame_orders_agree(oracle):
    """Lexicographic (the reference's order) and red-black sweeps converge to the same FP64 fixed point."""
    sc, rm = S.frame5_structure()
    sc = sc.without_static(rm)
    a = oracle.OracleWorld(sc)
    a.sor(0, 1.7, 1e-13, 300000, mode=oracle.MODE_LEX_F64)
    b = oracle.OracleWorld(sc)
    b.sor(0, 1.7, 1e-13, 300000, mode=oracle.MODE_REDBLACK_F64)
    pa, pb = a.phi64(), b.phi64()
    assert np.abs(pa - pb).max() / pa.max() < 1e-9


def test_reference_f32_sweeps_reach_residual(oracle):
    """The reference's own f32 lexicographic sweeps (sor_struct) reach its residual measure and stay near the
    FP64 fixed point; the red-black f32 variant behaves the same."""
    sc, _ = S.frame5_structure()
    ex = oracle.OracleWorld(sc)
    ex.sor(0, 1.7, 1e-13, 300000, mode=oracle.MODE_LEX_F64)
    exact = ex.phi64()
    for mode in (oracle.MODE_LEX_F32, oracle.MODE_REDBLACK_F32):
        w = oracle.OracleWorld(sc)
        sweeps, r = w.sor(0, 1.7, 1e-6, 100000, mode=mode)
        assert r < 1e-6 and sweeps < 20000
        assert np.abs(w.phi() - exact).max() / exact.max() < 1e-3


def test_resting_load_closed_form(oracle):
    """structural's body loads (src/lib.rs:1233-1259): a 300 kg brick resting on one structure brick, clear of the
    ground, puts its whole weight share on that brick: ext = 0.8 * 0 + 0.2 * 300."""
    xyz = np.array([[S.ORIGIN[0], 0, S.ORIGIN[2]]], np.int32)
    pose = np.zeros((1, 13), np.float32)
    pose[0, :3] = [0.0, 0.5, 0.0]          # brick centre (0.25, 0.75, 0.25): the cell 0.29 m below is the static one
    pose[0, 6] = 1.0
    sc = S.Scene(xyz, np.array([S.CONC], np.uint8), np.zeros(1, np.int32), np.zeros(1, np.uint8),
                 np.array([0, 1], np.uint32), np.array([S.ORIGIN], np.int32), np.array([S.CONC], np.uint8), pose).contiguous()
    w = oracle.OracleWorld(sc)
    w.structure_loads([0])
    assert w.ext()[0] == np.float32(0.2) * np.float32(300.0)
    w.structure_loads([0])
    assert w.ext()[0] == np.float32(np.float32(0.2) * np.float32(300.0) * np.float32(0.8) + np.float32(0.2) * np.float32(300.0))


def test_oracle_rest_contacts(oracle):
    """A single brick resting on the ground: its 4 lower cube corners touch, normal +y (src/lib.rs:1415-1421)."""
    pose = np.zeros((1, 13), np.float32)
    pose[0, :3] = [0.0, -0.25 + 0.24, 0.0]   # centre at y = 0.24: corners 1 cm under the ground
    pose[0, 6] = 1.0
    sc = S.Scene(body_first=np.array([0, 1], np.uint32), body_brick_xyz=np.array([S.ORIGIN], np.int32),
                 body_brick_mat=np.array([S.CONC], np.uint8), body_pose=pose).contiguous()
    w = oracle.OracleWorld(sc)
    w.step(1 / 60, iterations=8)
    ids, f, s = w.contacts()
    assert len(ids) == 4
    assert (ids[:, 1] == 0xFFFFFFFF).all() and (ids[:, 4] == 0xFFFFFFFF).all()
    np.testing.assert_array_equal(f[:, 3:6], np.tile([0, 1, 0], (4, 1)))
    assert (s[:, 0] > 0).all()


def test_oracle_order_modes_close(oracle):
    """Colour order and list order differ only in the order of impulses: one step of a small pile stays close."""
    sc = S.debris_scene(150, seed=4, obstacles=(2, 3), spacing=1.2)
    a, b = oracle.OracleWorld(sc), oracle.OracleWorld(sc)
    for _ in range(30):
        a.step(1 / 60, iterations=8, order=oracle.ORDER_LIST)
        b.step(1 / 60, iterations=8, order=oracle.ORDER_COLOR)
    sa, _, fa = a.bodies()
    sb, _, fb = b.bodies()
    ok = (fa & 1) & (fb & 1)
    com_a = sa[ok == 1, 1].mean()
    com_b = sb[ok == 1, 1].mean()
    assert abs(com_a - com_b) < 0.5


def test_box_sat_face_contact(oracle):
    """collide_boxes (engine/src/phys.rs:531-628): a unit box resting 1 cm into another gives 4 face points."""
    a = np.array([0, 0, 0, 0, 0, 0, 1, 0.5, 0.5, 0.5], np.float32)
    b = np.array([0, 0.99, 0, 0, 0, 0, 1, 0.5, 0.5, 0.5], np.float32)
    n, nrm, pts = oracle.collide_boxes(a, b, margin=0.02)
    assert n == 4
    np.testing.assert_allclose(nrm, [0, 1, 0])
    np.testing.assert_allclose(pts[:, 3], -0.01, atol=1e-6)
    n2, _, _ = oracle.collide_boxes(a, np.array([0, 1.5, 0, 0, 0, 0, 1, 0.5, 0.5, 0.5], np.float32), margin=0.02)
    assert n2 == 0


def test_box_sat_edge_contact(oracle):
    """Two boxes crossed edge to edge (45 degrees about different axes) touch in one edge-edge point."""
    s = np.sin(np.pi / 8); c = np.cos(np.pi / 8)
    a = np.array([0, 0, 0, 0, 0, s, c, 0.5, 0.5, 0.5], np.float32)          # 45 degrees about z
    b = np.array([0, 1.40, 0, s, 0, 0, c, 0.5, 0.5, 0.5], np.float32)       # 45 degrees about x, edge down
    n, nrm, pts = oracle.collide_boxes(a, b, margin=0.02)
    assert n == 1
    assert nrm[1] > 0.99
    assert pts[0, 3] < 0


def _proper(a, b, col, limit):
    seen = set()
    for x, y, c in zip(a, b, col):
        if c >= limit:
            continue
        for body in (x, y):
            if body == 0xFFFFFFFF:
                continue
            assert (body, c) not in seen
            seen.add((body, c))


def test_reference_colouring_restatement(oracle):
    """gpu/gpu_world.js:922-1038 restated: a proper colouring of the coloured manifolds; supports (a static side)
    claim in the first rounds; a body with more manifolds than colours sends the rest to the overflow pass."""
    rng = np.random.default_rng(3)
    n_bodies = 300
    a = rng.integers(0, n_bodies, 1500).astype(np.uint32)
    b = rng.integers(0, n_bodies, 1500).astype(np.uint32)
    b[b == a] = (b[b == a] + 1) % n_bodies
    b[rng.random(1500) < 0.3] = 0xFFFFFFFF
    col, used, ovf = oracle.ref_colouring(a, b, np.ones(1500, np.uint8), (b != 0xFFFFFFFF).astype(np.uint8), n_bodies)
    _proper(a, b, col, 16)
    assert used <= 16 and ovf == int((col >= 16).sum())
    # a star of 20 awake manifolds at body 0 with 4 colours: at most 4 coloured
    a2 = np.zeros(20, np.uint32)
    b2 = np.arange(1, 21, dtype=np.uint32)
    col2, used2, ovf2 = oracle.ref_colouring(a2, b2, np.ones(20, np.uint8), np.ones(20, np.uint8), 21, color_limit=4)
    _proper(a2, b2, col2, 4)
    assert used2 <= 4 and ovf2 >= 16


def test_long_horizon_orders_agree_statistically(oracle):
    """The colour order (the GPU's) and the reference's list order diverge bit-wise within a few steps of a pile; after
    300 steps of a 1,500-body debris scene with the reference's pinch removal, they agree as statistics: centre-of-mass
    height and each material's mean height within 5 cm, each material's height histogram within a total variation
    distance of 0.08, and each fragment size class's surviving fraction within 0.05 (measured: 1 mm, 4 mm, 0.012 and
    0.008)."""
    sc = S.debris_scene(1500, seed=4)
    a, b = oracle.OracleWorld(sc), oracle.OracleWorld(sc)
    for _ in range(300):
        a.step(1 / 60, iterations=8, order=oracle.ORDER_LIST)
        b.step(1 / 60, iterations=8, order=oracle.ORDER_COLOR)
    sa, _, fa = a.bodies()
    sb, _, fb = b.bodies()
    assert not np.array_equal(sa, sb)            # the orders really differ bit-wise
    ha, hb = S.horizon_stats(sc, sa, fa), S.horizon_stats(sc, sb, fb)
    d = S.horizon_distance(ha, hb)
    assert ha["alive"] < sc.n_bodies             # the pinch removal took part
    assert d["com_y"] <= 0.05 and d["mean_y"] <= 0.05
    assert d["height_tv"] <= 0.08
    assert d["survival"] <= 0.05

"""Closed-form known answers of the rigid step, checked on the CPU oracle.

The reference holds no numeric golden vectors for its sphere solve, so these pin the oracle's restatement of
src/lib.rs against answers that follow from the reference's own equations on cases simple enough to solve by hand:

  * free fall with drag: gravity at the start of each substep (src/lib.rs:1772), then the position update and the
    linear drag v *= 1 - 0.01 h of integrate (src/lib.rs:1703-1712), give a geometric recurrence with a closed form;
  * the rest timer: a brick resting on the ground accumulates h per substep and sleeps on the first substep whose
    timer exceeds 0.45 s (src/lib.rs:1720-1734);
  * a head-on pair of single-brick spheres: the normal effective mass of a central contact is m/2, and the first
    normal impulse is mn * (-vn + bias) with bias = max(min(0.2/h * (depth - 0.01), 1), -0.12 vn) (src/lib.rs:1551-1590);
  * the pinch clamps: a linear velocity change above 8 m/s in one substep is scaled back to 8 m/s, a rim-speed change
    above 6 m/s to 6 m/s (src/lib.rs:1746-1768).

Each expectation is computed in float64 from the formula (not by re-running the oracle's code), with the tolerance
stated beside it; where the reference's f32 evaluation order is itself the answer, a float32 evaluation of the
formula in that order is compared bit for bit.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S

G = 9.81
DT = 1.0 / 60.0


def body_scene(cells_per_body, poses, mat=S.CONC):
    """Bodies of the given local lattice cells (relative to the lattice origin cell) and 13-float poses."""
    first = [0]
    xyz = []
    for cells in cells_per_body:
        for c in cells:
            xyz.append([S.ORIGIN[0] + c[0], S.ORIGIN[1] + c[1], S.ORIGIN[2] + c[2]])
        first.append(len(xyz))
    pose = np.asarray(poses, np.float32).reshape(-1, 13)
    return S.Scene(body_first=np.array(first, np.uint32), body_brick_xyz=np.array(xyz, np.int32),
                   body_brick_mat=np.full(len(xyz), mat, np.uint8), body_pose=pose).contiguous()


def pose(p, v=(0, 0, 0), w=(0, 0, 0), q=(0, 0, 0, 1)):
    return [*p, *q, *v, *w]


# ---------------------------------------------------------------- free fall with drag
def test_free_fall_with_drag_closed_form(oracle):
    """No contacts: per substep v.y -= g h; p += v h; v *= c with c = 1 - 0.01 h (spin: w *= 1 - 0.05 h).
    With u_k the velocity after substep k: u_{k+1} = c (u_k - g h e_y), so u_k = u* + c^k (u_0 - u*) with
    u* = -c g h / (1 - c), and p_n = p_0 + h sum_{k<n} (u_k - g h e_y)."""
    sc = body_scene([[(0, 0, 0)]], [pose((0.0, 60.0, 0.0), v=(1.0, 2.0, -0.5), w=(0.3, 0.0, 0.0))])
    ow = oracle.OracleWorld(sc)
    st0, _, _ = ow.bodies()
    steps = 60
    for _ in range(steps):
        ow.step(DT, iterations=8)
    st, sl, fl = ow.bodies()
    h = DT / 2.0
    n = 2 * steps
    c = 1.0 - 0.01 * h
    gh = G * h
    u0 = st0[0, 7:10].astype(np.float64)
    # vertical
    ustar = -c * gh / (1.0 - c)
    k = np.arange(n)
    uy = ustar + c ** k * (u0[1] - ustar)
    py = st0[0, 1] + h * np.sum(uy - gh)
    vy = ustar + c ** n * (u0[1] - ustar)
    # horizontal: no gravity
    vx, vz = u0[0] * c ** n, u0[2] * c ** n
    px = st0[0, 0] + h * u0[0] * (1.0 - c ** n) / (1.0 - c)
    pz = st0[0, 2] + h * u0[2] * (1.0 - c ** n) / (1.0 - c)
    wx = float(st0[0, 10]) * (1.0 - 0.05 * h) ** n
    # f32 accumulation over 120 substeps: a few ulps of 60 m per substep
    np.testing.assert_allclose(st[0, [0, 1, 2]], [px, py, pz], rtol=2e-6, atol=2e-5)
    np.testing.assert_allclose(st[0, [7, 8, 9]], [vx, vy, vz], rtol=2e-6, atol=2e-6)
    # 120 successive f32 products (1 - 0.05 h): up to 120 roundings of 2^-24 each
    np.testing.assert_allclose(st[0, 10], wx, rtol=1e-5)
    assert fl[0] == 1 and sl[0] == 0.0     # alive, awake, never at rest (no contact)

    # the reference's f32 order, evaluated from the formula: bit for bit
    v = st0[0, 7:10].copy()
    p = st0[0, 0:3].copy()
    h32 = np.float32(DT) * np.float32(0.5)
    c32 = np.float32(1.0) - np.float32(0.01) * h32
    for _ in range(n):
        v[1] = np.float32(v[1] - np.float32(G) * h32)
        p = (p + v * h32).astype(np.float32)
        v = (v * c32).astype(np.float32)
    np.testing.assert_array_equal(st[0, 0:3], p)
    np.testing.assert_array_equal(st[0, 7:10], v)


# ---------------------------------------------------------------- the rest timer
def test_resting_brick_sleeps_on_the_predicted_substep(oracle):
    """A brick with its lower corners 1 cm into the ground is at rest from the first substep (4 contacts, |v|^2 far
    below the small-body threshold 0.16, no stress). Its timer grows by h per substep; it sleeps on the first
    substep whose timer exceeds 0.45 s, when v and w are zeroed."""
    sc = body_scene([[(0, 0, 0)]], [pose((0.0, -0.25 + 0.24, 0.0))])
    ow = oracle.OracleWorld(sc)
    h = np.float32(DT) * np.float32(0.5)
    timer = np.float32(0.0)
    predicted_substep = None
    for k in range(1, 200):
        timer = np.float32(timer + h)
        if timer > np.float32(0.45):
            predicted_substep = k
            break
    # 0.45 / (1/120) = 54 exactly in real numbers; f32 accumulation decides whether 54 or 55 substeps pass it
    assert predicted_substep in (54, 55)
    sleep_step = (predicted_substep + 1) // 2
    timer = np.float32(0.0)
    for step in range(1, sleep_step + 3):
        ow.step(DT, iterations=8)
        st, sl, fl = ow.bodies()
        if step < sleep_step:
            timer = np.float32(np.float32(timer + h) + h)
            assert fl[0] == 1, step                 # alive, awake
            assert sl[0] == timer, (step, sl[0], timer)
            assert float(np.dot(st[0, 7:10], st[0, 7:10])) < 0.16
        else:
            assert fl[0] == 3, step                 # alive, asleep
            np.testing.assert_array_equal(st[0, 7:13], np.zeros(6, np.float32))
    ids, f, s = ow.contacts()
    assert len(ids) == 0                          # asleep bodies generate no contacts


# ---------------------------------------------------------------- head-on pair
@pytest.mark.parametrize("gap,speed", [(0.48, 3.0), (0.52, 3.0), (0.50, 0.5)])
def test_head_on_pair_first_normal_impulse(oracle, gap, speed):
    """Two single concrete bricks (300 kg each) at the same height, centres `gap` apart along x, approaching at
    `speed` each. The contact runs from brick 0 to brick 1 (normal -x, pointing from b to a), its arm is parallel to
    the normal, so the angular terms vanish: mn = 1 / (1/300 + 1/300) = 150. vn = -2 speed, depth = 2 RB - gap,
    bias = min(0.2/h * max(depth - 0.01, 0), 1), raised to -0.12 vn when vn < -2. One iteration gives
    jn = mn (-vn + bias); further iterations add nothing (the normal velocity then equals the bias, and there is no
    tangential velocity to give friction work)."""
    x0 = -gap / 2.0
    sc = body_scene([[(0, 0, 0)], [(0, 0, 0)]],
                    [pose((x0 - 0.25, 20.0, -0.25), v=(speed, 0, 0)), pose((-x0 - 0.25, 20.0, -0.25), v=(-speed, 0, 0))])
    h = DT                                   # one substep of dt
    mn = 1.0 / (1.0 / 300.0 + 1.0 / 300.0)
    vn = -2.0 * speed
    depth = 2 * 0.27 - gap
    bias = min(0.2 / h * max(depth - 0.01, 0.0), 1.0)
    if vn < -2.0:
        bias = max(bias, -0.12 * vn)
    jn = mn * (-vn + bias)
    for iters in (1, 8):
        ow = oracle.OracleWorld(sc)
        ow.step(DT, iterations=iters, substeps=1)
        ids, f, s = ow.contacts()
        assert len(ids) == 1
        assert ids[0, 0] == 0 and ids[0, 1] == 1
        np.testing.assert_allclose(f[0, 3:6], [-1.0, 0.0, 0.0], atol=1e-7)
        np.testing.assert_allclose(f[0, 6], depth, rtol=1e-5)
        jn_, jt1, jt2, mn_, mt1, mt2, bias_, vn0 = s[0]
        assert mn_ == pytest.approx(mn, rel=1e-6)
        assert bias_ == pytest.approx(bias, rel=1e-6)
        assert vn0 == pytest.approx(-vn, rel=1e-6)
        assert jn_ == pytest.approx(jn, rel=1e-5)
        assert jt1 == 0.0 and jt2 == 0.0
        # the velocities after the impulse: v_a = speed - jn/300, v_b = -v_a; then linear drag and the small-body
        # rolling resistance of integrate (nc > 0, one brick): v *= (1 - 0.01 h)(1 - min(2 h, 0.3))
        st, _, _ = ow.bodies()
        damp = (1.0 - 0.01 * h) * (1.0 - min(2.0 * h, 0.3))
        va = (speed - jn / 300.0) * damp
        assert st[0, 7] == pytest.approx(va, rel=1e-5, abs=1e-6)
        assert st[1, 7] == pytest.approx(-va, rel=1e-5, abs=1e-6)


# ---------------------------------------------------------------- pinch clamps
def test_pinch_clamp_linear_8_mps(oracle):
    """A 2 x 2 x 1 slab (4 bricks: not small, so no rolling resistance) hits the ground at 20 m/s. The solve would
    stop it within the substep (a velocity change near 20 m/s); the pinch check scales the change back to 8 m/s
    along its direction: v = v_pre + dv * 8 / |dv| with v_pre the velocity after gravity. After integrate's drag
    (v *= 1 - 0.01 h) the clamped change is recovered exactly as |v / (1 - 0.01 h) - v_pre| = 8. With pinch removal
    on (the reference's default) the same 4-brick body is removed instead."""
    slab = [(0, 0, 0), (1, 0, 0), (0, 0, 1), (1, 0, 1)]
    sc = body_scene([slab], [pose((-0.5, -0.25 + 0.24, -0.5), v=(0.0, -20.0, 0.0))])
    ow = oracle.OracleWorld(sc)
    st0, _, _ = ow.bodies()
    h = DT
    ow.step(DT, iterations=8, substeps=1, pinch_kill=0)
    st, _, fl = ow.bodies()
    assert fl[0] == 1
    vpre = st0[0, 7:10].astype(np.float64) + np.array([0.0, -G * h, 0.0])
    v = st[0, 7:10].astype(np.float64) / (1.0 - 0.01 * h)
    assert np.linalg.norm(v - vpre) == pytest.approx(8.0, rel=1e-5)
    assert v[1] > vpre[1] + 7.9                       # the change points up
    ow2 = oracle.OracleWorld(sc)
    ow2.step(DT, iterations=8, substeps=1, pinch_kill=1)
    _, _, fl2 = ow2.bodies()
    assert fl2[0] == 0                                # <= 6 bricks, pinched: removed as src/lib.rs:1755-1760
    # a slow landing (2 m/s) changes v by less than 8 m/s: not clamped, and stopped by the contacts
    sc3 = body_scene([slab], [pose((-0.5, -0.25 + 0.24, -0.5), v=(0.0, -2.0, 0.0))])
    ow3 = oracle.OracleWorld(sc3)
    ow3.step(DT, iterations=8, substeps=1, pinch_kill=1)
    st3, _, fl3 = ow3.bodies()
    assert fl3[0] == 1 and st3[0, 8] > -0.5


def test_pinch_clamp_rim_speed_6_mps(oracle):
    """A rod of 6 bricks along x, tilted 30 degrees about z, lands on one end at 20 m/s. The end contact gives the rod
    a spin change whose rim speed |dw| * radius exceeds 6 m/s; the pinch check scales dw back to a rim speed of 6:
    w = w_pre + dw * 6 / (|dw| radius). w_pre = 0 (the rod starts without spin), and integrate damps spin by
    (1 - 0.05 h), so |w| radius / (1 - 0.05 h) = 6."""
    rod = [(i, 0, 0) for i in range(6)]
    a = np.deg2rad(30.0)
    q = (0.0, 0.0, np.sin(a / 2), np.cos(a / 2))
    # lowest corner of the rod about 1 cm under the ground: place the parent so the rotated rod's low end is at y 0
    sc = body_scene([rod], [pose((0.0, 0.0, 0.0), q=q)])
    ow = oracle.OracleWorld(sc)
    st0, _, _ = ow.bodies()
    # shift the body so its lowest brick corner sits 1 cm below the ground, then drop it at 20 m/s
    wp = ow.brick_positions()
    R = np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])
    corners = np.array([[sx, sy, sz] for sx in (-0.25, 0.25) for sy in (-0.25, 0.25) for sz in (-0.25, 0.25)]) @ R.T
    low = min((p + corners)[:, 1].min() for p in wp)
    st0[0, 1] -= low + 0.01
    st0[0, 7:10] = [0.0, -20.0, 0.0]
    ow.set_bodies(st0, np.zeros(1, np.float32), np.ones(1, np.uint8))
    rad = float(ow.setup()[0][0, 2])
    assert rad == pytest.approx(np.sqrt(1.25 ** 2) + 0.25 * 1.8, rel=1e-6)
    h = DT
    ow.step(DT, iterations=8, substeps=1, pinch_kill=0)
    st, _, fl = ow.bodies()
    assert fl[0] == 1
    w = st[0, 10:13].astype(np.float64) / (1.0 - 0.05 * h)
    assert np.linalg.norm(w) * rad == pytest.approx(6.0, rel=1e-5)

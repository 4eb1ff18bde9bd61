"""The debris-body load field (structural's body part, src/lib.rs:1262-1266, 1282-1365) in the CPU oracle, against
answers that follow from the reference's rules:

  * the sweep budget of 160,000 brick updates is shared in body order: a piece sweeps to its own stopping point (at
    least 2, residual below 4e-4, at most 60) or until the budget is spent, whichever comes first, and every piece
    after the budget is spent still gets 2 sweeps;
  * a loaded piece's bricks carry MASS (n - 1), n = |g - a| / g from the piece's change of velocity and spin over the
    frame;
  * a piece that no contact has supported for 10 frames starts its potentials over, and a piece that is not loaded
    lets its load time run down by 2 dt a frame;
  * a beam landing on one end fails and crushes joints; each crushed brick leaves its piece at the next rebuild, each
    failure can split it, and a crush the frame's budget of 300 cannot pay for is a failure instead.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S

DT = np.float32(1.0 / 60.0)
IT = 8
GR = np.float32(9.81)
MASS_CONC = np.float32(300.0)


def test_budget_is_shared_in_body_order(oracle):
    """Three 4,000-brick blocks on the ground, first frame: the first block would need more than 40 sweeps, so the
    budget stops it at ceil(160,000 / 4,000) = 40; the other two get 2 sweeps each."""
    ow = oracle.OracleWorld(S.body_blocks())
    ow.set_capacity(16, 16)
    ow.step(DT, iterations=IT)
    bodies, sweeps, updates, joints, over, failed, crushed, maxr, crush_after = ow.body_frame(DT)
    assert (bodies, sweeps, updates) == (3, 44, 176000)
    # every joint of the three blocks is judged once (each block: 19*8*25 + 20*7*25 + 20*8*24 = 11,140)
    assert joints == 3 * 11140 and failed == 0 and crushed == 0 and crush_after == 0
    resid, nmax, lt, mr = ow.body_state()
    assert np.all(lt == DT) and np.all(mr >= 0.0)
    assert resid[1] > 4e-4 and resid[2] > 4e-4   # 2 sweeps do not settle a fresh field


def test_inertial_load_from_the_change_of_velocity(oracle):
    """First frame of the blocks: the velocities of the last frame are those of the set-up (at rest), so each
    brick's load is MASS (n - 1) for the brick's acceleration (v - 0) / dt + w / dt x (p - pos) over g."""
    ow = oracle.OracleWorld(S.body_blocks())
    ow.set_capacity(16, 16)
    ow.step(DT, iterations=IT)
    st, _, _ = ow.bodies()
    wpos = ow.brick_positions()
    ow.body_frame(DT)
    _, ext = ow.body_phi()
    first = S.body_blocks().body_first
    idt = np.float32(1.0) / DT
    for b in range(3):
        v, w, pb = st[b, 7:10], st[b, 10:13], st[b, 0:3]
        al = v * idt
        aa = w * idt
        r = wpos[first[b]:first[b + 1]] - pb
        cr = np.stack([aa[1] * r[:, 2] - aa[2] * r[:, 1], aa[2] * r[:, 0] - aa[0] * r[:, 2],
                       aa[0] * r[:, 1] - aa[1] * r[:, 0]], 1).astype(np.float32)
        a = al + cr
        ge = np.stack([-a[:, 0], -GR - a[:, 1], -a[:, 2]], 1).astype(np.float32)
        n = np.minimum(np.sqrt((ge * ge).sum(1, dtype=np.float32)) / GR, np.float32(150.0))
        np.testing.assert_allclose(ext[first[b]:first[b + 1]], MASS_CONC * (n - np.float32(1.0)), rtol=2e-5, atol=2e-3)
    _, nmax, _, _ = ow.body_state()
    assert np.all(nmax >= 1.0)


def test_unsupported_piece_starts_over(oracle):
    """A block with a load field is lifted 10 m: it is no longer in contact (not loaded, its load time runs down by
    2 dt a frame) and, once no contact has supported it for 10 frames, its potentials are 0."""
    sc = S.body_blocks(n=1)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(4, 4)
    for _ in range(3):
        ow.step(DT, iterations=IT)
        ow.body_frame(DT)
    phi, _ = ow.body_phi()
    assert phi.max() > 0.0
    _, _, lt0, _ = ow.body_state()
    st, sl, fl = ow.bodies()
    st[0, 1] += 10.0
    st[0, 7:13] = 0.0
    ow.set_bodies(st, sl, fl)
    expect = lt0[0]
    for k in range(1, 13):
        ow.step(DT, iterations=IT)
        ow.body_frame(DT)
        phi, _ = ow.body_phi()
        _, _, lt, _ = ow.body_state()
        expect = max(np.float32(expect - np.float32(2.0) * DT), np.float32(0.0))
        assert lt[0] == expect, k
        if k <= 8:
            assert phi.max() > 0.0, k
    assert np.all(phi == 0.0)


def test_beam_landing_fails_and_crushes_joints(oracle):
    """A 60-brick concrete beam dropped on one end from 30 m: on landing its judged joints fatigue, fail and crush;
    every crushed brick leaves the beam at the next rebuild, and the failures split it into pieces."""
    ow = oracle.OracleWorld(S.tilted_beam())
    ow.set_capacity(64, 4000)
    tot = np.zeros(7, np.int64)
    removed = pieces = 0
    for _ in range(240):
        ow.step(DT, iterations=IT)
        r = ow.rebuild_bodies()
        removed += r[2]
        pieces += r[1]
        o = ow.body_frame(DT)
        assert o[8] == o[6]          # no structure crushed this frame: the pieces' crushes are the frame's
        tot += np.array(o[:7])
    assert tot[5] > 0 and tot[6] > 0
    assert removed == tot[6]
    assert pieces > 0


def test_crush_budget_spent_turns_crushes_into_failures(oracle):
    """Two copies of the beam in lockstep; on the first frame that crushes, the copy told that the frame's 300
    crushes are spent crushes nothing and fails at least the joints the other crushed, and every joint the other
    skipped after its crushes is judged."""
    worlds = [oracle.OracleWorld(S.tilted_beam()) for _ in range(2)]
    for ow in worlds:
        ow.set_capacity(64, 4000)
    for f in range(240):
        for ow in worlds:
            ow.step(DT, iterations=IT)
            ow.rebuild_bodies()
        a = worlds[0].body_frame(DT, 0)
        b = worlds[1].body_frame(DT, 300)
        if a[6]:
            assert b[6] == 0 and b[8] == 300
            assert b[5] >= a[5] + a[6]
            assert b[3] >= a[3]
            return
        assert a[:8] == b[:8]
    pytest.fail("the beam never crushed a brick")

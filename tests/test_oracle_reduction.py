"""Contact reduction and warm start in the CPU oracle (the GPU world's devices for large contact sets,
gpu/gpu_world.js:557-576, 834-920, restated for brick contacts), against answers that follow from their rules:

  * reduction: a body pair with more than 32 contacts keeps, for each of the 26 directions to a cube cell's
    neighbours, the contact whose point reaches furthest along it, and the deepest (ties to the later contact); the
    kept set is recomputed here from the unreduced contact list of the same step; the others carry no impulse and
    the pair's manifolds hold only the kept ones, so a block on the ground needs one colour instead of 125;
  * warm start: a stack of single bricks solved with few iterations sinks less than from zero and still stands;
    the table starts over after a rebuild (brick ids move).
"""
import numpy as np

from shatterforge_b200 import scenes as S

DT = np.float32(1.0 / 60.0)
STATIC = 0xFFFFFFFF


def f2o(x):
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return np.where(b & 0x80000000, (~b) & 0xFFFFFFFF, b | 0x80000000)


def expected_kept(ids, f):
    """The kept contacts of one step's list (ids: a, b, bo, ba, bb; f: point 3, normal 3, depth)."""
    keys = ids[:, 0].astype(np.uint64) << np.uint64(32) | np.where(ids[:, 1] == STATIC, 0, ids[:, 1] + 1).astype(np.uint64)
    keep = np.ones(len(ids), bool)
    p = f[:, :3].astype(np.float32)
    scores = []
    for k in range(26):
        j = k + 1 if k >= 13 else k
        dx, dy, dz = np.float32(j % 3 - 1), np.float32((j // 3) % 3 - 1), np.float32(j // 9 - 1)
        scores.append(f2o(p[:, 0] * dx + p[:, 1] * dy + p[:, 2] * dz))
    scores.append(f2o(f[:, 6]))
    for key in np.unique(keys):
        idx = np.nonzero(keys == key)[0]
        if len(idx) <= 32:
            continue
        win = set()
        for sc in scores:
            v = sc[idx]
            win.add(int(idx[np.nonzero(v == v.max())[0].max()]))
        keep[idx] = False
        keep[list(win)] = True
    return keep


def test_reduction_keeps_the_extremes_and_the_deepest(oracle):
    sc = S.body_blocks()
    plain = oracle.OracleWorld(sc)
    red = oracle.OracleWorld(sc)
    for ow, r in ((plain, 0), (red, 1)):
        ow.set_capacity(16, 16)
        ow.step(DT, iterations=8, reduce=r)
    ids, f, _ = plain.contacts()
    rids, rf, rs = red.contacts()
    np.testing.assert_array_equal(ids, rids)     # the list is generated before the reduction
    np.testing.assert_array_equal(f, rf)
    keep = expected_kept(ids, f)
    assert keep.sum() < len(keep) // 10
    kept = rs[:, 3] != 0.0                        # a kept contact has an effective mass; a left-out one reads zeros
    np.testing.assert_array_equal(kept, keep)
    assert not rs[~kept].any()
    m = red.manifolds()
    assert m[:, 3].sum() == keep.sum()
    assert plain.counts()["colors"] == 125 and red.counts()["colors"] == 1


def test_reduction_leaves_small_pairs_alone(oracle):
    """Compound debris of at most 64 bricks: pairs of at most 32 contacts are untouched, so a run with reduction on
    equals one without until a pair grows past 32."""
    sc = S.debris_scene(200, seed=5, kmax=8)
    a = oracle.OracleWorld(sc)
    b = oracle.OracleWorld(sc)
    for _ in range(90):
        a.step(DT, iterations=8)
        b.step(DT, iterations=8, reduce=1)
        ids, f, _ = a.contacts()
        if len(ids) and not expected_kept(ids, f).all():
            break
        np.testing.assert_array_equal(a.bodies()[0], b.bodies()[0])


def stack(n=6):
    xyz = np.tile(np.array(S.ORIGIN, np.int32), (n, 1))
    pose = np.zeros((n, 13), np.float32)
    pose[:, 6] = 1.0
    for k in range(n):
        pose[k, 1] = k * 0.5 + 0.001 * k
    return S.Scene(body_first=np.arange(n + 1, dtype=np.uint32), body_brick_xyz=xyz,
                   body_brick_mat=np.full(n, S.CONC, np.uint8), body_pose=pose).contiguous()


def test_warm_start_stack_sinks_less_and_stands(oracle):
    """Six single bricks stacked, 1, 2 or 4 iterations: over steps 10-40 (before the stack sleeps) the deepest
    contact is shallower with warm start (measured 0.022 / 0.017 / 0.012 m against 0.038 / 0.025 / 0.017 m), and
    after 120 steps the stack still stands."""
    for it in (1, 2, 4):
        depth = {}
        for warm in (0, 1):
            ow = oracle.OracleWorld(stack())
            md = []
            for _ in range(120):
                ow.step(DT, iterations=it, warm=warm)
                _, f, _ = ow.contacts()
                md.append(f[:, 6].max() if len(f) else 0.0)
            st, _, fl = ow.bodies()
            assert st[-1, 1] > 2.5, (it, warm)               # the top brick is still on the stack (fallen: below 1.5)
            depth[warm] = max(md[10:40])
        assert depth[1] < 0.8 * depth[0], (it, depth)


def test_warm_start_carries_the_last_impulse(oracle):
    """A resting brick: with no iteration the solve only applies what it starts from, so each substep's impulses
    are 0.8 of the last's (a geometric decay from the first solved substep), and without warm start they are 0."""
    sc = stack(1)
    ow = oracle.OracleWorld(sc)
    for _ in range(5):
        ow.step(DT, iterations=8, warm=1)
    _, _, s = ow.contacts()
    jn = s[:, 0].copy()
    assert (jn > 0).any()
    ow.step(DT, iterations=0, substeps=1, warm=1)
    _, _, s1 = ow.contacts()
    np.testing.assert_array_equal(s1[:, 0], jn * np.float32(0.8))
    cold = oracle.OracleWorld(sc)
    for _ in range(5):
        cold.step(DT, iterations=8)
    cold.step(DT, iterations=0, substeps=1)
    assert not cold.contacts()[2][:, 0].any()


def test_warm_table_starts_over_after_a_rebuild(oracle):
    sc = stack(1)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(4, 4)
    for _ in range(5):
        ow.step(DT, iterations=8, warm=1)
    ow.remove_bricks(body_bricks=[])
    ow.step(DT, iterations=0, substeps=1, warm=1)
    assert ow.contacts()[2][:, 0].any()            # nothing moved: the table holds
    # a rebuild of a marked body (its only brick kept) moves nothing in place but starts the table over
    b2 = oracle.OracleWorld(S.tilted_beam(length=8, angle_deg=0.0, height=0))
    b2.set_capacity(8, 64)
    for _ in range(5):
        b2.step(DT, iterations=8, warm=1)
    b2.remove_bricks(body_bricks=[3])
    assert b2.rebuild_bodies()[0] == 1
    b2.step(DT, iterations=0, substeps=1, warm=1)
    assert not b2.contacts()[2][:, 0].any()

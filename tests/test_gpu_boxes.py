"""The box world on the GPU (sf_box_world_*: the engine crate's World::step, engine/src/phys.rs:152-354) against the
oracle's colour-order restatement, bit for bit: every box's pose, velocities and sleep state, the step's counts, and
each manifold's pair, points, normal, impulses, sticking flag and colour; plus the reference's own gates on the GPU's
results (stack drift and speed, the pile's height range against the reference's list order).
"""
import numpy as np
import pytest

from shatterforge_b200 import boxes as X

pytestmark = pytest.mark.gpu

DT = np.float32(1.0 / 60.0)


def stats_tuple(st):
    return (st.awake, st.pairs, st.manifolds, st.points, st.colours)


def compare(w, ow, scene=0, manifolds=True):
    np.testing.assert_array_equal(w.state(scene), ow.state())
    assert stats_tuple(w.stats(scene)) == ow.stats()
    assert w.stats(scene).status == 0
    if manifolds:
        np.testing.assert_array_equal(w.manifolds(scene), ow.manifolds())


def run_pair(oracle, recs, params, steps, every=1, manifolds_every=10):
    w = X.BoxWorld(recs, params)
    ow = oracle.OracleBoxWorld(recs, params, oracle.ORDER_COLOR)
    for k in range(1, steps + 1):
        w.step(DT)
        ow.step(DT)
        if k % every == 0 or k == steps:
            compare(w, ow, manifolds=k % manifolds_every == 0 or k == steps)
        else:
            assert stats_tuple(w.stats()) == ow.stats(), k
    return w, ow


def test_pile_2000_against_oracle(sf, oracle):
    """The reference's pile of 2,000 boxes (4 sub-steps, no sleep) for its 2 s: every step's counts, the state every
    5 steps, the manifolds every 10; the height range stays within the reference's GPU tolerance of its CPU."""
    w, ow = run_pair(oracle, X.pile(2000), X.box_params(allow_sleep=0, substeps=4), 120, every=5)
    y = w.state()[:, 1]
    assert abs(y.min() - 0.117) < 0.02 and abs(y.max() - 4.828) < 0.1


@pytest.mark.parametrize("sleep", [0, 1])
def test_stack_20_against_oracle(sf, oracle, sleep):
    """The 20-box gate stack for 10 s at 12 sub-steps: bit-exact, and within the gate (drift < 10 mm, < 10 mm/s)."""
    recs = X.stack(20)
    w, ow = run_pair(oracle, recs, X.box_params(allow_sleep=sleep), 600, every=60, manifolds_every=120)
    s = w.state()
    assert np.linalg.norm(s[19, :3] - np.array([0.0, recs[19, 1], 0.0])) < 0.01
    assert np.linalg.norm(s[:, 7:10], axis=1).max() < 0.01
    if sleep:
        assert s[:, 21].sum() == 0


def test_tilted_box_and_column_against_oracle(sf, oracle):
    w, _ = run_pair(oracle, X.tilted_box(), X.box_params(), 300, every=10)
    assert abs(w.state()[0, 1] - 0.125) < 0.005
    w, _ = run_pair(oracle, X.offset_column(), X.box_params(), 600, every=20)
    s = w.state()
    assert s[:, 1].max() < 3.0 and s[:, 1].min() > 0.2


def test_scenes_in_one_launch_against_their_oracles(sf, oracle):
    """Five scenes in one world (a 600-box pile, the stack, the tilted box, the column, a pile with a static floor
    slab and a static wall that sleeping boxes lie against and get woken from): each equals its own oracle."""
    floor = X.pile(300)
    floor[:, 1] += np.float32(1.0)
    slab = np.array([[4.0, 0.5, 3.0, 0, 0, 0, 1, 4.0, 0.5, 4.0, 0.0], [-0.6, 2.0, 3.0, 0, 0, 0, 1, 0.3, 2.0, 4.0, 0.0]],
                    np.float32)
    scenes = [X.pile(600), X.stack(20), X.tilted_box(), X.offset_column(), np.concatenate([slab, floor])]
    p = X.box_params()
    w = X.BoxWorld(scenes, p)
    ows = [oracle.OracleBoxWorld(s, p, oracle.ORDER_COLOR) for s in scenes]
    for k in range(1, 241):
        w.step(DT)
        for ow in ows:
            ow.step(DT)
        for i, ow in enumerate(ows):
            assert stats_tuple(w.stats(i)) == ow.stats(), (k, i)
        if k % 40 == 0:
            for i, ow in enumerate(ows):
                compare(w, ow, scene=i)
    assert w.state(4)[2:, 21].sum() < len(floor)          # some of the pile on the slab has gone to sleep


def test_pile_20000_full_size_against_oracle(sf, oracle):
    """The reference's throughput case: 20,000 boxes, 12 sub-steps, no sleep. 20 steps bit-exact (the pile is still
    landing: the most pairs and colours), with the counts every step."""
    recs = X.pile(20000)
    p = X.box_params(allow_sleep=0)
    w = X.BoxWorld(recs, p)
    ow = oracle.OracleBoxWorld(recs, p, oracle.ORDER_COLOR)
    for k in range(20):
        w.step(DT)
        ow.step(DT)
        assert stats_tuple(w.stats()) == ow.stats(), k
    compare(w, ow)
    assert w.stats().pairs > 50000


def test_rubble_of_convex_cells_against_oracle(sf, oracle):
    """Convex cells of the hull library in the box world (every fifth a plain box): pairs through the convex-cell SAT,
    cells on the ground in one or two patches; 240 steps with sleep on, the counts every step, the state and the
    manifolds every 20."""
    from test_oracle_boxes import rubble
    recs, lib, ids = rubble(500)
    p = X.box_params()
    w = X.BoxWorld(recs, p)
    w.set_hulls(lib, ids)
    ow = oracle.OracleBoxWorld(recs, p, oracle.ORDER_COLOR)
    ow.set_hulls(lib, ids)
    for k in range(1, 241):
        w.step(DT)
        ow.step(DT)
        assert stats_tuple(w.stats()) == ow.stats(), k
        if k % 20 == 0:
            compare(w, ow)
    assert (w.manifolds()[:, 1] == 0xFFFFFFFE).any()


def test_rubble_6000_on_a_cluster_against_oracle(sf, oracle):
    """6,000 boxes and cells (a cluster scene) for 30 steps at 12 sub-steps without sleep, bit-exact."""
    from test_oracle_boxes import rubble
    recs, lib, ids = rubble(6000, seed=5)
    p = X.box_params(allow_sleep=0)
    w = X.BoxWorld(recs, p)
    w.set_hulls(lib, ids)
    ow = oracle.OracleBoxWorld(recs, p, oracle.ORDER_COLOR)
    ow.set_hulls(lib, ids)
    for k in range(30):
        w.step(DT)
        ow.step(DT)
        assert stats_tuple(w.stats()) == ow.stats(), k
    compare(w, ow)


def test_capacity_refusal_leaves_the_other_scenes_stepping(sf, oracle):
    """A scene whose box covers millions of grid cells (half extents of 100 m) is past the grid's capacity: each step
    returns SF_ERR_CAPACITY with that scene's status flag set and the scene left as it was, while the other scene steps
    exactly as its oracle."""
    giant = np.array([[0.0, 101.0, 0.0, 0, 0, 0, 1, 100.0, 100.0, 100.0, 1.0]], np.float32)
    stk = X.stack(20)
    p = X.box_params()
    w = X.BoxWorld([stk, giant], p)
    ow = oracle.OracleBoxWorld(stk, p, oracle.ORDER_COLOR)
    before = w.state(1).copy()
    for _ in range(30):
        with pytest.raises(sf.SfError) as e:
            w.step(DT)
        assert e.value.status == sf.SF_ERR_CAPACITY
        ow.step(DT)
    assert w.stats(1).status == 1
    np.testing.assert_array_equal(w.state(1), before)
    compare(w, ow, scene=0)

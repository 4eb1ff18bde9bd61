"""The box world's oracle (the engine crate's World::step, engine/src/phys.rs:152-354, restated in
oracle/sf_oracle.cpp) pinned by the reference's own published results, then the colour order the GPU uses checked
against the same bars:

  * the 20-box stack gate (engine/src/phys.rs:673-684): the reference reports 6.93 mm of top drift and 1.7 mm/s of
    peak speed in the last second, without sleep, at 12 sub-steps (docs/GPU.md:156, docs/PHASE0.md:11); the list-order
    restatement gives the same to the printed digits;
  * the 2,000-box pile after 2 s at 4 sub-steps without sleep (gpu/test_gpu.cjs:1049-1062): the reference's CPU world
    spans y 0.117-4.828 m (docs/GPU.md:158); the list order gives the same, and the colour order stays within the
    reference's own GPU-against-CPU tolerance (0.02 m low, 0.1 m high);
  * `single_box_rests`, `tilted_stack_falls_and_settles` (engine/src/phys.rs:664-697) in both orders;
  * the colouring is proper and both orders build the same manifolds from the same state.
"""
import numpy as np
import pytest

from shatterforge_b200 import boxes as X

DT = np.float32(1.0 / 60.0)


def run_stack(oracle, order, sleep, steps=600):
    ow = oracle.OracleBoxWorld(X.stack(20), X.box_params(allow_sleep=sleep), order)
    top0 = X.stack(20)[19, 1]
    maxv = 0.0
    for f in range(steps):
        ow.step(DT)
        if f >= 540:
            v = ow.state()[:, 7:10].astype(np.float64)
            maxv = max(maxv, float(np.sqrt((v * v).sum(1)).max()))
    d = ow.state()[19, :3].astype(np.float64) - np.array([0.0, top0, 0.0])
    return float(np.sqrt((d * d).sum())), maxv, ow


def test_stack_gate_matches_the_published_figures(oracle):
    drift, maxv, _ = run_stack(oracle, oracle.ORDER_LIST, 0)
    assert round(drift * 1e3, 2) == 6.93, drift
    assert round(maxv * 1e3, 1) == 1.7, maxv
    drift, maxv, ow = run_stack(oracle, oracle.ORDER_LIST, 1)
    assert drift < 0.01 and maxv < 0.01
    assert ow.state()[:, 21].sum() == 0          # asleep after settling


@pytest.mark.parametrize("order", [0, 1])
def test_stack_gate_in_both_orders(oracle, order):
    for sleep in (0, 1):
        drift, maxv, _ = run_stack(oracle, order, sleep)
        assert drift < 0.01 and maxv < 0.01, (order, sleep, drift, maxv)


def pile_range(oracle, order, n=2000, steps=120):
    ow = oracle.OracleBoxWorld(X.pile(n), X.box_params(allow_sleep=0, substeps=4), order)
    ow.step(DT, steps)
    y = ow.state()[:, 1]
    assert np.isfinite(ow.state()).all()
    return float(y.min()), float(y.max())


def test_pile_matches_the_published_range(oracle):
    lo, hi = pile_range(oracle, oracle.ORDER_LIST)
    assert (round(lo, 3), round(hi, 3)) == (0.117, 4.828), (lo, hi)
    clo, chi = pile_range(oracle, oracle.ORDER_COLOR)
    assert abs(clo - lo) < 0.02 and abs(chi - hi) < 0.1, (clo, chi, lo, hi)


@pytest.mark.parametrize("order", [0, 1])
def test_single_box_rests(oracle, order):
    ow = oracle.OracleBoxWorld(X.tilted_box(), X.box_params(), order)
    ow.step(DT, 300)
    s = ow.state()[0]
    assert 0.1 < s[1] < 0.3 and np.linalg.norm(s[7:10]) < 0.01
    assert abs(s[1] - 0.125) < 0.005                   # flat on its smallest half extent (docs/GPU.md:154)


@pytest.mark.parametrize("order", [0, 1])
def test_offset_column_topples_and_settles(oracle, order):
    ow = oracle.OracleBoxWorld(X.offset_column(), X.box_params(), order)
    ow.step(DT, 600)
    s = ow.state()
    assert s[:, 1].max() < 3.0 and s[:, 1].min() > 0.2
    assert (np.linalg.norm(s[:, 7:10], axis=1) < 0.05).all()


def test_colouring_is_proper_and_orders_agree(oracle):
    """From the same state both orders find the same manifolds (pairs, points, normals); in the colour order no two
    manifolds of a colour share a moving body, and a manifold's colour is the smallest its higher-priority
    neighbours left free."""
    a = oracle.OracleBoxWorld(X.pile(2000), X.box_params(allow_sleep=0, substeps=4), oracle.ORDER_LIST)
    b = oracle.OracleBoxWorld(X.pile(2000), X.box_params(allow_sleep=0, substeps=4), oracle.ORDER_COLOR)
    a.step(DT, 40)
    b.step(DT, 40)      # the orders drift apart; take one more step of each from its own state and check structure
    a.step(DT)
    b.step(DT)
    ma, mb = a.manifolds(), b.manifolds()
    assert a.stats()[1] > 2000 and b.stats()[2] == len(mb)
    keys = mb[:, 0].astype(np.uint64) << np.uint64(32) | mb[:, 1].astype(np.uint64)
    assert (np.diff(keys.astype(np.float64)) > 0).all()          # key order, no duplicates
    awake = b.state()[:, 21] > 0
    col = mb[:, 14]
    for c in np.unique(col):
        sel = mb[col == c]
        bodies = np.concatenate([sel[:, 0], sel[sel[:, 1] != 0xFFFFFFFF, 1]])
        assert len(np.unique(bodies)) == len(bodies), c        # every body here was moving during the step
    assert b.stats()[4] == col.max() + 1
    # the same manifold set from one state: a fresh pile's first step
    a = oracle.OracleBoxWorld(X.pile(2000), X.box_params(allow_sleep=0, substeps=4), oracle.ORDER_LIST)
    b = oracle.OracleBoxWorld(X.pile(2000), X.box_params(allow_sleep=0, substeps=4), oracle.ORDER_COLOR)
    a.step(DT)
    b.step(DT)
    ma, mb = a.manifolds(), b.manifolds()
    order = np.lexsort((ma[:, 1], ma[:, 0]))
    cols = [0, 1, 2, 4, 5, 6]                  # pair, count, normal (sticking depends on the solve order)
    np.testing.assert_array_equal(ma[order][:, cols], mb[:, cols])
    assert a.stats()[:4] == b.stats()[:4]
    assert awake.any()


def quat_rot(q):
    x, y, z, w = [float(v) for v in q]
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def rubble(n, seed=3, box_every=5):
    """The reference's pile with most boxes replaced by convex cells of the hull library (every fifth a plain box)."""
    from shatterforge_b200 import hulls
    lib = hulls.library().packed()
    ids = np.random.default_rng(seed).integers(1, len(lib), n).astype(np.uint32)
    ids[::box_every] = 0
    return X.pile(n), lib, ids


@pytest.mark.parametrize("order", [0, 1])
def test_convex_cell_comes_to_rest_on_its_corners(oracle, order):
    """A convex cell dropped tilted from 1 m (the WebGPU world's hull shapes, gpu/gpu_world.js:786-833): after 5 s it
    is at rest with its lowest corner on the ground (within 1 cm), and a cell resting on a face of more than four
    corners has its corners in two ground patches."""
    from shatterforge_b200 import hulls
    lib = hulls.library().packed()
    for cell in (1, 7, 30):
        rec = X.tilted_box()
        ow = oracle.OracleBoxWorld(rec, X.box_params(), order)
        ow.set_hulls(lib, np.array([cell], np.uint32))
        ow.step(DT, 300)
        s = ow.state()[0]
        assert np.linalg.norm(s[7:10]) < 0.05, (cell, s[7:10])
        nv = int(lib[cell, 0, 0])
        verts = lib[cell, 1:1 + nv, :3] * rec[0, 7:10]
        wy = (verts @ quat_rot(s[3:7]).T)[:, 1] + s[1]
        assert abs(wy.min()) < 0.01, (cell, wy.min())


@pytest.mark.parametrize("order", [0, 1])
def test_rubble_pile_settles(oracle, order):
    recs, lib, ids = rubble(500)
    ow = oracle.OracleBoxWorld(recs, X.box_params(), order)
    ow.set_hulls(lib, ids)
    ow.step(DT, 240)
    s = ow.state()
    assert np.isfinite(s).all()
    assert s[:, 1].max() < 2.0 and np.linalg.norm(s[:, 7:10], axis=1).max() < 0.5
    m = ow.manifolds()
    assert (m[:, 1] == 0xFFFFFFFE).any()          # second ground patches of cells lying on a face

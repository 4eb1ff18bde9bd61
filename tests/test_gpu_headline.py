"""Parity at the benchmark's own sizes, through the C ABI.

The benchmark steps the whole 256-scene debris mix in one world and solves all 37 structures of the
structure lattice at once; these tests check those runs against the CPU oracle:

  * the 256-scene mix stepped to its contact peak in one batched world; then one more batched step, compared scene by
    scene (the smallest, the median and the largest, about 20,000 bodies) with the oracle stepping that scene alone
    from the GPU's state: contact lists, manifolds with their colours, islands and body state bit for bit;
  * 60 steps of the median scene from rest, bit for bit against the colour-order oracle;
  * the 5-storey frame with 1,024 loose bricks for 200 steps, past the debris landing on the ground and
    on the frame's roof, bit for bit;
  * the full structure lattice (about 375,000 bricks) solved in one call, each structure against the FP64
    red-black oracle at the same sweep cap: potentials, sweep counts and residuals bit for bit;
  * a long horizon: 300 steps of the median scene with the reference's pinch removal, against the oracle in the
    reference's own list order, by centre-of-mass height and per-material height and fragment-survival histograms.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
STATIC = 0xFFFFFFFF


@pytest.fixture(scope="module")
def mix():
    """The benchmark's mix: 256 scenes, body counts log-uniform in 500-20,000 (seed 3, as bench.py builds it)."""
    return S.debris_mix()


def _by_size(scenes):
    order = np.argsort([s.n_bodies for s in scenes])
    return {"smallest": int(order[0]), "median": int(order[len(order) // 2]), "largest": int(order[-1])}


def _scene_state(w, k):
    st, sl, fl = w.bodies()
    a, b = w.body_off[k], w.body_off[k + 1]
    p = w.brick_positions()
    return st[a:b], sl[a:b], fl[a:b], p[w.brick_off[k]:w.brick_off[k + 1]]


def _local_labels(lab, off):
    out = lab.copy()
    live = lab != STATIC
    out[live] -= np.uint32(off)
    return out


def test_mix_at_contact_peak_one_step_per_scene(sf, oracle, mix):
    """The whole mix, batched as the benchmark runs it (8 iterations, pinch removal off, colouring verified), 110
    steps in (the largest scenes' bodies are landing: the contact peak of the mix); then one more step, each chosen
    scene compared with the oracle stepping that scene alone from the GPU's state."""
    w = sf.World(mix, iterations=8, pinch_kill=0, verify=1)
    w.step(DT, nsteps=110)
    picks = _by_size(mix)
    before = {k: _scene_state(w, k) for k in picks.values()}
    w.step(DT)
    assert w.stats().error_word == 0
    st_all, sl_all, fl_all = w.bodies()
    lab_all = w.islands()
    for name, k in picks.items():
        sc = mix[k]
        st, sl, fl, wp = before[k]
        ow = oracle.OracleWorld(sc)
        ow.set_bodies(st, sl, fl)
        ow.set_brick_positions(wp)
        ow.step(DT, iterations=8, order=oracle.ORDER_COLOR, pinch_kill=0)
        ids, f, s = w.contacts(k)
        oids, of, os_ = ow.contacts()
        assert len(ids) == len(oids), name
        if name == "largest":
            assert len(ids) > 20000, len(ids)     # at the peak: tens of thousands of contacts in this scene
        np.testing.assert_array_equal(ids, oids, err_msg=name)
        np.testing.assert_array_equal(f, of, err_msg=name)
        np.testing.assert_array_equal(s, os_, err_msg=name)
        np.testing.assert_array_equal(w.manifolds(k), ow.manifolds(), err_msg=name)
        a, b = w.body_off[k], w.body_off[k + 1]
        ost, osl, ofl = ow.bodies()
        np.testing.assert_array_equal(fl_all[a:b], ofl, err_msg=name)
        np.testing.assert_array_equal(st_all[a:b], ost, err_msg=name)
        np.testing.assert_array_equal(sl_all[a:b], osl, err_msg=name)
        np.testing.assert_array_equal(_local_labels(lab_all[a:b], a), ow.islands(), err_msg=name)
    w.close()


def test_median_scene_sixty_steps_from_rest(sf, oracle, mix):
    k = _by_size(mix)["median"]
    sc = mix[k]
    w = sf.World(sc, iterations=8, pinch_kill=0)
    ow = oracle.OracleWorld(sc)
    for _ in range(60):
        w.step(DT)
        ow.step(DT, iterations=8, order=oracle.ORDER_COLOR, pinch_kill=0)
    st, sl, fl = w.bodies()
    ost, osl, ofl = ow.bodies()
    np.testing.assert_array_equal(fl, ofl)
    np.testing.assert_array_equal(st, ost)
    np.testing.assert_array_equal(sl, osl)
    ids, f, s = w.contacts()
    oids, of, os_ = ow.contacts()
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(s, os_)
    assert len(ids) > 1000


def test_frame_with_debris_past_landing(sf, oracle):
    """The 5-storey frame with its debris for 200 steps: the loose bricks start 2-12 m up beside the frame and have all landed (on the ground,
    on each other) well before the end; the reference's pinch removal is on, as in the reference."""
    sc = S.frame5_debris_scene()
    w = sf.World(sc, iterations=8)
    ow = oracle.OracleWorld(sc)
    for _ in range(200):
        w.step(DT)
        ow.step(DT, iterations=8, order=oracle.ORDER_COLOR)
    st, sl, fl = w.bodies()
    ost, osl, ofl = ow.bodies()
    np.testing.assert_array_equal(fl, ofl)
    np.testing.assert_array_equal(st, ost)
    np.testing.assert_array_equal(sl, osl)
    alive = (fl & 1) == 1
    assert st[alive, 1].max() < 2.0               # everything that is left has come down (it started 2-12 m up)
    assert ((fl & 3) == 3).sum() > sc.n_bodies // 4  # and much of it is asleep


def test_full_structure_lattice_against_fp64(sf, oracle):
    """All 37 structures (about 375,000 bricks) in one solve (the benchmark's call: one thread-block cluster per
    structure), stopped at 3,000 sweeps or the residual 1e-6; each structure equals the FP64 red-black oracle run
    alone to the same limits, bit for bit."""
    sc = S.structure_lattice(seed=2)
    assert sc.n_static >= 370000 and len(sc.structure_ids()) == 37
    w = sf.World(sc)
    w.structure_solve(-1, omega=1.7, tol=1e-6, max_sweeps=3000)
    assert w.stats().cluster_solves == 1
    sw, rs = w.solve_detail()
    phi = w.phi64()
    ow = oracle.OracleWorld(sc)
    for s in sc.structure_ids():
        osw, ors = ow.sor(s, 1.7, 1e-6, 3000, mode=oracle.MODE_REDBLACK_F64)
        assert sw[s] == osw, (s, sw[s], osw)
        assert rs[s] == ors, (s, rs[s], ors)
    np.testing.assert_array_equal(phi, ow.phi64())


def test_long_horizon_against_reference_order(sf, oracle, mix):
    """300 steps of the median scene (3,623 bodies) with pinch removal on: the GPU (colour order) against the
    oracle in the reference's list order, which differ in impulse order and so diverge bit-wise within a few steps.
    Bounds: centre-of-mass height and each material's mean height within 5 cm, each material's height histogram
    within a total variation distance of 0.08, each fragment size class's surviving fraction within 0.05."""
    k = _by_size(mix)["median"]
    sc = mix[k]
    w = sf.World(sc, iterations=8)
    ow = oracle.OracleWorld(sc)
    for _ in range(300):
        w.step(DT)
        ow.step(DT, iterations=8, order=oracle.ORDER_LIST)
    st, _, fl = w.bodies()
    ost, _, ofl = ow.bodies()
    a, b = S.horizon_stats(sc, st, fl), S.horizon_stats(sc, ost, ofl)
    d = S.horizon_distance(a, b)
    print("long horizon, GPU vs reference order:", d, "alive", a["alive"], b["alive"])
    assert d["com_y"] <= 0.05 and d["mean_y"] <= 0.05
    assert d["height_tv"] <= 0.08
    assert d["survival"] <= 0.05

"""Contact reduction and warm start on the GPU (sf_params.reduce / warm_start: the GPU world's devices for large
contact sets, gpu/gpu_world.js:557-576, 834-920, restated for brick contacts) against the oracle's restatement, bit
for bit: the kept contacts, their manifolds and colours, the warm-started impulses, the world after every step, and
the table starting over after rebuilds and detachments.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S
from test_gpu_connectivity import DT, IT, compare_world
from test_gpu_splitting import compare_bonds
from test_gpu_damage import damage_counts
from test_gpu_bodyload import compare_fields, frame_pair
from test_oracle_reduction import expected_kept, stack

pytestmark = pytest.mark.gpu


def compare_contacts(w, ow, scene=0):
    ids, f, s = w.contacts(scene)
    oids, of, os_ = ow.contacts()
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(f, of)
    np.testing.assert_array_equal(s, os_)
    np.testing.assert_array_equal(w.manifolds(scene), ow.manifolds())


def test_blocks_reduced_against_oracle(sf, oracle):
    """Three 4,000-brick blocks on the ground: each pair's 2,000 contacts reduce to the extremes and the deepest,
    one colour instead of 125; 20 steps (until they sleep) equal the oracle's contacts, manifolds and bodies."""
    sc = S.body_blocks()
    w = sf.World(sc, iterations=IT, reduce=1)
    ow = oracle.OracleWorld(sc)
    for k in range(20):
        w.step(DT)
        ow.step(DT, iterations=IT, reduce=1)
        if k == 0:
            ids, f, s = w.contacts(0)
            keep = expected_kept(ids, f)
            np.testing.assert_array_equal(s[:, 3] != 0.0, keep)
            assert w.stats().colors == 1
        compare_contacts(w, ow)
        compare_world(w, ow)


def test_stack_warm_started_against_oracle(sf, oracle):
    """Six single bricks stacked, one iteration a substep, warm start on: 120 steps, every step's contacts (with the
    warm-started impulses) and bodies equal the oracle's."""
    sc = stack()
    w = sf.World(sc, iterations=1, warm_start=1)
    ow = oracle.OracleWorld(sc)
    for k in range(120):
        w.step(DT)
        ow.step(DT, iterations=1, warm=1)
        compare_contacts(w, ow)
        st, sl, fl = w.bodies()
        ost, osl, ofl = ow.bodies()
        np.testing.assert_array_equal(st, ost)
        np.testing.assert_array_equal(fl, ofl)


def test_compound_debris_reduced_and_warm_against_oracle(sf, oracle):
    """300 compound bodies (1-256 bricks) land and pile up with both on: 150 steps bit-exact, the contacts every 10."""
    sc = S.debris_scene(300, seed=11, kmax=64)
    w = sf.World(sc, iterations=IT, reduce=1, warm_start=1)
    ow = oracle.OracleWorld(sc)
    for k in range(150):
        w.step(DT)
        ow.step(DT, iterations=IT, reduce=1, warm=1)
        if k % 10 == 9:
            compare_contacts(w, ow)
            st, sl, fl = w.bodies()
            ost, osl, ofl = ow.bodies()
            np.testing.assert_array_equal(st, ost)
            np.testing.assert_array_equal(sl, osl)
            np.testing.assert_array_equal(fl, ofl)


def test_beam_landing_warm_table_starts_over_against_oracle(sf, oracle):
    """The beam dropped on one end, warm start and reduction on, with the body frame and the rebuilds its failures
    cause (each rebuild starts the table over): 240 frames, every report and the world at the end equal."""
    sc = S.tilted_beam()
    w = sf.World(sc, iterations=IT, detach_bodies=64, detach_bricks=4000, reduce=1, warm_start=1)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(64, 4000)
    rebuilt = 0
    for f in range(1, 241):
        w.step(DT)
        ow.step(DT, iterations=IT, reduce=1, warm=1)
        rep = w.rebuild_bodies()
        assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == ow.rebuild_bodies(), f
        rebuilt += rep.bodies
        frame_pair(w, ow)
    compare_fields(w, ow)
    compare_world(w, ow)
    compare_bonds(w, ow)
    assert rebuilt > 0


def test_tower_collapse_reduced_and_warm_against_oracle(sf, oracle):
    """The 16-storey tower without eight ground columns in the full frame order, damage on, contact reduction and
    warm start on, and the default limit of 128 colours (without reduction the landing 46,818-brick piece needs
    more): 420 frames, every report equal, the world and the fields at frames 300 and 420."""
    tw, rm = S.tower16_structure()
    sc = tw.without_static(rm)
    ids = sc.structure_ids()
    w = sf.World(sc, iterations=IT, detach_bodies=4000, detach_bricks=60000, damage=1, reduce=1, warm_start=1)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(4000, 60000)
    for s in ids:
        w.structure_warm(s)
        ow.structure_warm(s)
    peak_colors = 0
    for f in range(1, 421):
        w.step(DT)
        ow.step(DT, iterations=IT, damage=1, reduce=1, warm=1)
        peak_colors = max(peak_colors, w.stats().colors)
        damage_counts(w, ow)
        rep = w.rebuild_bodies()
        assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == ow.rebuild_bodies(), f
        r1, _, _ = w.connectivity()
        (p1, d1, _), _, _ = ow.connectivity()
        w.structure_loads(ids)
        ow.structure_loads(ids)
        fr_ = w.structure_frame(f, ids, dt=DT)
        o = ow.structure_frame(f, DT, ids)
        assert (fr_.sweeps, fr_.warm_sweeps, fr_.joints, fr_.failed, fr_.crushed) == (o[0], o[1], o[3], o[5], o[6]), f
        frame_pair(w, ow, fr_.crushed, o[6])
        r2, _, _ = w.connectivity()
        (p2, d2, _), _, _ = ow.connectivity()
        assert (r1.pieces, r1.detached, r2.pieces, r2.detached) == (p1, d1, p2, d2), f
        if f in (300, 420):
            compare_fields(w, ow)
            compare_world(w, ow)
            compare_bonds(w, ow)
    assert peak_colors <= 128


def test_three_scenes_against_their_oracles(sf, oracle):
    """Three scenes in one world with damage, contact reduction and warm start on: the blocks (the body frame's
    budget per scene), the landing beam (failures, crushes, rebuilds, which start only that scene's warm-start
    entries over) and the plough scene (bricks knocked loose from its glass pane into that scene's spare bodies, with
    that scene's draws). Each scene equals its own oracle; the world's reports are the oracles' sums."""
    scenes = [S.body_blocks(), S.tilted_beam(), S.plough_scene()]
    w = sf.World(scenes, iterations=IT, detach_bodies=200, detach_bricks=400, damage=1, reduce=1, warm_start=1,
                 max_colors=256)
    ows = []
    for sc in scenes:
        ow = oracle.OracleWorld(sc)
        ow.set_capacity(200, 400)
        ows.append(ow)
    loose = 0
    for f in range(1, 181):
        w.step(DT)
        for ow in ows:
            ow.step(DT, iterations=IT, damage=1, reduce=1, warm=1)
        r, hit = w.damage()
        oc = [ow.read_damage(plough=True) for ow in ows]
        tot = tuple(sum(c[0][k] for c in oc) for k in range(7))
        assert (r.contacts, r.crushed, r.removed, r.severed, r.cracked, r.ploughed, r.scraped) == tot, f
        np.testing.assert_array_equal(hit, oc[2][1])
        loose += r.ploughed
        rep = w.rebuild_bodies()
        orep = [ow.rebuild_bodies() for ow in ows]
        osum = tuple(sum(x[k] for x in orep) for k in range(5))
        assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == osum, f
        b = w.bodies_frame(DT, 0)
        ob = [ow.body_frame(DT, 0) for ow in ows]
        got = (b.bodies, b.sweeps, b.brick_updates, b.joints, b.over, b.failed, b.crushed, b.crushes_used)
        want = tuple(sum(x[k] for x in ob) for k in (0, 1, 2, 3, 4, 5, 6, 8))
        assert got == want, (f, got, want)
        assert b.max_ratio == max(x[7] for x in ob), f
        if f in (60, 180):
            for k, ow in enumerate(ows):
                compare_world(w, ow, scene=k)
                compare_bonds(w, ow, scene=k)
                compare_fields(w, ow, scene=k)
    assert loose > 10

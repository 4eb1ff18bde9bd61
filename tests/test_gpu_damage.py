"""Damage on contact on the GPU (sf_params.damage: impact_damage / crush_at, src/lib.rs:1602-1702, between the pinch
clamps and integration) against the oracle's restatement, bit for bit, in the reference's frame order: the substeps
with damage, rebuild_body of the marked bodies, connectivity, and for structures the loads and the load-path frame.
Every step's damage counters and the structures a hit woke must match, and the whole world state every few steps.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S
from test_gpu_connectivity import DT, IT, compare_world
from test_gpu_splitting import compare_bonds

pytestmark = pytest.mark.gpu


def damage_counts(w, ow):
    r, hit = w.damage()
    oc, ohit = ow.read_damage(plough=True)
    assert (r.contacts, r.crushed, r.removed, r.severed, r.cracked, r.ploughed, r.scraped) == oc
    np.testing.assert_array_equal(hit, ohit)
    return r


def test_damage_compound_debris_against_oracle(sf, oracle):
    """200 compound bodies (1-64 bricks) fall onto the ground and static obstacles with damage on: landings crush
    bricks of bodies and obstacles, bodies split as they are rebuilt. 120 steps, bit-exact."""
    sc = S.debris_scene(200, seed=21, kmax=64)
    w = sf.World(sc, iterations=IT, detach_bodies=2000, detach_bricks=20000, damage=1)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(2000, 20000)
    crushed = pieces = 0
    for k in range(120):
        w.step(DT)
        ow.step(DT, iterations=IT, damage=1)
        r = damage_counts(w, ow)
        crushed += r.crushed
        rep = w.rebuild_bodies()
        assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == ow.rebuild_bodies(), k
        pieces += rep.pieces
        if k % 10 == 9:
            compare_world(w, ow)
            compare_bonds(w, ow)
    assert crushed > 50 and pieces > 10


def test_damage_debris_on_the_frame_against_oracle(sf, oracle):
    """512 bricks of debris fall beside and onto the 5-storey frame with damage on, frame by frame in the
    reference's order (substeps with damage, rebuild, connectivity, loads, load-path frame, connectivity): every
    frame's damage counters, woken structures, rebuild and walk reports match; the world state every 25 frames."""
    sc = S.frame5_debris_scene(seed=1, n_debris=512)
    ids = sc.structure_ids()
    w = sf.World(sc, iterations=IT, detach_bodies=2000, detach_bricks=20000, damage=1)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(2000, 20000)
    for s in ids:
        w.structure_warm(s)
        ow.structure_warm(s)
    crushed = 0
    for f in range(1, 151):
        w.step(DT)
        ow.step(DT, iterations=IT, damage=1)
        crushed += damage_counts(w, ow).crushed
        rep = w.rebuild_bodies()
        assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == ow.rebuild_bodies(), f
        r1, _, _ = w.connectivity()
        (p1, d1, _), _, _ = ow.connectivity()
        w.structure_loads(ids)
        ow.structure_loads(ids)
        fr_ = w.structure_frame(f, ids, dt=DT)
        o = ow.structure_frame(f, DT, ids)
        assert (fr_.sweeps, fr_.warm_sweeps, fr_.joints, fr_.failed, fr_.crushed) == (o[0], o[1], o[3], o[5], o[6]), f
        r2, _, _ = w.connectivity()
        (p2, d2, _), _, _ = ow.connectivity()
        assert (r1.pieces, r1.detached, r2.pieces, r2.detached) == (p1, d1, p2, d2), f
        if f % 25 == 0:
            compare_world(w, ow)
    assert crushed > 5


def test_tower_collapse_with_damage_against_oracle(sf, oracle):
    """The 16-storey tower (47,760 bricks) with eight ground columns removed, frame by frame in the reference's order
    with damage on: its joints go live, footings fail and are crushed, the tower detaches as a 46,818-brick body
    (frame 254) that then settles, crushing and shedding pieces. 300 frames; every frame's reports match, and the
    whole world (bodies, set-up, brick positions, potentials, static and body bonds) at frames 260, 280 and 300."""
    tw, rm = S.tower16_structure()
    sc = tw.without_static(rm)
    ids = sc.structure_ids()
    w = sf.World(sc, iterations=IT, detach_bodies=4000, detach_bricks=60000, damage=1)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(4000, 60000)
    for s in ids:
        w.structure_warm(s)
        ow.structure_warm(s)
    detached = 0
    for f in range(1, 301):
        w.step(DT)
        ow.step(DT, iterations=IT, damage=1)
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
        r2, now, top = w.connectivity()
        (p2, d2, _), onow, otop = ow.connectivity()
        assert (r1.pieces, r1.detached, r2.pieces, r2.detached) == (p1, d1, p2, d2), f
        detached += r1.detached + r2.detached
        if f in (260, 280, 300):
            compare_world(w, ow)
            compare_bonds(w, ow)
    assert detached > 45000


def test_plough_against_oracle(sf, oracle):
    """plough (src/lib.rs:1493-1550) with damage on: single concrete bricks flying at a glass pane knock panes loose
    as one-brick bodies (spare capacity, the scene's draws for their velocity and spin, the later contacts with them
    switched off), and a 54-brick block driven into a timber wall scrapes it (damage_brick). 120 steps, every step's
    damage counts and structures hit, the world (bodies, set-up, brick positions, static and body bonds) every 10."""
    sc = S.plough_scene()
    w = sf.World(sc, iterations=IT, detach_bodies=200, detach_bricks=400, damage=1)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(200, 400)
    loose = scraped = 0
    for k in range(120):
        w.step(DT)
        ow.step(DT, iterations=IT, damage=1)
        r = damage_counts(w, ow)
        loose += r.ploughed
        scraped += r.scraped
        rep = w.rebuild_bodies()
        assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == ow.rebuild_bodies(), k
        if k % 10 == 9:
            compare_world(w, ow)
            compare_bonds(w, ow)
    assert loose > 10 and scraped > 5


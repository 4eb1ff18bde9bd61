"""The debris-body load field on the GPU (sf_bodies_frame: structural's body part, src/lib.rs:1262-1266, 1282-1365)
against the oracle's restatement, bit for bit: which pieces are swept and how often under the shared budget, their
FP64 potentials and inertial loads, residuals, peak load factors, load times, the judged joints' decisions, ratios
and bonds, the crushes counted on from the structures' pass, and the world after the rebuilds those decisions cause.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S
from test_gpu_connectivity import DT, IT, compare_world
from test_gpu_splitting import compare_bonds
from test_gpu_damage import damage_counts

pytestmark = pytest.mark.gpu


def compare_fields(w, ow, scene=0):
    r = w.scene_ranges(scene)
    b0, nb, k0, nk = r[2], r[6], r[4], r[7]
    phi, ext, resid, nmax, lt, maxr = w.body_fields()
    ophi, oext = ow.body_phi()
    ores, onm, olt, omr = ow.body_state()
    np.testing.assert_array_equal(phi[k0:k0 + nk], ophi)
    np.testing.assert_array_equal(ext[k0:k0 + nk], oext)
    np.testing.assert_array_equal(resid[b0:b0 + nb], ores)
    np.testing.assert_array_equal(nmax[b0:b0 + nb], onm)
    np.testing.assert_array_equal(lt[b0:b0 + nb], olt)
    np.testing.assert_array_equal(maxr[b0:b0 + nb], omr)


def frame_pair(w, ow, crushes=0, ocrushes=0):
    """One body frame on both; the reports must agree."""
    r = w.bodies_frame(DT, crushes)
    o = ow.body_frame(DT, ocrushes)
    got = (r.bodies, r.sweeps, r.brick_updates, r.joints, r.over, r.failed, r.crushed, r.max_ratio, r.crushes_used)
    assert got == o, (got, o)
    return r


def test_blocks_share_the_budget_against_oracle(sf, oracle):
    """Three 4,000-brick blocks land on the ground: the first frame's budget stops the first block at 40 sweeps and
    gives the others 2; 12 frames of fields, joints and settling (every fourth frame by id) agree with the oracle."""
    sc = S.body_blocks()
    w = sf.World(sc, iterations=IT, detach_bodies=16, detach_bricks=16, max_colors=256)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(16, 16)
    for f in range(1, 13):
        w.step(DT)
        ow.step(DT, iterations=IT)
        r = frame_pair(w, ow)
        if f == 1:
            assert (r.bodies, r.sweeps, r.brick_updates, r.judged) == (3, 44, 176000, 3)
        compare_fields(w, ow)
    compare_world(w, ow)


def test_beam_landing_against_oracle(sf, oracle):
    """The 60-brick beam dropped on one end from 30 m: its joints fatigue, fail and crush on landing; the rebuilds
    split it. 240 frames in the reference's order (step, rebuild, body frame), every report equal, and the world,
    body bonds and fields equal at the landing and after."""
    sc = S.tilted_beam()
    w = sf.World(sc, iterations=IT, detach_bodies=64, detach_bricks=4000)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(64, 4000)
    failed = crushed = 0
    for f in range(1, 241):
        w.step(DT)
        ow.step(DT, iterations=IT)
        rep = w.rebuild_bodies()
        assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == ow.rebuild_bodies(), f
        r = frame_pair(w, ow)
        failed += r.failed
        crushed += r.crushed
        if f in (150, 160, 200, 240):
            compare_fields(w, ow)
            compare_world(w, ow)
            compare_bonds(w, ow)
    assert failed > 0 and crushed > 0


def test_crush_budget_counts_on_from_the_structures(sf, oracle):
    """The beam again, told on every frame that the structures' pass used 295 of the frame's 300 crushes: at most 5
    crushes a frame, the rest failures, as the oracle decides them."""
    sc = S.tilted_beam()
    w = sf.World(sc, iterations=IT, detach_bodies=64, detach_bricks=4000)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(64, 4000)
    for f in range(1, 201):
        w.step(DT)
        ow.step(DT, iterations=IT)
        rep = w.rebuild_bodies()
        assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == ow.rebuild_bodies(), f
        r = frame_pair(w, ow, 295, 295)
        assert r.crushed <= 5 and r.crushes_used == 295 + r.crushed
    compare_fields(w, ow)
    compare_world(w, ow)


def test_compound_debris_fields_against_oracle(sf, oracle):
    """300 compound bodies (1-256 bricks) fall and come to rest, damage on: every frame's body pass (loaded pieces,
    sweeps, joints) agrees, and the fields and the world agree every 30 frames."""
    sc = S.debris_scene(300, seed=31, kmax=64)
    w = sf.World(sc, iterations=IT, detach_bodies=2000, detach_bricks=20000, damage=1)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(2000, 20000)
    swept = 0
    for f in range(1, 181):
        w.step(DT)
        ow.step(DT, iterations=IT, damage=1)
        damage_counts(w, ow)
        rep = w.rebuild_bodies()
        assert (rep.bodies, rep.pieces, rep.removed, rep.dissolved, rep.lone) == ow.rebuild_bodies(), f
        swept += frame_pair(w, ow).bodies
        if f % 30 == 0:
            compare_fields(w, ow)
            compare_world(w, ow)
            compare_bonds(w, ow)
    assert swept > 150


def test_tower_collapse_with_body_joints_against_oracle(sf, oracle):
    """The 16-storey tower without eight ground columns, in the reference's full frame order with damage on: step,
    rebuild, connectivity, loads, structure frame, body frame (its crush budget counted on from the structure
    frame's), connectivity. The tower detaches as one 46,818-brick piece; its field (cut by the budget to 4 sweeps a
    frame) and its joints decide failures and crushes that break it up as it lands. 420 frames, every report equal,
    the whole world and the fields at frames 300, 360 and 420."""
    tw, rm = S.tower16_structure()
    sc = tw.without_static(rm)
    ids = sc.structure_ids()
    w = sf.World(sc, iterations=IT, detach_bodies=4000, detach_bricks=60000, damage=1, max_colors=1024)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(4000, 60000)
    for s in ids:
        w.structure_warm(s)
        ow.structure_warm(s)
    failed = crushed = 0
    for f in range(1, 421):
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
        r = frame_pair(w, ow, fr_.crushed, o[6])
        failed += r.failed
        crushed += r.crushed
        r2, _, _ = w.connectivity()
        (p2, d2, _), _, _ = ow.connectivity()
        assert (r1.pieces, r1.detached, r2.pieces, r2.detached) == (p1, d1, p2, d2), f
        if f in (300, 360, 420):
            compare_fields(w, ow)
            compare_world(w, ow)
            compare_bonds(w, ow)
    assert failed > 50 and crushed > 10

"""Damage on contact (crush_at / impact_damage, src/lib.rs:1602-1702) in the CPU oracle, against answers that follow
from the reference's rules:

  * crush_at spends EB per brick on the bricks nearest the point, starting at the hit brick and growing through
    intact bonds (ties go to the first queued, the +x neighbour before the -x one); the brick it cannot afford is
    cracked: damage_brick weakens its bonds by 0.6 e_left / EB of their capacity;
  * each crushed brick is ground away when the draw (h01 of the fixed seed and the draw count, src/lib.rs:341-345)
    is below PULV of its material, else severed (its bonds zeroed); either way its structure is pending;
  * below 0.15 EB nothing happens;
  * in a step, the bricks crushed per substep never exceed the budget of 2,500, and crushed = ground + severed.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S

EB_CONC = 15000.0
PULV_CONC = 0.7
CAPH_CONC = 12000.0
SEED = 0x243F6A88


def h01(h, k):
    """h01 (src/lib.rs:341-345) in 32-bit arithmetic."""
    m = 0xFFFFFFFF
    x = (h + k * 0x9E3779B9) & m
    x ^= x >> 16
    x = (x * 0x7feb352d) & m
    x ^= x >> 15
    x = (x * 0x846ca68b) & m
    x ^= x >> 16
    return np.float32(x >> 8) / np.float32(16777216.0)


def row_scene(n=5, y=5):
    xyz = np.array([[S.ORIGIN[0] + x, y, S.ORIGIN[2]] for x in range(n)], np.int32)
    return S.Scene(xyz, np.full(n, S.CONC, np.uint8), np.zeros(n, np.int32), np.zeros(n, np.uint8)).contiguous()


def centre(x, y, z=0):
    return (x * 0.5 + 0.25, y * 0.5 + 0.25, z * 0.5 + 0.25)


def test_crush_spends_eb_per_brick_and_cracks_the_next(oracle):
    sc = row_scene()
    ow = oracle.OracleWorld(sc)
    b0, _ = ow.bonds()
    crushed = ow.crush_at(2, 2 * EB_CONC + 10000.0, centre(2, 5))
    assert crushed == 2
    b, _ = ow.bonds()
    # brick 2 first, then its +x neighbour 3 (a tie with -x, which was queued second); brick 1 is cracked by
    # 0.6 * 10000 / 15000 = 0.4 of each bond's capacity: its own +x bond and brick 0's +x bond (which joins 0 and 1)
    f = np.float32(0.6) * np.float32(10000.0) / np.float32(EB_CONC)
    expect = np.float32(CAPH_CONC) - (np.float32(CAPH_CONC) * f + np.float32(0.0))
    assert b[0, 0] == expect
    # the crushed bricks: ground away or severed by the first two draws
    for k, brick in enumerate((2, 3)):
        ground = h01(SEED, k) < np.float32(PULV_CONC)
        if not ground:
            assert (b[brick] == 0).all()
    (cand, cr, removed, severed, cracked), _ = ow.read_damage()
    assert cr == 2 and removed + severed == 2 and cracked == 1
    assert ow.pending()[0] == 1


def test_too_little_energy_does_nothing(oracle):
    ow = oracle.OracleWorld(row_scene())
    b0, _ = ow.bonds()
    assert ow.crush_at(2, 0.15 * EB_CONC - 1.0, centre(2, 5)) == 0
    b, _ = ow.bonds()
    np.testing.assert_array_equal(b, b0)
    assert ow.pending()[0] == 0


def test_crush_grows_through_bonds_only(oracle):
    """A gap in the row (no bond across it) stops the growth: with energy for five bricks only the two bricks of
    the hit piece are crushed."""
    xyz = np.array([[S.ORIGIN[0] + x, 5, S.ORIGIN[2]] for x in (0, 1, 3, 4, 5)], np.int32)
    sc = S.Scene(xyz, np.full(5, S.CONC, np.uint8), np.zeros(5, np.int32), np.zeros(5, np.uint8)).contiguous()
    ow = oracle.OracleWorld(sc)
    assert ow.crush_at(0, 5 * EB_CONC + 1.0, centre(0, 5)) == 2


def test_damage_in_steps_respects_the_budget(oracle):
    """Compound debris falling with damage on: per substep at most 2,500 bricks are crushed, every crushed brick is
    ground or severed, and the marked bodies split when rebuilt."""
    sc = S.debris_scene(200, seed=21, kmax=64)
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(2000, 20000)
    crushed = pieces = 0
    for _ in range(120):
        ow.step(1.0 / 60.0, iterations=8, damage=1)
        (cand, cr, removed, severed, cracked), _ = ow.read_damage()
        assert cr <= 2 * 2500 and cr == removed + severed
        crushed += cr
        pieces += ow.rebuild_bodies()[1]
    assert crushed > 50 and pieces > 10


def run_plough(oracle, spare_bodies=200, steps=40):
    sc = S.plough_scene()
    ow = oracle.OracleWorld(sc)
    ow.set_capacity(spare_bodies, 2 * spare_bodies)   # spare bodies and bricks, as sf_params.detach_*
    loose = scraped = 0
    hits = np.zeros(2, np.uint8)
    for _ in range(steps):
        ow.step(1.0 / 60.0, iterations=8, damage=1)
        (cand, cr, removed, severed, cracked, lo, sc_), h = ow.read_damage(plough=True)
        loose += lo
        scraped += sc_
        hits |= h
    return sc, ow, loose, scraped, hits


def test_plough_knocks_glass_loose_and_scrapes_timber(oracle):
    """plough (src/lib.rs:1493-1550): concrete bricks flying at 8 m/s into a glass pane (momentum 300 kg x 8 m/s
    against 0.35 x 1,500) knock panes loose as one-brick glass bodies; the 54-brick block (more than 40 bricks) at
    8 m/s into timber (0.35 x 9,000) damages the bricks it hits instead. Both structures are hit and pending."""
    sc, ow, loose, scraped, hits = run_plough(oracle)
    assert loose > 10 and scraped > 5
    assert hits.all()
    assert ow.nb == sc.n_bodies + loose
    assert (ow.pending()[:2] == 1).all()
    st, _, fl = ow.bodies()
    assert (fl[sc.n_bodies:] & 1).all()               # the loosened panes are live bodies


def test_plough_needs_a_spare_body(oracle):
    """Without spare capacity nothing is knocked loose (ensure_bodies fails: the contact stays on and is solved),
    while the block still scrapes the timber."""
    sc, ow, loose, scraped, hits = run_plough(oracle, spare_bodies=0)
    assert loose == 0 and scraped > 5
    assert ow.nb == sc.n_bodies

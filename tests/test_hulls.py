"""The hull library (gpu/gpu_world.js:2112-2209, engine/src/hull.rs:83-149) and the convex-cell SAT.

Pins from the reference's own tests: gpu/test_hulls.cjs and engine/src/hull.rs:238 — 63 cells in 16 patterns, and
the cells of every pattern tile the cube (their volumes add up to it).
"""
import numpy as np
import pytest

from shatterforge_b200 import hulls


@pytest.fixture(scope="module")
def lib():
    return hulls.library()


def test_library_has_the_reference_cell_count(lib):
    assert len(lib.patterns) == 16
    assert len(lib) == 63
    assert [len(p) for p in lib.patterns] == [2 + (k % 5) for k in range(16)]


def test_patterns_tile_the_cube(lib):
    for p in lib.patterns:
        assert abs(sum(lib.cells[c]["vol"] for c in p) - 1.0) < 1e-9


def test_cells_respect_the_gpu_limits(lib):
    for c in lib.cells:
        assert len(c["V"]) <= 16 and len(c["faces"]) <= 12 and len(c["seg"]) <= 24 and len(c["dirs"]) <= 12
        assert all(len(f) <= 8 for _, _, f in c["faces"])
        # every vertex inside every face plane (box coordinates)
        for v in c["V"]:
            for n, d, _ in c["faces"]:
                assert np.dot(n, v) <= d + 1e-6


def test_packed_layout(lib):
    d = lib.packed()
    assert d.shape == (63, 80, 4)
    assert tuple(d[0, 0]) == (8, 6, 12, 3)          # the cube: 8 vertices, 6 faces, 12 edges, 3 directions
    for i, c in enumerate(lib.cells):
        assert int(d[i, 0, 1]) == len(c["faces"])
        assert sum(int(d[i, 77 + k // 4, k % 4]) for k in range(12)) == sum(len(f) for _, _, f in c["faces"])


def _shape(p, q, h, t):
    return np.array(list(p) + list(q) + list(h) + [t], np.float32)


def test_oracle_stacked_cubes_face_contact(oracle, lib):
    data = lib.packed()
    a = _shape((0, 0, 0), (0, 0, 0, 1), (0.5, 0.5, 0.5), 0)
    b = _shape((0, 0.99, 0), (0, 0, 0, 1), (0.5, 0.5, 0.5), 0)
    n, nrm, pts = oracle.collide_hulls(data, a, b, margin=0.02)
    assert n == 4
    np.testing.assert_allclose(nrm, [0, 1, 0], atol=1e-6)
    np.testing.assert_allclose(pts[:, 3], -0.01, atol=1e-5)
    g = _shape((0, 0, 0), (0, 0, 0, 1), (0.5, 0.5, 0.5), -1)
    n2, nrm2, pts2 = oracle.collide_hulls(data, _shape((0, 0.49, 0), (0, 0, 0, 1), (0.5, 0.5, 0.5), 0), g, margin=0.02)
    assert n2 == 4 and nrm2[1] == -1.0
    np.testing.assert_allclose(pts2[:, 3], -0.01, atol=1e-5)


def test_oracle_hull_matches_box_sat_on_cubes(oracle, lib):
    """Hull 0 is the cube: on separated and touching box pairs the two narrow phases agree on contact or none."""
    rng = np.random.default_rng(4)
    data = lib.packed()
    agree = 0
    for _ in range(200):
        pa = rng.uniform(-0.4, 0.4, 3); pb = rng.uniform(-0.4, 0.4, 3) + np.array([0, 0.9, 0])
        qa = rng.normal(size=4); qa /= np.linalg.norm(qa)
        qb = rng.normal(size=4); qb /= np.linalg.norm(qb)
        h = (0.3, 0.3, 0.3)
        nh, _, _ = oracle.collide_hulls(data, _shape(pa, qa, h, 0), _shape(pb, qb, h, 0), margin=0.02)
        nb, _, _ = oracle.collide_boxes(np.array(list(pa) + list(qa) + list(h), np.float32),
                                        np.array(list(pb) + list(qb) + list(h), np.float32), margin=0.02)
        agree += (nh > 0) == (nb > 0)
    assert agree >= 195

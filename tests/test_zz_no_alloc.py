"""The scratch-free load-path solve (sf_structure_solve_static) against the regular one.

Some callers cannot allocate GPU memory — a host engine that owns the device and gives this library no allocator,
or a frame loop that must not allocate while it runs. sf_structure_solve_static serves them from a fixed static
device array. These tests call it through the C ABI twice in a row (the array keeps the previous call's contents,
so the second call shows that everything which must start at zero is cleared) and compare each result with
sf_world_create + sf_structure_solve on the same bricks, bit for bit, as the parity tests compare potentials.
This file runs last so that a failure here stops nothing else.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S

pytestmark = pytest.mark.gpu


def frame(seed, storeys, w, with_glass=False):
    rng = np.random.default_rng(seed)
    x0, z0 = S.ORIGIN[0] - w // 2, S.ORIGIN[2] - w // 2
    cols = sorted({0, w // 2, w - 1})

    def mats(xyz):
        m = np.full(len(xyz), S.CONC, np.uint8)
        m[rng.random(len(xyz)) < 0.3] = S.MASON
        if with_glass:
            m[(xyz[:, 1] % 6 == 3) & (rng.random(len(xyz)) < 0.2)] = S.GLASS
        return m

    xyz, mat, sid, inf = S.frame_structure(x0, z0, w, w, storeys, 6, cols, cols, 0, mats)
    keep = S.grounded_mask(xyz, mat, sid, inf)
    xyz, mat, sid, inf = xyz[keep], mat[keep], sid[keep], inf[keep]
    ext = (rng.random(len(xyz)) * 50.0).astype(np.float32)
    return S.Scene(xyz, mat, sid, inf).contiguous(), ext


def solve_in_world(sf, sc, ext, omega, tol):
    w = sf.World(sc)
    w.set_ext(ext)
    rep = w.structure_solve(0, omega=omega, tol=tol, max_sweeps=50000)
    sw, rs = w.solve_detail()
    phi = w.phi64()
    w.close()
    return phi, int(sw[0]), float(rs[0]), rep


def test_static_solve_matches_world_solve_twice(sf):
    cases = [frame(1, 3, 14), frame(2, 4, 12, with_glass=True)]
    for sc, ext in cases:   # two calls in a row: the second reuses the array the first left behind
        assert sc.n_static <= sf.STATIC_MAX_BRICKS
        phi, sweeps, resid = sf.structure_solve_static(sc.static_xyz, sc.static_mat, sc.static_infill, ext,
                                                       omega=1.7, tol=1e-6, max_sweeps=50000)
        ref_phi, ref_sweeps, ref_resid, _ = solve_in_world(sf, sc, ext, 1.7, 1e-6)
        assert sweeps == ref_sweeps and sweeps > 10
        assert resid == ref_resid and resid < 1e-6
        np.testing.assert_array_equal(phi, ref_phi)


def test_static_solve_rejects_oversize(sf):
    n = sf.STATIC_MAX_BRICKS + 1
    xyz = np.array([[(k % 600) + 10, (k // 600) % 100, 300 + k // 60000] for k in range(n)], np.int32)
    with pytest.raises(sf.SfError) as e:
        sf.structure_solve_static(xyz, np.full(n, S.CONC, np.uint8))
    assert e.value.status == sf.SF_ERR_CAPACITY
    # few bricks, but one per chunk: more chunks than the array holds
    m = sf.STATIC_MAX_CHUNKS + 8
    xyz = np.array([[8 * (k % 70) + 3, 0, 8 * (k // 70) + 3] for k in range(m)], np.int32)
    with pytest.raises(sf.SfError) as e:
        sf.structure_solve_static(xyz, np.full(m, S.CONC, np.uint8))
    assert e.value.status == sf.SF_ERR_CAPACITY
    # and the entry point still works afterwards
    sc, ext = frame(3, 2, 10)
    phi, sweeps, resid = sf.structure_solve_static(sc.static_xyz, sc.static_mat, sc.static_infill, ext)
    ref_phi, ref_sweeps, _, _ = solve_in_world(sf, sc, ext, 1.7, 1e-6)
    assert sweeps == ref_sweeps
    np.testing.assert_array_equal(phi, ref_phi)


def test_static_solve_equals_fp64_oracle(sf, oracle):
    """On its own: the scratch-free solve equals the FP64 red-black oracle at the same residual, bit for bit."""
    sc, ext = frame(4, 3, 12)
    phi, sweeps, resid = sf.structure_solve_static(sc.static_xyz, sc.static_mat, sc.static_infill, ext,
                                                   omega=1.7, tol=1e-6, max_sweeps=50000)
    ow = oracle.OracleWorld(sc)
    ow.set_ext(ext)
    osw, ors = ow.sor(0, 1.7, 1e-6, 50000, mode=oracle.MODE_REDBLACK_F64)
    assert sweeps == osw and resid == ors
    np.testing.assert_array_equal(phi, ow.phi64())


@pytest.mark.parametrize("bad", ["outside", "duplicate", "material"])
def test_static_solve_rejects_bad_bricks_then_works(sf, bad):
    """The device-side input checks: a brick outside the lattice, two bricks in one cell, a material outside 1..8
    each return SF_ERR_ARG; the next call with good bricks gives the regular solve's result."""
    sc, ext = frame(5, 2, 10)
    xyz, mat = sc.static_xyz.copy(), sc.static_mat.copy()
    if bad == "outside":
        xyz[7] = [640, 3, 300]
    elif bad == "duplicate":
        xyz[9] = xyz[4]
    else:
        mat[11] = 9
    with pytest.raises(sf.SfError) as e:
        sf.structure_solve_static(xyz, mat, sc.static_infill, ext)
    assert e.value.status == sf.SF_ERR_ARG
    with pytest.raises(ValueError):
        sf.structure_solve_static(sc.static_xyz, sc.static_mat[:-1], sc.static_infill, ext)
    phi, sweeps, resid = sf.structure_solve_static(sc.static_xyz, sc.static_mat, sc.static_infill, ext)
    ref_phi, ref_sweeps, ref_resid, _ = solve_in_world(sf, sc, ext, 1.7, 1e-6)
    assert sweeps == ref_sweeps and resid == ref_resid
    np.testing.assert_array_equal(phi, ref_phi)

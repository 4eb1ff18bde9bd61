"""The C-ABI library loads and exports every function include/sf.h declares; host-side logic without a GPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(sf_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("sf_world_create", "sf_world_step", "sf_structure_solve", "sf_structure_check", "sf_read_contacts",
                 "sf_read_islands", "sf_read_phi", "sf_collide_boxes"):
        assert must in names


def test_library_exports_every_declared_symbol(sf):
    lib = sf.load()
    names = declared_functions()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding knows the prototype of each
    assert names <= set(sf.PROTOTYPES), names - set(sf.PROTOTYPES)


def test_params_default_matches_reference(sf):
    p = sf.default_params()
    assert p.substeps == 2 and p.iterations == 10 and p.pinch_kill == 1 and p.sleep_mode == sf.SF_SLEEP_BODY


def test_status_strings(sf):
    lib = sf.load()
    assert lib.sf_status_string(0) == b"ok"
    assert b"timed out" in lib.sf_status_string(4)


def test_no_device_fails_loudly(sf):
    """Without a CUDA device the library refuses to build a world; nothing falls back to a CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from shatterforge_b200 import scenes as S
    sc, _ = S.frame5_structure()
    with pytest.raises(sf.SfError) as e:
        sf.World(sc)
    assert e.value.status == sf.SF_ERR_CUDA


def test_generators_shapes():
    from shatterforge_b200 import scenes as S
    sc, rm = S.frame5_structure()
    assert sc.n_static == 3150 and rm.sum() == 12
    c1 = S.frame5_debris_scene()
    assert c1.n_bodies == 1024 and c1.n_body_bricks == 1024
    d = S.debris_scene(500, seed=7)
    assert d.n_bodies == 500 and d.body_first[-1] == d.n_body_bricks
    assert d.n_static > 0 and (d.static_sid == -1).all()
    t, trm = S.tower16_structure()
    assert t.n_static == 47808 and trm.sum() == 48
    assert (t.static_infill == (t.static_mat == S.GLASS)).all() and t.static_infill.sum() == 16 * 534
    t2 = t.without_static(trm)
    assert S.grounded_mask(t2.static_xyz, t2.static_mat, t2.static_sid, t2.static_infill).all()
    c2 = S.tower16_debris_scene(n_bodies=600)
    ks = np.diff(c2.body_first.astype(np.int64))
    assert c2.n_bodies == 600 and ks.min() >= 1 and ks.max() <= 512 and ks.max() >= 128
    # the structure lattice: 37 frames, about 378,000 bricks after ungrounded pieces are pruned (none should be),
    # glass only as window panels standing on slabs
    lat = S.structure_lattice(seed=2)
    assert len(lat.structure_ids()) == 37 and 370000 <= lat.n_static <= 390000
    glass = lat.static_mat == S.GLASS
    assert 0.03 < glass.mean() < 0.06 and (lat.static_infill[glass] == 1).all()


def test_xorshift_matches_reference_stream():
    from shatterforge_b200.scenes import XorShift32
    r = XorShift32(0x9E3779B9)
    # x ^= x << 13; x ^= x >> 17; x ^= x << 5 (src/lib.rs:324-329), computed by hand for the first value
    x = 0x9E3779B9
    x ^= (x << 13) & 0xFFFFFFFF; x ^= x >> 17; x ^= (x << 5) & 0xFFFFFFFF
    assert r.u32() == x


def test_grounded_mask_drops_floating_pieces():
    from shatterforge_b200 import scenes as S
    xyz = np.array([[10, 0, 10], [10, 1, 10], [20, 5, 20], [21, 5, 20]], np.int32)
    mat = np.full(4, S.CONC, np.uint8)
    keep = S.grounded_mask(xyz, mat, np.zeros(4, np.int32), np.zeros(4, np.uint8))
    assert keep.tolist() == [True, True, False, False]


def test_box_world_rejects_bad_arguments(sf):
    """sf_box_world_create checks its arguments before it touches a device: null pointers, scene bounds that go
    down or do not start at 0, and a non-positive cell give SF_ERR_ARG."""
    import ctypes as C
    from shatterforge_b200 import boxes as X
    lib = sf.load()
    h = C.c_void_p()
    p = X.box_params()
    recs = X.stack(4)
    rp = recs.ctypes.data_as(C.POINTER(C.c_float))
    assert lib.sf_box_world_create(None, None, 1, C.byref(p), C.byref(h)) == sf.SF_ERR_ARG
    for first in ([0, 4, 2], [1, 4]):
        f = np.array(first, np.uint32)
        assert lib.sf_box_world_create(rp, f.ctypes.data_as(C.POINTER(C.c_uint32)), len(first) - 1, C.byref(p),
                                       C.byref(h)) == sf.SF_ERR_ARG
    bad = X.box_params(cell=0.0)
    f = np.array([0, 4], np.uint32)
    assert lib.sf_box_world_create(rp, f.ctypes.data_as(C.POINTER(C.c_uint32)), 1, C.byref(bad), C.byref(h)) == sf.SF_ERR_ARG
    assert lib.sf_box_world_step(None, 1.0 / 60.0, 1) == sf.SF_ERR_ARG

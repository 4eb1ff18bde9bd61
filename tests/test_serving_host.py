"""Host-side logic of the scene pools and the server, without a GPU: the slot a scene needs, the device bytes a
pool's slots take (the number admission by budget is made on), the bytes of a saved scene, and that a pool refuses
to come up without a device instead of falling back to anything.
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S


@pytest.fixture(scope="module")
def sv():
    from shatterforge_b200 import serving
    return serving


def _chunks(xyz):
    return len({(int(x) >> 3, int(y) >> 3, int(z) >> 3) for x, y, z in xyz})


def test_slot_for_counts_the_scene(sv):
    sc = S.debris_scene(90, seed=3, obstacles=(2, 4), spacing=1.3, p_geom=0.4, kmax=8)
    b, k, st, ch = sv.slot_for(sc)
    assert (b, k, st) == (sc.n_bodies, sc.n_body_bricks, sc.n_static)
    assert ch == _chunks(sc.static_xyz)
    # headroom rounds every count up
    b2, k2, st2, ch2 = sv.slot_for(sc, 1.25)
    assert b2 == int(np.ceil(sc.n_bodies * 1.25)) and k2 == int(np.ceil(sc.n_body_bricks * 1.25))
    assert st2 == int(np.ceil(sc.n_static * 1.25)) and ch2 == int(np.ceil(ch * 1.25))


def test_slot_for_a_scene_without_statics_or_bodies(sv):
    sc = S.Scene()
    assert sv.slot_for(sc) == (1, 1, 0, 0)


def test_pool_bytes_add_up_over_slots(sv):
    a, b = (1000, 4000, 2000, 30), (50, 200, 0, 0)
    ba, bb = sv.pool_bytes([a]), sv.pool_bytes([b])
    assert ba > 0 and bb > 0
    assert sv.pool_bytes([a, b]) == ba + bb
    assert sv.pool_bytes([a, a, a]) == 3 * ba
    assert sv.pool_bytes([]) == 0
    # more of anything costs more
    for i in range(4):
        bigger = list(a)
        bigger[i] += 100
        assert sv.pool_bytes([tuple(bigger)]) > ba


def test_snapshot_bytes_grow_with_the_scene(sf):
    f = sf.load().sf_pool_snapshot_bytes
    assert f(10, 40) > 0
    assert f(20, 40) > f(10, 40) and f(10, 80) > f(10, 40)


def test_pool_without_device_fails_loudly(sf, sv):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    sc = S.debris_scene(40, seed=4, obstacles=(2, 3), spacing=1.3, p_geom=0.4, kmax=6)
    with pytest.raises(sf.SfError) as e:
        sv.ScenePool([sv.slot_for(sc)])
    assert e.value.status == sf.SF_ERR_CUDA

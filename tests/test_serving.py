"""Scene pools and the request server: every result equals the same work done alone.

Pool: a scene stepped in a slot among other loaded scenes, saved, evicted and restored into another slot ends
bit-exact where the scene stepped alone ends. Server: a random arrival stream of scene-step and structure-solve
requests, served with continuous batching (and with batching off), gives each request the result the same
requests give in order on a world of their own (bit-exact body state; bit-exact potentials, sweeps and residuals).
"""
import numpy as np
import pytest

from shatterforge_b200 import scenes as S

pytestmark = pytest.mark.gpu


def scene(seed, n):
    return S.debris_scene(n, seed=seed, obstacles=(2, 4), spacing=1.3, p_geom=0.4, kmax=12)


@pytest.fixture(scope="module")
def sv():
    from shatterforge_b200 import serving
    return serving


def cover(sv, scs, headroom=1.0):
    """A slot capacity that holds each of the scenes."""
    caps = [sv.slot_for(s, headroom) for s in scs]
    return tuple(max(c[i] for c in caps) for i in range(4))


def test_pool_slot_equals_world(sf, sv):
    scs = [scene(60 + k, 70 + 40 * k) for k in range(3)]
    cap = cover(sv, scs, 1.2)
    pool = sv.ScenePool([cap] * 4, iterations=8)
    for k, s in enumerate(scs):
        pool.load(k, s)
    pool.step(1 / 60, nsteps=50)
    for k, s in enumerate(scs):
        w = sf.World(s, iterations=8)
        w.step(1 / 60, nsteps=50)
        st, sl, fl = w.bodies()
        pst, psl, pfl = pool.bodies(k)
        np.testing.assert_array_equal(pst, st)
        np.testing.assert_array_equal(psl, sl)
        np.testing.assert_array_equal(pfl, fl)


def test_pool_save_restore_is_exact(sf, sv):
    a, b = scene(70, 150), scene(71, 120)
    cap = cover(sv, [a, b], 1.1)
    pool = sv.ScenePool([cap, cap], iterations=8)
    pool.load(0, a)
    pool.step_slots([0], nsteps=35)
    snap = pool.save(0)
    pool.load(0, b)                 # the slot is reused meanwhile
    pool.step_slots([0], nsteps=10)
    pool.restore(1, a, snap)        # a comes back in the other slot
    pool.step_slots([1], nsteps=40)
    w = sf.World(a, iterations=8)
    w.step(1 / 60, nsteps=75)
    st, sl, fl = w.bodies()
    pst, psl, pfl = pool.bodies(1)
    np.testing.assert_array_equal(pst, st)
    np.testing.assert_array_equal(psl, sl)
    np.testing.assert_array_equal(pfl, fl)


def _arrivals(rng, n_scenes, n_struct, n, rate):
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    reqs = []
    for k in range(n):
        if rng.random() < 0.7:
            reqs.append(("step", int(rng.integers(n_scenes)), int(rng.integers(1, 9)), float(t[k])))
        else:
            reqs.append(("solve", int(rng.integers(n_struct)), 0, float(t[k])))
    return reqs


@pytest.mark.parametrize("batching", [True, False])
def test_server_results_equal_alone(sf, sv, batching):
    rng = np.random.default_rng(9)
    scs = [scene(80 + k, int(rng.integers(60, 260))) for k in range(6)]
    structs = S.structure_lattice(scale=0.03, n_struct=5)
    big = cover(sv, scs, 1.05)
    # three slots for six scenes: scenes are evicted and restored while requests keep coming
    srv = sv.Server(slots=[big] * 3, structures=structs, batching=batching, sweeps_per_tick=64, iterations=8)
    ids = [srv.add_scene(s) for s in scs]
    reqs = _arrivals(rng, len(scs), len(structs.structure_ids()), 90, rate=400.0)
    srv.start()
    tickets = {}
    for kind, wid, n, t in reqs:
        if kind == "step":
            tickets[srv.submit_step(ids[wid], n, t_arrival=t, want_state=True)] = (kind, wid, n)
        else:
            sid = structs.structure_ids()[wid]
            mask = np.nonzero(structs.static_sid == sid)[0]
            lb = rng.choice(mask, 3)
            lv = rng.uniform(50, 400, 3).astype(np.float32)
            tickets[srv.submit_solve(sid, omega=1.7, tol=1e-6, max_sweeps=6000, loads=(lb, lv), t_arrival=t)] = (kind, sid, (lb, lv))
    srv.drain(300000)
    res = {r["ticket"]: r for r in srv.poll(cap=len(reqs) + 8)}
    assert len(res) == len(reqs) and all(r["status"] == 0 for r in res.values())
    st = srv.stats()
    if batching:
        assert st["evictions"] > 0 and st["restores"] > 0
    phi = srv.phi64()
    # alone: each scene's requests in ticket order on its own world; each structure's on one structures world
    worlds = [sf.World(s, iterations=8) for s in scs]
    sw = sf.World(structs)
    for tk in sorted(tickets):
        kind, wid, x = tickets[tk]
        r = res[tk]
        if kind == "step":
            worlds[wid].step(1 / 60, nsteps=x)
            np.testing.assert_array_equal(r["state"], worlds[wid].bodies()[0])
            assert r["steps"] == x
        else:
            sv.structure_add_loads(sw, x[0], x[1])
            rep = sv.structure_solve_set(sw, [wid], 1.7, 1e-6, 6000)
            sweeps, resid = sw.solve_detail()
            assert r["sweeps"] == sweeps[wid], (tk, r["sweeps"], sweeps[wid])
            assert r["residual"] == resid[wid]
    np.testing.assert_array_equal(phi, sw.phi64())
    lat = np.array([r["t_done"] - r["t_arrival"] for r in res.values()])
    assert (lat >= 0).all()
    srv.close()


def test_server_rejects_bad_requests(sf, sv):
    sc = scene(90, 50)
    srv = sv.Server(slots=[sv.slot_for(sc)], iterations=8)
    i = srv.add_scene(sc)
    with pytest.raises(sf.SfError):
        srv.submit_step(i + 5, 2)
    with pytest.raises(sf.SfError):
        srv.submit_step(i, 0)
    with pytest.raises(sf.SfError):
        srv.submit_solve(0)           # no structures world
    with pytest.raises(sf.SfError):
        srv.add_scene(scene(91, 400))  # fits no slot
    srv.close()


def test_server_budget_is_enforced(sf, sv):
    sc = scene(92, 50)
    need = sv.pool_bytes([sv.slot_for(sc)] * 4)
    with pytest.raises(sf.SfError):
        sv.Server(slots=[sv.slot_for(sc)] * 4, budget_bytes=need // 2)


def test_server_scene_initial_state_equals_alone(sf, sv):
    """A scene registered with a running world's state is served from that state: the result equals the same steps
    on a world given the same state."""
    sc = scene(95, 150)
    src = sf.World(sc, iterations=8)
    src.step(1 / 60, nsteps=90)
    state = src.bodies()
    srv = sv.Server(slots=[sv.slot_for(sc)], iterations=8)
    i = srv.add_scene(sc)
    srv.set_scene_state(i, *state)
    srv.start()
    t = srv.submit_step(i, 7, want_state=True)
    srv.drain(60000)
    r = {x["ticket"]: x for x in srv.poll()}[t]
    w = sf.World(sc, iterations=8)
    w.set_bodies(*state)
    w.step(1 / 60, nsteps=7)
    np.testing.assert_array_equal(r["state"], w.bodies()[0])
    srv.close()


def test_pool_refuses_topology_params(sf, sv):
    """A pool has no spare capacity for detached pieces: damage or detach capacity is refused (SF_ERR_ARG); a pool
    with contact reduction and warm start steps a reloaded slot as a fresh world of the same scene does."""
    s0 = scene(71, 90)
    cap = cover(sv, [s0], 1.2)
    for kw in ({"damage": 1}, {"detach_bodies": 4, "detach_bricks": 16}):
        with pytest.raises(sf.SfError) as e:
            sv.ScenePool([cap] * 2, iterations=8, **kw)
        assert e.value.status == sf.SF_ERR_ARG
    pool = sv.ScenePool([cap] * 2, iterations=8, reduce=1, warm_start=1)
    pool.load(0, s0)
    pool.step(1 / 60, nsteps=30)
    pool.load(0, s0)                          # the same scene again: its warm-start entries start over
    pool.step(1 / 60, nsteps=30)
    w = sf.World(s0, iterations=8, reduce=1, warm_start=1)
    w.step(1 / 60, nsteps=30)
    st, sl, fl = pool.bodies(0)
    wst, wsl, wfl = w.bodies()
    np.testing.assert_array_equal(st, wst)
    np.testing.assert_array_equal(fl, wfl)
    pool.close()

"""Batched and served forms of the physics path: scene pools and the request server (C ABI in include/sf.h).

ScenePool   fixed-capacity scene slots in one world; scenes are loaded, stepped together (all slots or a chosen
            subset), saved to host memory and restored bit for bit.
Server      the native request loop: scene-step requests on a pool, structure-solve requests on a resident
            structures world, continuous batching (one tick steps every scene with work; one persistent launch
            solves every structure with work), admission by slots sized to a device-memory budget, LRU eviction
            of idle scenes to pinned host memory. `batching=False` runs the same requests one at a time.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (SF_REQ_SOLVE, SF_REQ_STEP, Params, PoolSlot, Request, Result, SceneDesc, ServerDesc, ServerStats,
               SolveReport, Stats, _check, _ptr, default_params, fill_scene_desc, load, world_desc)
from .scenes import Scene, NY, NZ


def slot_for(scene: Scene, headroom: float = 1.0) -> tuple[int, int, int, int]:
    """(bodies, bricks, statics, chunks) a slot needs to hold `scene`."""
    xyz = scene.static_xyz
    if len(xyz):
        key = ((xyz[:, 1] >> 3) * (NZ // 8) + (xyz[:, 2] >> 3)) * (640 // 8) + (xyz[:, 0] >> 3)
        chunks = int(len(np.unique(key)))
    else:
        chunks = 0
    f = lambda n: int(np.ceil(n * headroom))  # noqa: E731
    return (max(1, f(scene.n_bodies)), max(1, f(scene.n_body_bricks)), f(scene.n_static), f(chunks))


def pool_bytes(slots) -> int:
    arr = (PoolSlot * len(slots))(*[PoolSlot(*s) for s in slots])
    out = C.c_uint64()
    _check(load().sf_pool_bytes(len(slots), arr, C.byref(out)), "sf_pool_bytes")
    return int(out.value)


class ScenePool:
    def __init__(self, slots, params: Params | None = None, **param_kw):
        self._lib = load()
        self.slots = [tuple(int(v) for v in s) for s in slots]
        arr = (PoolSlot * len(self.slots))(*[PoolSlot(*s) for s in self.slots])
        self.params = params if params is not None else default_params(**param_kw)
        h = C.c_void_p()
        _check(self._lib.sf_pool_create(len(self.slots), arr, C.byref(self.params), C.byref(h)), "sf_pool_create")
        self._h = h
        self.loaded: dict[int, Scene] = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sf_world_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, slot: int, scene: Scene):
        scene = scene.contiguous()
        d = fill_scene_desc(SceneDesc(), scene)
        _check(self._lib.sf_pool_load(self._h, int(slot), C.byref(d)), "sf_pool_load")
        self.loaded[int(slot)] = scene

    def clear(self, slot: int):
        _check(self._lib.sf_pool_clear(self._h, int(slot)), "sf_pool_clear")
        self.loaded.pop(int(slot), None)

    def save(self, slot: int) -> np.ndarray:
        n = C.c_uint64()
        _check(self._lib.sf_pool_save(self._h, int(slot), None, 0, C.byref(n)), "sf_pool_save")
        buf = np.zeros(int(n.value), np.uint8)
        _check(self._lib.sf_pool_save(self._h, int(slot), buf.ctypes.data_as(C.c_void_p), buf.nbytes, None), "sf_pool_save")
        return buf

    def restore(self, slot: int, scene: Scene, snap: np.ndarray):
        scene = scene.contiguous()
        d = fill_scene_desc(SceneDesc(), scene)
        snap = np.ascontiguousarray(snap, np.uint8)
        _check(self._lib.sf_pool_restore(self._h, int(slot), C.byref(d), snap.ctypes.data_as(C.c_void_p), snap.nbytes),
               "sf_pool_restore")
        self.loaded[int(slot)] = scene

    def bodies(self, slot: int):
        n = self.loaded[int(slot)].n_bodies
        st = np.zeros((n, 13), np.float32)
        sl = np.zeros(n, np.float32)
        fl = np.zeros(n, np.uint8)
        _check(self._lib.sf_pool_read_bodies(self._h, int(slot), _ptr(st, C.c_float), _ptr(sl, C.c_float),
                                             _ptr(fl, C.c_uint8)), "sf_pool_read_bodies")
        return st, sl, fl

    def write_bodies(self, slot: int, state13, sleep, flags):
        st = np.ascontiguousarray(state13, np.float32)
        sl = np.ascontiguousarray(sleep, np.float32)
        fl = np.ascontiguousarray(flags, np.uint8)
        _check(self._lib.sf_pool_write_bodies(self._h, int(slot), _ptr(st, C.c_float), _ptr(sl, C.c_float),
                                              _ptr(fl, C.c_uint8)), "sf_pool_write_bodies")

    def step(self, dt: float = 1.0 / 60.0, nsteps: int = 1) -> Stats:
        _check(self._lib.sf_world_step(self._h, float(dt), int(nsteps)), "sf_world_step")
        return self.stats()

    def step_slots(self, slots, dt: float = 1.0 / 60.0, nsteps: int = 1) -> Stats:
        m = np.zeros(len(self.slots), np.uint8)
        m[list(slots)] = 1
        _check(self._lib.sf_world_step_scenes(self._h, float(dt), int(nsteps), _ptr(m, C.c_uint8)), "sf_world_step_scenes")
        return self.stats()

    def stats(self) -> Stats:
        s = Stats()
        _check(self._lib.sf_get_stats(self._h, C.byref(s)), "sf_get_stats")
        return s


class Server:
    def __init__(self, slots=(), structures=None, budget_bytes: int = 0, dt: float = 1.0 / 60.0,
                 sweeps_per_tick: int = 128, batching: bool = True, params: Params | None = None, **param_kw):
        self._lib = load()
        self.slots = [tuple(int(v) for v in s) for s in slots]
        arr = (PoolSlot * max(len(self.slots), 1))(*[PoolSlot(*s) for s in self.slots])
        self._keep = [arr]
        desc = ServerDesc()
        desc.n_slots = len(self.slots)
        desc.slots = arr
        self.structures = None
        if structures is not None:
            if isinstance(structures, Scene):
                structures = [structures]
            wd, keep = world_desc(structures)
            self._keep += [wd, keep]
            desc.structures = C.pointer(wd)
            self.structures = keep[0]
        desc.budget_bytes = int(budget_bytes)
        desc.dt = float(dt)
        desc.sweeps_per_tick = int(sweeps_per_tick)
        desc.batching = 1 if batching else 0
        desc.params = params if params is not None else default_params(**param_kw)
        h = C.c_void_p()
        _check(self._lib.sf_server_create(C.byref(desc), C.byref(h)), "sf_server_create")
        self._h = h
        self._outs: dict[int, np.ndarray] = {}
        self.scenes: list[Scene] = []

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sf_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, scene: Scene) -> int:
        scene = scene.contiguous()
        d = fill_scene_desc(SceneDesc(), scene)
        i = C.c_uint32()
        _check(self._lib.sf_server_add_scene(self._h, C.byref(d), C.byref(i)), "sf_server_add_scene")
        self.scenes.append(scene)
        return int(i.value)

    def set_scene_state(self, scene: int, state13, sleep, flags):
        """Body state the scene starts from at its first load (a world that has already been running)."""
        st = np.ascontiguousarray(state13, np.float32)
        sl = np.ascontiguousarray(sleep, np.float32)
        fl = np.ascontiguousarray(flags, np.uint8)
        _check(self._lib.sf_server_set_scene_state(self._h, int(scene), _ptr(st, C.c_float), _ptr(sl, C.c_float),
                                                   _ptr(fl, C.c_uint8)), "sf_server_set_scene_state")

    def start(self):
        _check(self._lib.sf_server_start(self._h), "sf_server_start")

    def submit_step(self, scene: int, nsteps: int, t_arrival: float = 0.0, want_state: bool = False) -> int:
        r = Request()
        r.kind, r.world, r.nsteps, r.t_arrival = SF_REQ_STEP, int(scene), int(nsteps), float(t_arrival)
        out = None
        if want_state:
            out = np.zeros((self.scenes[scene].n_bodies, 13), np.float32)
            r.out_state13 = _ptr(out, C.c_float)
        t = C.c_uint64()
        _check(self._lib.sf_server_submit(self._h, C.byref(r), C.byref(t)), "sf_server_submit")
        if out is not None:
            self._outs[int(t.value)] = out
        return int(t.value)

    def submit_solve(self, structure: int, omega: float = 1.7, tol: float = 1e-6, max_sweeps: int = 20000,
                     loads=None, t_arrival: float = 0.0) -> int:
        r = Request()
        r.kind, r.world, r.omega, r.tol, r.max_sweeps, r.t_arrival = (SF_REQ_SOLVE, int(structure), float(omega),
                                                                     float(tol), int(max_sweeps), float(t_arrival))
        if loads is not None and len(loads[0]):
            lb = np.ascontiguousarray(loads[0], np.uint32)
            lv = np.ascontiguousarray(loads[1], np.float32)
            r.n_loads, r.load_brick, r.load_value = len(lb), _ptr(lb, C.c_uint32), _ptr(lv, C.c_float)
        t = C.c_uint64()
        _check(self._lib.sf_server_submit(self._h, C.byref(r), C.byref(t)), "sf_server_submit")
        return int(t.value)

    def poll(self, cap: int = 4096, wait_ms: int = 0) -> list[dict]:
        buf = (Result * cap)()
        n = C.c_uint32()
        _check(self._lib.sf_server_poll(self._h, buf, cap, C.byref(n), int(wait_ms)), "sf_server_poll")
        out = []
        for k in range(n.value):
            r = buf[k]
            d = {f: getattr(r, f) for f, _ in Result._fields_ if f != "reserved"}
            d["state"] = self._outs.pop(int(r.ticket), None)
            out.append(d)
        return out

    def drain(self, timeout_ms: int = 600000):
        _check(self._lib.sf_server_drain(self._h, int(timeout_ms)), "sf_server_drain")

    def stats(self) -> dict:
        s = ServerStats()
        _check(self._lib.sf_server_get_stats(self._h, C.byref(s)), "sf_server_get_stats")
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def phi64(self) -> np.ndarray:
        n = sum(s.n_static for s in self.structures)
        phi = np.zeros(max(n, 1), np.float64)
        _check(self._lib.sf_server_read_phi64(self._h, _ptr(phi, C.c_double)), "sf_server_read_phi64")
        return phi[:n]


def structure_solve_set(world, structures, omega: float = 1.7, tol: float = 1e-6, max_sweeps: int = 20000) -> SolveReport:
    """sf_structure_solve_set on a World."""
    ids = np.ascontiguousarray(structures, np.int32)
    r = SolveReport()
    _check(load().sf_structure_solve_set(world._h, _ptr(ids, C.c_int32), len(ids), float(omega), float(tol),
                                         int(max_sweeps), C.byref(r)), "sf_structure_solve_set")
    return r


def structure_add_loads(world, bricks, values):
    b = np.ascontiguousarray(bricks, np.uint32)
    v = np.ascontiguousarray(values, np.float32)
    _check(load().sf_structure_add_loads(world._h, len(b), _ptr(b, C.c_uint32), _ptr(v, C.c_float)),
           "sf_structure_add_loads")

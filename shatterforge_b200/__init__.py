"""shatterforge_b200 — B200 (sm_100a) implementation of Shatterforge's per-step physics path.

Python face of the C ABI in include/sf.h (loaded with ctypes from the in-tree shared library). The calls mirror
the reference engine's entry points:

    World.step(dt)             the rigid part of `step(dt)` (src/lib.rs:3640-3651)
    World.structure_solve()    the load-path sweeps of `structural` / `warm_step` (src/lib.rs:1005-1079)
    World.structure_check()    the joint pass of `structural` (stress_brick, src/lib.rs:1153-1227)

Errors raise SfError carrying the sf_status code; nothing falls back to a CPU path — if the library or a CUDA
device is missing, the call fails.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from .scenes import Scene  # noqa: F401

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_lib" / "libsf_b200.so"

SF_OK, SF_ERR_ARG, SF_ERR_CAPACITY, SF_ERR_CUDA, SF_ERR_TIMEOUT, SF_ERR_BUDGET, SF_ERR_STATE, SF_ERR_VERIFY = range(8)
SF_SLEEP_BODY, SF_SLEEP_ISLAND = 0, 1
STATIC = 0xFFFFFFFF
J_HOLD, J_FATIGUE, J_FAIL, J_CRUSH, J_ABSENT = 0, 1, 2, 3, 255

_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_f32p = C.POINTER(C.c_float)


class SfError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: status {status} ({_status_name(status)}): {last_error()}")
        self.status = status


class SceneDesc(C.Structure):
    _fields_ = [("n_static", C.c_uint32), ("static_xyz", _i32p), ("static_mat", _u8p), ("static_sid", _i32p),
                ("static_infill", _u8p), ("n_bodies", C.c_uint32), ("body_first", _u32p), ("body_brick_xyz", _i32p),
                ("body_brick_mat", _u8p), ("body_pose", _f32p)]


class WorldDesc(C.Structure):
    _fields_ = [("n_scenes", C.c_uint32), ("scenes", C.POINTER(SceneDesc)), ("structure_offset_per_scene", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("substeps", C.c_uint32), ("iterations", C.c_uint32), ("sleep_mode", C.c_uint32),
                ("pinch_kill", C.c_uint32), ("max_colors", C.c_uint32), ("contact_capacity", C.c_uint32),
                ("verify", C.c_uint32), ("solve_blocks", C.c_uint32), ("manifold_chunk", C.c_uint32),
                ("sor_cluster", C.c_uint32), ("detach_bodies", C.c_uint32), ("detach_bricks", C.c_uint32),
                ("damage", C.c_uint32), ("reduce", C.c_uint32), ("warm_start", C.c_uint32),
                ("reserved", C.c_uint32 * 1)]


class Stats(C.Structure):
    _fields_ = [("contacts", C.c_uint64), ("manifolds", C.c_uint64), ("ref_would_drop", C.c_uint64),
                ("colors", C.c_uint32), ("color_rounds", C.c_uint32), ("islands", C.c_uint32), ("alive", C.c_uint32),
                ("awake", C.c_uint32), ("error_word", C.c_uint32), ("contact_capacity", C.c_uint64),
                ("ms_last_step", C.c_double), ("launches", C.c_uint64), ("graph_launches", C.c_uint64),
                ("cluster_solves", C.c_uint64)]


SF_PHASES = 9
PHASE_NAMES = ["pose", "hash", "contacts", "manifolds", "colour", "prep", "solve", "islands", "integrate"]


class Profile(C.Structure):
    _fields_ = [("ms", C.c_double * SF_PHASES), ("substeps", C.c_uint64), ("solve_launches", C.c_uint64),
                ("solve_contact_iters", C.c_uint64), ("contacts_sum", C.c_uint64), ("launches", C.c_uint64),
                ("gen_ms", C.c_double), ("gen_bricks", C.c_uint64)]


class SolveReport(C.Structure):
    _fields_ = [("structures", C.c_uint32), ("max_sweeps_done", C.c_uint32), ("brick_sweeps", C.c_uint64),
                ("max_residual", C.c_double), ("ms", C.c_double)]


class CheckReport(C.Structure):
    _fields_ = [("joints", C.c_uint64), ("over", C.c_uint64), ("failed", C.c_uint64), ("crushed", C.c_uint64),
                ("max_ratio", C.c_float), ("ms", C.c_double)]


class FrameReport(C.Structure):
    _fields_ = [("sweeps", C.c_uint32), ("warm_sweeps", C.c_uint32), ("brick_updates", C.c_uint64), ("ms", C.c_double),
                ("live", C.c_uint32), ("max_ratio", C.c_float), ("joints", C.c_uint64), ("over", C.c_uint64),
                ("failed", C.c_uint64), ("crushed", C.c_uint64)]


class ConnectReport(C.Structure):
    _fields_ = [("structures", C.c_uint32), ("pieces", C.c_uint32), ("detached", C.c_uint32), ("retry", C.c_uint32),
                ("listed", C.c_uint64), ("ms", C.c_double)]


class RebuildReport(C.Structure):
    _fields_ = [("bodies", C.c_uint32), ("pieces", C.c_uint32), ("removed", C.c_uint32), ("dissolved", C.c_uint32),
                ("lone", C.c_uint32), ("reserved", C.c_uint32), ("ms", C.c_double)]


class DamageReport(C.Structure):
    _fields_ = [("contacts", C.c_uint64), ("crushed", C.c_uint64), ("removed", C.c_uint64), ("severed", C.c_uint64),
                ("cracked", C.c_uint64), ("ploughed", C.c_uint64), ("scraped", C.c_uint64)]


class BodiesReport(C.Structure):
    _fields_ = [("bodies", C.c_uint32), ("sweeps", C.c_uint32), ("brick_updates", C.c_uint64),
                ("judged", C.c_uint32), ("crushes_used", C.c_uint32), ("joints", C.c_uint64), ("over", C.c_uint64),
                ("failed", C.c_uint64), ("crushed", C.c_uint64), ("max_ratio", C.c_float), ("reserved", C.c_float),
                ("ms", C.c_double)]


class WorldInfo(C.Structure):
    _fields_ = [("n_scenes", C.c_uint32), ("n_static", C.c_uint32), ("n_bodies", C.c_uint32),
                ("n_body_bricks", C.c_uint32), ("n_structures", C.c_uint32), ("n_chunks", C.c_uint32)]


class PoolSlot(C.Structure):
    _fields_ = [("bodies", C.c_uint32), ("bricks", C.c_uint32), ("statics", C.c_uint32), ("chunks", C.c_uint32)]


class ServerDesc(C.Structure):
    _fields_ = [("n_slots", C.c_uint32), ("slots", C.POINTER(PoolSlot)), ("structures", C.POINTER(WorldDesc)),
                ("budget_bytes", C.c_uint64), ("dt", C.c_float), ("sweeps_per_tick", C.c_uint32),
                ("batching", C.c_uint32), ("params", Params)]


class Request(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("world", C.c_uint32), ("nsteps", C.c_uint32), ("omega", C.c_float),
                ("tol", C.c_float), ("max_sweeps", C.c_uint32), ("n_loads", C.c_uint32), ("reserved", C.c_uint32),
                ("load_brick", C.POINTER(C.c_uint32)), ("load_value", C.POINTER(C.c_float)),
                ("t_arrival", C.c_double), ("out_state13", C.POINTER(C.c_float))]


class Result(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("kind", C.c_uint32), ("world", C.c_uint32), ("status", C.c_uint32),
                ("steps", C.c_uint32), ("sweeps", C.c_uint32), ("reserved", C.c_uint32), ("residual", C.c_double),
                ("t_arrival", C.c_double), ("t_start", C.c_double), ("t_done", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("pending", C.c_uint64), ("step_ticks", C.c_uint64),
                ("solve_ticks", C.c_uint64), ("loads", C.c_uint64), ("restores", C.c_uint64),
                ("evictions", C.c_uint64), ("pool_bytes", C.c_uint64), ("busy_s", C.c_double), ("now_s", C.c_double)]


SF_REQ_STEP, SF_REQ_SOLVE = 1, 2
_vp = C.c_void_p
_u64p = C.POINTER(C.c_uint64)

# every exported function: name -> (restype, argtypes)
PROTOTYPES = {
    "sf_params_default": (None, [C.POINTER(Params)]),
    "sf_world_create": (C.c_int32, [C.POINTER(WorldDesc), C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "sf_world_destroy": (None, [C.c_void_p]),
    "sf_status_string": (C.c_char_p, [C.c_int32]),
    "sf_last_error": (C.c_char_p, []),
    "sf_version": (C.c_int32, []),
    "sf_world_step": (C.c_int32, [C.c_void_p, C.c_float, C.c_uint32]),
    "sf_world_step_scenes": (C.c_int32, [C.c_void_p, C.c_float, C.c_uint32, C.POINTER(C.c_uint8)]),
    "sf_world_set_stream": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "sf_set_profiling": (C.c_int32, [C.c_void_p, C.c_int32]),
    "sf_read_profile": (C.c_int32, [C.c_void_p, C.POINTER(Profile)]),
    "sf_reset_profile": (C.c_int32, [C.c_void_p]),
    "sf_read_tuning": (C.c_int32, [C.c_void_p, C.c_uint32, _i32p, C.c_uint32]),
    "sf_check_wait_timeout": (C.c_int32, [C.c_uint32, C.POINTER(C.c_double)]),
    "sf_structure_solve": (C.c_int32, [C.c_void_p, C.c_int32, C.c_float, C.c_float, C.c_uint32, C.POINTER(SolveReport)]),
    "sf_structure_check": (C.c_int32, [C.c_void_p, C.c_int32, C.c_float, C.c_int32, C.POINTER(CheckReport)]),
    "sf_read_solve_detail": (C.c_int32, [C.c_void_p, _u32p, C.POINTER(C.c_double)]),
    "sf_structure_warm": (C.c_int32, [C.c_void_p, C.c_int32]),
    "sf_structure_frame": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_float, _i32p, C.c_uint32, C.POINTER(FrameReport)]),
    "sf_read_structure_state": (C.c_int32, [C.c_void_p, _i32p, _u8p, _f32p, C.POINTER(C.c_double)]),
    "sf_structure_connect": (C.c_int32, [C.c_void_p, _i32p, C.c_uint32, _u32p, _i32p, C.POINTER(ConnectReport)]),
    "sf_world_connectivity": (C.c_int32, [C.c_void_p, _u32p, _i32p, C.POINTER(ConnectReport)]),
    "sf_world_scene_ranges": (C.c_int32, [C.c_void_p, C.c_uint32, _u32p]),
    "sf_world_remove_bricks": (C.c_int32, [C.c_void_p, _u32p, C.c_uint32, _u32p, C.c_uint32]),
    "sf_world_rebuild_bodies": (C.c_int32, [C.c_void_p, C.POINTER(RebuildReport)]),
    "sf_read_body_bonds": (C.c_int32, [C.c_void_p, _f32p, _u32p]),
    "sf_read_damage": (C.c_int32, [C.c_void_p, C.POINTER(DamageReport), _u8p]),
    "sf_bodies_frame": (C.c_int32, [C.c_void_p, C.c_float, C.c_uint32, C.POINTER(BodiesReport)]),
    "sf_read_body_fields": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double), _f32p, C.POINTER(C.c_double), _f32p, _f32p,
                                        _f32p]),
    "sf_structure_loads": (C.c_int32, [C.c_void_p, _i32p, C.c_uint32]),
    "sf_world_get_info": (C.c_int32, [C.c_void_p, C.POINTER(WorldInfo)]),
    "sf_get_stats": (C.c_int32, [C.c_void_p, C.POINTER(Stats)]),
    "sf_read_bodies": (C.c_int32, [C.c_void_p, _f32p, _f32p, _u8p]),
    "sf_write_bodies": (C.c_int32, [C.c_void_p, _f32p, _f32p, _u8p]),
    "sf_read_body_setup": (C.c_int32, [C.c_void_p, _f32p, _f32p]),
    "sf_read_brick_positions": (C.c_int32, [C.c_void_p, _f32p]),
    "sf_read_contacts": (C.c_int32, [C.c_void_p, C.c_uint32, _u32p, _f32p, _f32p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "sf_read_manifolds": (C.c_int32, [C.c_void_p, C.c_uint32, _u32p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "sf_read_islands": (C.c_int32, [C.c_void_p, _u32p]),
    "sf_read_phi": (C.c_int32, [C.c_void_p, _f32p]),
    "sf_read_phi64": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "sf_write_phi": (C.c_int32, [C.c_void_p, _f32p]),
    "sf_write_ext": (C.c_int32, [C.c_void_p, _f32p]),
    "sf_read_ext": (C.c_int32, [C.c_void_p, _f32p]),
    "sf_read_bonds": (C.c_int32, [C.c_void_p, _f32p, _u32p, _u8p]),
    "sf_read_joints": (C.c_int32, [C.c_void_p, _f32p, _f32p, _u8p, _u32p]),
    "sf_collide_boxes": (C.c_int32, [_f32p, _f32p, C.c_uint32, C.c_float, _f32p, _i32p]),
    "sf_collide_hulls": (C.c_int32, [_f32p, C.c_uint32, _f32p, _f32p, C.c_uint32, C.c_float, C.c_int32, _f32p, _i32p]),
    "sf_box_world_create": (C.c_int32, [_f32p, _u32p, C.c_uint32, C.c_void_p, C.POINTER(_vp)]),
    "sf_box_world_destroy": (None, [_vp]),
    "sf_box_world_step": (C.c_int32, [_vp, C.c_float, C.c_uint32]),
    "sf_box_world_set_hulls": (C.c_int32, [_vp, _f32p, C.c_uint32, _u32p]),
    "sf_box_world_read": (C.c_int32, [_vp, _f32p]),
    "sf_box_world_stats": (C.c_int32, [_vp, C.c_uint32, C.c_void_p]),
    "sf_box_world_manifolds": (C.c_int32, [_vp, C.c_uint32, _u32p, C.c_uint32, _u32p]),
    "sf_structure_solve_static": (C.c_int32, [C.c_uint32, _i32p, _u8p, _u8p, _f32p, C.c_float, C.c_float, C.c_uint32,
                                              C.POINTER(C.c_double), _u32p, C.POINTER(C.c_double), C.c_void_p]),
    "sf_structure_solve_set": (C.c_int32, [_vp, _i32p, C.c_uint32, C.c_float, C.c_float, C.c_uint32, C.POINTER(SolveReport)]),
    "sf_structure_add_loads": (C.c_int32, [_vp, C.c_uint32, _u32p, _f32p]),
    "sf_pool_bytes": (C.c_int32, [C.c_uint32, C.POINTER(PoolSlot), _u64p]),
    "sf_pool_create": (C.c_int32, [C.c_uint32, C.POINTER(PoolSlot), C.POINTER(Params), C.POINTER(_vp)]),
    "sf_pool_load": (C.c_int32, [_vp, C.c_uint32, C.POINTER(SceneDesc)]),
    "sf_pool_clear": (C.c_int32, [_vp, C.c_uint32]),
    "sf_pool_snapshot_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32]),
    "sf_pool_save": (C.c_int32, [_vp, C.c_uint32, _vp, C.c_uint64, _u64p]),
    "sf_pool_restore": (C.c_int32, [_vp, C.c_uint32, C.POINTER(SceneDesc), _vp, C.c_uint64]),
    "sf_pool_read_bodies": (C.c_int32, [_vp, C.c_uint32, _f32p, _f32p, _u8p]),
    "sf_pool_write_bodies": (C.c_int32, [_vp, C.c_uint32, _f32p, _f32p, _u8p]),
    "sf_server_set_scene_state": (C.c_int32, [_vp, C.c_uint32, _f32p, _f32p, _u8p]),
    "sf_server_create": (C.c_int32, [C.POINTER(ServerDesc), C.POINTER(_vp)]),
    "sf_server_add_scene": (C.c_int32, [_vp, C.POINTER(SceneDesc), _u32p]),
    "sf_server_start": (C.c_int32, [_vp]),
    "sf_server_submit": (C.c_int32, [_vp, C.POINTER(Request), _u64p]),
    "sf_server_poll": (C.c_int32, [_vp, C.POINTER(Result), C.c_uint32, _u32p, C.c_uint32]),
    "sf_server_drain": (C.c_int32, [_vp, C.c_uint32]),
    "sf_server_get_stats": (C.c_int32, [_vp, C.POINTER(ServerStats)]),
    "sf_server_read_phi64": (C.c_int32, [_vp, C.POINTER(C.c_double)]),
    "sf_server_destroy": (None, [_vp]),
}

STATIC_MAX_BRICKS = 8192
STATIC_MAX_CHUNKS = 128


def structure_solve_static(xyz, mat, infill=None, ext=None, omega: float = 1.7, tol: float = 1e-6,
                           max_sweeps: int = 20000, stream_handle: int | None = None):
    """Load-path solve of one structure with no GPU allocation (sf_structure_solve_static): for callers that
    cannot allocate device memory. Returns (f64 potentials, sweeps, final residual)."""
    lib = load()
    x = np.ascontiguousarray(xyz, np.int32).reshape(-1, 3)
    n = x.shape[0]
    m = np.ascontiguousarray(mat, np.uint8)
    inf = np.ascontiguousarray(infill if infill is not None else np.zeros(n, np.uint8), np.uint8)
    e = None if ext is None else np.ascontiguousarray(ext, np.float32)
    # the library copies n entries from each array: a shorter one would be read past its end
    for name, a in (("mat", m), ("infill", inf), ("ext", e)):
        if a is not None and a.shape != (n,):
            raise ValueError(f"{name} has shape {a.shape}; {n} bricks need shape ({n},)")
    phi = np.zeros(n, np.float64)
    sw = C.c_uint32()
    rs = C.c_double()
    _check(lib.sf_structure_solve_static(n, _ptr(x, C.c_int32), _ptr(m, C.c_uint8), _ptr(inf, C.c_uint8),
                                         None if e is None else _ptr(e, C.c_float), float(omega), float(tol),
                                         int(max_sweeps), _ptr(phi, C.c_double), C.byref(sw), C.byref(rs),
                                         C.c_void_p(stream_handle or 0)), "sf_structure_solve_static")
    return phi, sw.value, rs.value

_lib = None


def library_path() -> Path:
    return Path(os.environ.get("SF_B200_LIB", LIB_PATH))


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load the sm_100a library (building it first if the sources are newer and nvcc is present)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if build_if_missing and "SF_B200_LIB" not in os.environ:
        from . import build as _b
        try:
            if _b.needs_build():
                _b.build()
        except RuntimeError:
            if not path.exists():
                raise
    if not path.exists():
        raise FileNotFoundError(f"{path} is missing: build it with python -m shatterforge_b200.build")
    lib = C.CDLL(str(path))
    for name, (res, args) in PROTOTYPES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    try:
        return (load().sf_last_error() or b"").decode()
    except Exception:  # pragma: no cover - only when the library itself cannot load
        return ""


def _status_name(s: int) -> str:
    names = ["ok", "bad argument", "capacity exceeded", "CUDA error", "device wait timed out",
             "memory budget exceeded", "call out of order", "device self-check failed"]
    return names[s] if 0 <= s < len(names) else "unknown"


def _check(status: int, what: str) -> None:
    if status != SF_OK:
        raise SfError(status, what)


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def default_params(**kw) -> Params:
    p = Params()
    load().sf_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def fill_scene_desc(d: SceneDesc, s: Scene) -> SceneDesc:
    """Point a SceneDesc at a (contiguous) scene's arrays; the scene must outlive the calls that read it."""
    d.n_static = s.n_static
    d.static_xyz = _ptr(s.static_xyz, C.c_int32)
    d.static_mat = _ptr(s.static_mat, C.c_uint8)
    d.static_sid = _ptr(s.static_sid, C.c_int32)
    d.static_infill = _ptr(s.static_infill, C.c_uint8)
    d.n_bodies = s.n_bodies
    d.body_first = _ptr(s.body_first, C.c_uint32)
    d.body_brick_xyz = _ptr(s.body_brick_xyz, C.c_int32)
    d.body_brick_mat = _ptr(s.body_brick_mat, C.c_uint8)
    d.body_pose = _ptr(s.body_pose, C.c_float)
    return d


def world_desc(scenes):
    """(WorldDesc, keep-alive) for a list of scenes."""
    scenes = [s.contiguous() for s in scenes]
    descs = (SceneDesc * len(scenes))()
    for d, s in zip(descs, scenes):
        fill_scene_desc(d, s)
    return WorldDesc(len(scenes), descs, 0), (scenes, descs)


class World:
    """A set of independent scenes resident on the GPU, stepped together (one launch per phase for all)."""

    def __init__(self, scenes, params: Params | None = None, **param_kw):
        lib = load()
        self._lib = lib
        if isinstance(scenes, Scene):
            scenes = [scenes]
        self.scenes = [s.contiguous() for s in scenes]
        wd, _keep = world_desc(self.scenes)
        self.params = params if params is not None else default_params(**param_kw)
        h = C.c_void_p()
        _check(lib.sf_world_create(C.byref(wd), C.byref(self.params), C.byref(h)), "sf_world_create")
        self._h = h
        info = WorldInfo()
        _check(lib.sf_world_get_info(h, C.byref(info)), "sf_world_get_info")
        self.info = info
        # per scene its ranges (capacities include the spare bodies and bricks for detached pieces)
        r = np.array([self.scene_ranges(k) for k in range(len(self.scenes))], np.int64).reshape(-1, 8)
        self.static_off = np.append(r[:, 0], r[-1, 0] + r[-1, 1]) if len(r) else np.zeros(1, np.int64)
        self.body_off = np.append(r[:, 2], r[-1, 2] + r[-1, 3]) if len(r) else np.zeros(1, np.int64)
        self.brick_off = np.append(r[:, 4], r[-1, 4] + r[-1, 5]) if len(r) else np.zeros(1, np.int64)

    # -- lifecycle
    def close(self):
        if getattr(self, "_h", None):
            self._lib.sf_world_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- streams and profiling
    def set_stream(self, stream_handle: int | None):
        """Route the world's device work to a cudaStream_t (an integer handle, e.g. torch's .cuda_stream)."""
        _check(self._lib.sf_world_set_stream(self._h, C.c_void_p(stream_handle or 0)), "sf_world_set_stream")

    def set_profiling(self, on: bool = True):
        _check(self._lib.sf_set_profiling(self._h, 1 if on else 0), "sf_set_profiling")

    def profile(self) -> dict:
        p = Profile()
        _check(self._lib.sf_read_profile(self._h, C.byref(p)), "sf_read_profile")
        return {"ms": dict(zip(PHASE_NAMES, list(p.ms))), "substeps": p.substeps, "solve_launches": p.solve_launches,
                "solve_contact_iters": p.solve_contact_iters, "contacts_sum": p.contacts_sum, "launches": p.launches,
                "gen_ms": p.gen_ms, "gen_bricks": p.gen_bricks}

    def tuning(self) -> dict:
        """Blocks per SM the autotuner settled on, per size bucket (log2 of work items), for each tuned kernel."""
        out = {}
        for name, which in (("solve", 0), ("colour", 1), ("sor", 2)):
            a = np.full(40, -1, np.int32)
            _check(self._lib.sf_read_tuning(self._h, which, _ptr(a, C.c_int32), 40), "sf_read_tuning")
            out[name] = {int(b): int(v) for b, v in enumerate(a) if v >= 0}
        return out

    def reset_profile(self):
        _check(self._lib.sf_reset_profile(self._h), "sf_reset_profile")

    # -- hot path
    def step(self, dt: float = 1.0 / 60.0, nsteps: int = 1) -> "Stats":
        _check(self._lib.sf_world_step(self._h, float(dt), int(nsteps)), "sf_world_step")
        return self.stats()

    def step_scenes(self, mask, dt: float = 1.0 / 60.0, nsteps: int = 1) -> "Stats":
        """Step only the scenes whose mask entry is non-zero; the others stay exactly as they are."""
        m = np.ascontiguousarray(mask, np.uint8)
        if m.shape != (len(self.scenes),):
            raise ValueError(f"mask has shape {m.shape}, the world has {len(self.scenes)} scenes")
        _check(self._lib.sf_world_step_scenes(self._h, float(dt), int(nsteps), _ptr(m, C.c_uint8)), "sf_world_step_scenes")
        return self.stats()

    def structure_solve(self, structure: int = -1, omega: float = 1.7, tol: float = 1e-6, max_sweeps: int = 20000) -> SolveReport:
        r = SolveReport()
        _check(self._lib.sf_structure_solve(self._h, int(structure), float(omega), float(tol), int(max_sweeps), C.byref(r)),
               "sf_structure_solve")
        return r

    def structure_loads(self, structures):
        """Resting-body loads onto the listed structures (src/lib.rs:1233-1259); updates ext."""
        s = np.ascontiguousarray(structures, np.int32)
        _check(self._lib.sf_structure_loads(self._h, _ptr(s, C.c_int32), len(s)), "sf_structure_loads")

    def solve_detail(self):
        n = self.info.n_structures
        sw = np.zeros(max(n, 1), np.uint32)
        rs = np.zeros(max(n, 1), np.float64)
        _check(self._lib.sf_read_solve_detail(self._h, _ptr(sw, C.c_uint32), _ptr(rs, C.c_double)), "sf_read_solve_detail")
        return sw[:n], rs[:n]

    def structure_warm(self, structure: int):
        """warm_struct: 560 warm-up sweeps pending for a structure not yet solved (once)."""
        _check(self._lib.sf_structure_warm(self._h, int(structure)), "sf_structure_warm")

    def structure_frame(self, frame: int, active, dt: float = 1.0 / 60.0) -> FrameReport:
        """One frame of the reference's load-path schedule over the listed active structures (sf_structure_frame)."""
        a = np.ascontiguousarray(active, np.int32)
        r = FrameReport()
        _check(self._lib.sf_structure_frame(self._h, int(frame), float(dt), _ptr(a, C.c_int32), len(a), C.byref(r)),
               "sf_structure_frame")
        return r

    def structure_state(self):
        """Per structure: pending warm-up sweeps, solved flag, settle timer, residual of its last sweep."""
        n = max(self.info.n_structures, 1)
        warm = np.zeros(n, np.int32); solved = np.zeros(n, np.uint8); settle = np.zeros(n, np.float32)
        resid = np.zeros(n, np.float64)
        _check(self._lib.sf_read_structure_state(self._h, _ptr(warm, C.c_int32), _ptr(solved, C.c_uint8),
                                                 _ptr(settle, C.c_float), _ptr(resid, C.c_double)), "sf_read_structure_state")
        k = self.info.n_structures
        return warm[:k], solved[:k], settle[:k], resid[:k]

    def scene_ranges(self, scene: int):
        """(static_off, n_static, body_off, body capacity, brick_off, brick capacity, bodies used, bricks used)."""
        out = np.zeros(8, np.uint32)
        _check(self._lib.sf_world_scene_ranges(self._h, int(scene), _ptr(out, C.c_uint32)), "sf_world_scene_ranges")
        return tuple(int(x) for x in out)

    def _conn_out(self):
        n = max(self.info.n_structures, 1)
        return np.zeros(n, np.uint32), np.zeros(n, np.int32), ConnectReport()

    def structure_connect(self, structures):
        """conn_struct of the listed structures, in order: unsupported pieces become bodies. Returns (report, now,
        top) with now / top per structure id (bricks still standing, height in cells) for the listed ones."""
        a = np.ascontiguousarray(structures, np.int32)
        now, top, r = self._conn_out()
        _check(self._lib.sf_structure_connect(self._h, _ptr(a, C.c_int32), len(a), _ptr(now, C.c_uint32),
                                              _ptr(top, C.c_int32), C.byref(r)), "sf_structure_connect")
        return r, now, top

    def connectivity(self):
        """connectivity(): every structure pending since the last call (a joint failed or a brick was crushed, or a
        piece did not fit), in structure order. Returns as structure_connect."""
        now, top, r = self._conn_out()
        _check(self._lib.sf_world_connectivity(self._h, _ptr(now, C.c_uint32), _ptr(top, C.c_int32), C.byref(r)),
               "sf_world_connectivity")
        return r, now, top

    def remove_bricks(self, statics=(), body_bricks=()):
        """remove_brick of world static ids and world body-brick ids (sf_world_remove_bricks)."""
        a = np.ascontiguousarray(statics, np.uint32)
        b = np.ascontiguousarray(body_bricks, np.uint32)
        _check(self._lib.sf_world_remove_bricks(self._h, _ptr(a, C.c_uint32), len(a), _ptr(b, C.c_uint32), len(b)),
               "sf_world_remove_bricks")

    def rebuild_bodies(self) -> RebuildReport:
        """rebuild_body of every body marked since the last call (sf_world_rebuild_bodies)."""
        r = RebuildReport()
        _check(self._lib.sf_world_rebuild_bodies(self._h, C.byref(r)), "sf_world_rebuild_bodies")
        return r

    def damage(self):
        """Damage counters since the last read and per structure whether a hit woke it (sf_read_damage)."""
        r = DamageReport()
        h = np.zeros(max(self.info.n_structures, 1), np.uint8)
        _check(self._lib.sf_read_damage(self._h, C.byref(r), _ptr(h, C.c_uint8)), "sf_read_damage")
        return r, h[:self.info.n_structures]

    def bodies_frame(self, dt: float = 1.0 / 60.0, crushes_used: int = 0) -> BodiesReport:
        """The debris pieces' load field and joints for this frame (sf_bodies_frame), after structure_frame, whose
        crushes (FrameReport.crushed) the pieces' crushes count on from."""
        r = BodiesReport()
        _check(self._lib.sf_bodies_frame(self._h, float(dt), int(crushes_used), C.byref(r)), "sf_bodies_frame")
        return r

    def body_fields(self):
        """(phi64 and inertial load per body brick; residual, peak load factor, load time, largest ratio per body)."""
        nd, nb = self.info.n_body_bricks, self.info.n_bodies
        phi = np.zeros(max(nd, 1), np.float64); ext = np.zeros(max(nd, 1), np.float32)
        resid = np.zeros(max(nb, 1), np.float64)
        nmax, lt, maxr = (np.zeros(max(nb, 1), np.float32) for _ in range(3))
        _check(self._lib.sf_read_body_fields(self._h, _ptr(phi, C.c_double), _ptr(ext, C.c_float),
                                             _ptr(resid, C.c_double), _ptr(nmax, C.c_float), _ptr(lt, C.c_float),
                                             _ptr(maxr, C.c_float)), "sf_read_body_fields")
        return phi[:nd], ext[:nd], resid[:nb], nmax[:nb], lt[:nb], maxr[:nb]

    def body_bonds(self):
        """Per body brick: bonds (+x, +y, +z, foundation) and face neighbours (world body-brick ids)."""
        nd = self.info.n_body_bricks
        b = np.zeros((nd, 4), np.float32)
        nb = np.zeros((nd, 6), np.uint32)
        _check(self._lib.sf_read_body_bonds(self._h, _ptr(b, C.c_float), _ptr(nb, C.c_uint32)), "sf_read_body_bonds")
        return b, nb

    def structure_check(self, structure: int = -1, dt: float = 1.0 / 60.0, live: bool = True) -> CheckReport:
        r = CheckReport()
        _check(self._lib.sf_structure_check(self._h, int(structure), float(dt), 1 if live else 0, C.byref(r)),
               "sf_structure_check")
        return r

    # -- read-outs
    def stats(self) -> Stats:
        s = Stats()
        _check(self._lib.sf_get_stats(self._h, C.byref(s)), "sf_get_stats")
        return s

    def bodies(self, out=None):
        """(state13, sleep, flags); `out` = three C-contiguous arrays of those shapes and types to fill instead (e.g.
        pinned host buffers, which the device writes directly)."""
        nb = self.info.n_bodies
        if out is not None:
            st, sl, fl = out
            if st.shape != (nb, 13) or st.dtype != np.float32 or sl.shape != (nb,) or sl.dtype != np.float32 or \
                    fl.shape != (nb,) or fl.dtype != np.uint8 or not all(a.flags.c_contiguous for a in out):
                raise ValueError("out arrays must be C-contiguous float32 [nb, 13], float32 [nb], uint8 [nb]")
        else:
            st = np.zeros((nb, 13), np.float32)
            sl = np.zeros(nb, np.float32)
            fl = np.zeros(nb, np.uint8)
        _check(self._lib.sf_read_bodies(self._h, _ptr(st, C.c_float), _ptr(sl, C.c_float), _ptr(fl, C.c_uint8)), "sf_read_bodies")
        return st, sl, fl

    def set_bodies(self, state13, sleep, flags):
        st = np.ascontiguousarray(state13, np.float32)
        sl = np.ascontiguousarray(sleep, np.float32)
        fl = np.ascontiguousarray(flags, np.uint8)
        _check(self._lib.sf_write_bodies(self._h, _ptr(st, C.c_float), _ptr(sl, C.c_float), _ptr(fl, C.c_uint8)), "sf_write_bodies")

    def body_setup(self):
        b12 = np.zeros((self.info.n_bodies, 12), np.float32)
        l3 = np.zeros((self.info.n_body_bricks, 3), np.float32)
        _check(self._lib.sf_read_body_setup(self._h, _ptr(b12, C.c_float), _ptr(l3, C.c_float)), "sf_read_body_setup")
        return b12, l3

    def brick_positions(self):
        p = np.zeros((self.info.n_body_bricks, 3), np.float32)
        _check(self._lib.sf_read_brick_positions(self._h, _ptr(p, C.c_float)), "sf_read_brick_positions")
        return p

    def contacts(self, scene: int = 0):
        n = C.c_uint64()
        _check(self._lib.sf_read_contacts(self._h, scene, None, None, None, 0, C.byref(n)), "sf_read_contacts")
        k = n.value
        ids = np.zeros((k, 5), np.uint32)
        f = np.zeros((k, 7), np.float32)
        s = np.zeros((k, 8), np.float32)
        _check(self._lib.sf_read_contacts(self._h, scene, _ptr(ids, C.c_uint32), _ptr(f, C.c_float), _ptr(s, C.c_float), k,
                                          C.byref(n)), "sf_read_contacts")
        return ids, f, s

    def manifolds(self, scene: int = 0):
        n = C.c_uint64()
        _check(self._lib.sf_read_manifolds(self._h, scene, None, 0, C.byref(n)), "sf_read_manifolds")
        out = np.zeros((n.value, 4), np.uint32)
        _check(self._lib.sf_read_manifolds(self._h, scene, _ptr(out, C.c_uint32), n.value, C.byref(n)), "sf_read_manifolds")
        return out

    def islands(self):
        lab = np.zeros(self.info.n_bodies, np.uint32)
        _check(self._lib.sf_read_islands(self._h, _ptr(lab, C.c_uint32)), "sf_read_islands")
        return lab

    def phi(self):
        p = np.zeros(self.info.n_static, np.float32)
        _check(self._lib.sf_read_phi(self._h, _ptr(p, C.c_float)), "sf_read_phi")
        return p

    def phi64(self):
        p = np.zeros(self.info.n_static, np.float64)
        _check(self._lib.sf_read_phi64(self._h, _ptr(p, C.c_double)), "sf_read_phi64")
        return p

    def set_phi(self, phi):
        p = np.ascontiguousarray(phi, np.float32)
        _check(self._lib.sf_write_phi(self._h, _ptr(p, C.c_float)), "sf_write_phi")

    def set_ext(self, ext):
        e = np.ascontiguousarray(ext, np.float32)
        _check(self._lib.sf_write_ext(self._h, _ptr(e, C.c_float)), "sf_write_ext")

    def ext(self):
        e = np.zeros(self.info.n_static, np.float32)
        _check(self._lib.sf_read_ext(self._h, _ptr(e, C.c_float)), "sf_read_ext")
        return e

    def bonds(self):
        ns = self.info.n_static
        b = np.zeros((ns, 4), np.float32)
        nb = np.zeros((ns, 6), np.uint32)
        m = np.zeros(ns, np.uint8)
        _check(self._lib.sf_read_bonds(self._h, _ptr(b, C.c_float), _ptr(nb, C.c_uint32), _ptr(m, C.c_uint8)), "sf_read_bonds")
        return b, nb, m

    def joints(self):
        ns = self.info.n_static
        r = np.zeros((ns, 4), np.float32)
        b = np.zeros((ns, 4), np.float32)
        d = np.zeros((ns, 4), np.uint8)
        k = np.zeros((ns, 4), np.uint32)
        _check(self._lib.sf_read_joints(self._h, _ptr(r, C.c_float), _ptr(b, C.c_float), _ptr(d, C.c_uint8), _ptr(k, C.c_uint32)),
               "sf_read_joints")
        return r, b, d, k


def check_wait_timeout(limit_ms: int = 200) -> tuple[int, float]:
    """Run the device-wait self-check: returns (status, device ms waited); SF_ERR_TIMEOUT is the expected status."""
    ms = C.c_double()
    st = load().sf_check_wait_timeout(int(limit_ms), C.byref(ms))
    return int(st), float(ms.value)


def collide_hulls(hull_data: np.ndarray, shapes_a: np.ndarray, shapes_b: np.ndarray, margin: float = 0.02,
                  reduce: bool = False):
    """Batched convex-cell SAT (gpu/gpu_world.js:421-530). hull_data: [n_hulls, 80, 4] (shatterforge_b200.hulls);
    shapes: [n, 11] (centre, quaternion, half extents, hull id; a b-shape hull id < 0 is the ground).
    Returns (count[n], normal[n,3], points[n,8,4])."""
    lib = load()
    h = np.ascontiguousarray(hull_data, np.float32).reshape(-1, 80, 4)
    a = np.ascontiguousarray(shapes_a, np.float32).reshape(-1, 11)
    b = np.ascontiguousarray(shapes_b, np.float32).reshape(-1, 11)
    n = a.shape[0]
    out = np.zeros((n, 36), np.float32)
    cnt = np.zeros(n, np.int32)
    _check(lib.sf_collide_hulls(_ptr(h, C.c_float), h.shape[0], _ptr(a, C.c_float), _ptr(b, C.c_float), n, float(margin),
                                1 if reduce else 0, _ptr(out, C.c_float), _ptr(cnt, C.c_int32)), "sf_collide_hulls")
    return cnt, out[:, :3], out[:, 4:].reshape(n, 8, 4)


def collide_boxes(boxes_a: np.ndarray, boxes_b: np.ndarray, margin: float = 0.02):
    """Batched box-box SAT (engine/src/phys.rs:502-628): returns (count[n], normal[n,3], points[n,4,4])."""
    lib = load()
    a = np.ascontiguousarray(boxes_a, np.float32).reshape(-1, 10)
    b = np.ascontiguousarray(boxes_b, np.float32).reshape(-1, 10)
    n = a.shape[0]
    out = np.zeros((n, 20), np.float32)
    cnt = np.zeros(n, np.int32)
    _check(lib.sf_collide_boxes(_ptr(a, C.c_float), _ptr(b, C.c_float), n, float(margin), _ptr(out, C.c_float),
                                _ptr(cnt, C.c_int32)), "sf_collide_boxes")
    return cnt, out[:, :3], out[:, 4:].reshape(n, 4, 4)

"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg).

ctypes face of oracle/sf_oracle.cpp, the CPU restatement of the reference's hot path. The product library never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libsf_oracle.so"

ORDER_LIST, ORDER_COLOR = 0, 1
SLEEP_BODY, SLEEP_ISLAND = 0, 1
MODE_LEX_F32, MODE_LEX_F64, MODE_REDBLACK_F32, MODE_REDBLACK_F64 = 0, 1, 2, 3

_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)
_u64p = C.POINTER(C.c_uint64)


class StepParams(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("substeps", C.c_uint32), ("order", C.c_uint32), ("sleep_mode", C.c_uint32),
                ("pinch_kill", C.c_uint32), ("chunk", C.c_uint32), ("damage", C.c_uint32), ("reduce", C.c_uint32),
                ("warm", C.c_uint32)]


_lib = None


NATIVE_LIB = HERE / "_build" / "native" / "libsf_oracle.so"


def build() -> Path:
    src = HERE / "sf_oracle.cpp"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def build_native() -> Path:
    """The same oracle compiled with -march=native for the host this runs on (always rebuilt: the file may have been
    made on another machine). Used only to time the CPU baseline."""
    subprocess.run(["make", "-s", "-C", str(HERE), "native"], check=True)
    return NATIVE_LIB


_native = None


def use_native() -> None:
    """Route every later OracleWorld through the -march=native build (call before the first OracleWorld)."""
    global _lib, _native
    path = build_native()
    _native = path
    _lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    path = _native or LIB
    if not path.exists():
        build()
    lib = C.CDLL(str(path))
    lib.ow_create.restype = C.c_void_p
    lib.ow_create.argtypes = [C.c_uint32, _i32p, _u8p, _i32p, _u8p, C.c_uint32, _u32p, _i32p, _u8p, _f32p]
    lib.ow_destroy.argtypes = [C.c_void_p]
    lib.ow_counts.argtypes = [C.c_void_p, _u64p]
    lib.ow_get_bodies.argtypes = [C.c_void_p, _f32p, _f32p, _u8p]
    lib.ow_set_bodies.argtypes = [C.c_void_p, _f32p, _f32p, _u8p]
    lib.ow_get_setup.argtypes = [C.c_void_p, _f32p, _f32p]
    lib.ow_get_wpos.argtypes = [C.c_void_p, _f32p]
    lib.ow_set_wpos.argtypes = [C.c_void_p, _f32p]
    lib.ow_get_bonds.argtypes = [C.c_void_p, _f32p, _u32p]
    lib.ow_step.argtypes = [C.c_void_p, C.c_float, C.POINTER(StepParams)]
    lib.ow_contacts_only.argtypes = [C.c_void_p, C.c_float, C.c_int]
    lib.ow_get_contacts.restype = C.c_uint64
    lib.ow_get_contacts.argtypes = [C.c_void_p, _u32p, _f32p, _f32p]
    lib.ow_get_islands.argtypes = [C.c_void_p, _u32p]
    lib.ow_get_manifolds.restype = C.c_uint64
    lib.ow_get_manifolds.argtypes = [C.c_void_p, _u32p]
    lib.ow_sor.restype = C.c_double
    lib.ow_sor.argtypes = [C.c_void_p, C.c_int32, C.c_float, C.c_double, C.c_uint32, C.c_int32, _u32p]
    lib.ow_get_phi.argtypes = [C.c_void_p, _f32p]
    lib.ow_get_phi64.argtypes = [C.c_void_p, _f64p]
    lib.ow_set_phi.argtypes = [C.c_void_p, _f32p]
    lib.ow_structure_warm.argtypes = [C.c_void_p, C.c_int32]
    lib.ow_structure_frame.argtypes = [C.c_void_p, C.c_uint32, C.c_float, _i32p, C.c_uint32, _u32p]
    lib.ow_structure_state.argtypes = [C.c_void_p, _i32p, _u8p, _f32p, C.POINTER(C.c_double)]
    lib.ow_set_ext.argtypes = [C.c_void_p, _f32p]
    lib.ow_stress.restype = C.c_uint64
    lib.ow_stress.argtypes = [C.c_void_p, C.c_int32, C.c_float, C.c_int32, C.c_uint64, _u32p, _f32p, _f32p]
    lib.ow_remove_static.argtypes = [C.c_void_p, C.c_uint32]
    lib.ow_structure_loads.argtypes = [C.c_void_p, _i32p, C.c_uint32]
    lib.ow_get_ext.argtypes = [C.c_void_p, _f32p]
    lib.ow_set_capacity.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
    lib.ow_connect.argtypes = [C.c_void_p, _i32p, C.c_uint32, _u32p, _u32p, _i32p]
    lib.ow_connectivity.argtypes = [C.c_void_p, _u32p, _u32p, _i32p]
    lib.ow_conn_pending.argtypes = [C.c_void_p, _u8p]
    lib.ow_remove_bricks.argtypes = [C.c_void_p, _u32p, C.c_uint32, _u32p, C.c_uint32]
    lib.ow_rebuild_bodies.argtypes = [C.c_void_p, _u32p]
    lib.ow_body_bonds.argtypes = [C.c_void_p, _f32p, _u32p]
    lib.ow_read_damage.argtypes = [C.c_void_p, _u64p, _u8p]
    lib.ow_body_frame.argtypes = [C.c_void_p, C.c_float, C.c_uint32, _u32p]
    lib.ow_body_state.argtypes = [C.c_void_p, _f64p, _f32p, _f32p, _f32p]
    lib.ow_body_phi.argtypes = [C.c_void_p, _f64p, _f32p]
    lib.ow_crush_at.restype = C.c_uint32
    lib.ow_crush_at.argtypes = [C.c_void_p, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float, C.c_uint32]
    lib.ow_collide_hulls.restype = C.c_int32
    lib.ow_collide_hulls.argtypes = [_f32p, _f32p, _f32p, C.c_float, C.c_int32, _f32p]
    lib.ow_ref_colouring.argtypes = [C.c_uint32, _u32p, _u32p, _u32p, _u8p, _u8p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                     _u32p, _u32p]
    lib.ow_collide_boxes_batch.restype = C.c_uint64
    lib.ow_collide_boxes_batch.argtypes = [_f32p, _f32p, C.c_uint32, C.c_float, C.c_int32]
    lib.ow_collide_hulls_batch.restype = C.c_uint64
    lib.ow_collide_hulls_batch.argtypes = [_f32p, _f32p, _f32p, C.c_uint32, C.c_float, C.c_int32]
    lib.ow_collide_boxes.restype = C.c_int32
    lib.ow_collide_boxes.argtypes = [_f32p, _f32p, C.c_float, C.c_int32, _f32p]
    lib.obx_create.restype = C.c_void_p
    lib.obx_create.argtypes = [_f32p, C.c_uint32, C.c_void_p, C.c_int32]
    lib.obx_destroy.argtypes = [C.c_void_p]
    lib.obx_set_hulls.argtypes = [C.c_void_p, _f32p, C.c_uint32, _u32p]
    lib.obx_step.argtypes = [C.c_void_p, C.c_float, C.c_uint32]
    lib.obx_read.argtypes = [C.c_void_p, _f32p]
    lib.obx_stats.argtypes = [C.c_void_p, _u32p]
    lib.obx_manifolds.restype = C.c_uint32
    lib.obx_manifolds.argtypes = [C.c_void_p, _u32p, C.c_uint32]
    _lib = lib
    return lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class OracleWorld:
    """One scene in the CPU restatement."""

    def __init__(self, scene):
        self.lib = load()
        s = scene.contiguous()
        self.scene = s
        self.h = self.lib.ow_create(s.n_static, _p(s.static_xyz, C.c_int32), _p(s.static_mat, C.c_uint8),
                                    _p(s.static_sid, C.c_int32), _p(s.static_infill, C.c_uint8), s.n_bodies,
                                    _p(s.body_first, C.c_uint32), _p(s.body_brick_xyz, C.c_int32),
                                    _p(s.body_brick_mat, C.c_uint8), _p(s.body_pose, C.c_float))
        if not self.h:
            raise ValueError("oracle rejected the scene")
        self.ns = s.n_static
        self.n_struct = int(s.static_sid.max()) + 1 if s.n_static else 0

    # body and body-brick counts grow when connectivity detaches pieces
    @property
    def nb(self):
        return self.counts()["n_bodies"]

    @property
    def nd(self):
        return self.counts()["n_body_bricks"]

    def close(self):
        if self.h:
            self.lib.ow_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def counts(self):
        out = np.zeros(9, np.uint64)
        self.lib.ow_counts(self.h, _p(out, C.c_uint64))
        keys = ["n_static", "n_body_bricks", "n_bodies", "contacts", "manifolds", "colors", "would_drop", "frame", "chunks"]
        return dict(zip(keys, (int(x) for x in out)))

    def bodies(self):
        st = np.zeros((self.nb, 13), np.float32)
        sl = np.zeros(self.nb, np.float32)
        fl = np.zeros(self.nb, np.uint8)
        self.lib.ow_get_bodies(self.h, _p(st, C.c_float), _p(sl, C.c_float), _p(fl, C.c_uint8))
        return st, sl, fl

    def set_bodies(self, st, sl, fl):
        st = np.ascontiguousarray(st, np.float32); sl = np.ascontiguousarray(sl, np.float32); fl = np.ascontiguousarray(fl, np.uint8)
        self.lib.ow_set_bodies(self.h, _p(st, C.c_float), _p(sl, C.c_float), _p(fl, C.c_uint8))

    def setup(self):
        b12 = np.zeros((self.nb, 12), np.float32)
        l3 = np.zeros((self.nd, 3), np.float32)
        self.lib.ow_get_setup(self.h, _p(b12, C.c_float), _p(l3, C.c_float))
        return b12, l3

    def brick_positions(self):
        p = np.zeros((self.nd, 3), np.float32)
        self.lib.ow_get_wpos(self.h, _p(p, C.c_float))
        return p

    def set_brick_positions(self, wpos):
        p = np.ascontiguousarray(wpos, np.float32)
        self.lib.ow_set_wpos(self.h, _p(p, C.c_float))

    def bonds(self):
        b = np.zeros((self.ns, 4), np.float32)
        nb = np.zeros((self.ns, 6), np.uint32)
        self.lib.ow_get_bonds(self.h, _p(b, C.c_float), _p(nb, C.c_uint32))
        return b, nb

    def step(self, dt=1.0 / 60.0, iterations=10, substeps=2, order=ORDER_COLOR, sleep_mode=SLEEP_BODY, pinch_kill=1, chunk=16,
             damage=0, reduce=0, warm=0):
        p = StepParams(iterations, substeps, order, sleep_mode, pinch_kill, chunk, damage, reduce, warm)
        self.lib.ow_step(self.h, float(dt), C.byref(p))

    def contacts(self):
        n = self.counts()["contacts"]
        ids = np.zeros((n, 5), np.uint32)
        f = np.zeros((n, 7), np.float32)
        s = np.zeros((n, 8), np.float32)
        self.lib.ow_get_contacts(self.h, _p(ids, C.c_uint32), _p(f, C.c_float), _p(s, C.c_float))
        return ids, f, s

    def islands(self):
        lab = np.zeros(self.nb, np.uint32)
        self.lib.ow_get_islands(self.h, _p(lab, C.c_uint32))
        return lab

    def manifolds(self):
        n = self.counts()["manifolds"]
        out = np.zeros((n, 4), np.uint32)
        self.lib.ow_get_manifolds(self.h, _p(out, C.c_uint32))
        return out

    def sor(self, structure, omega=1.7, tol=1e-6, max_sweeps=100000, mode=MODE_LEX_F32):
        sw = C.c_uint32()
        r = self.lib.ow_sor(self.h, int(structure), float(omega), float(tol), int(max_sweeps), int(mode), C.byref(sw))
        return sw.value, r

    def structure_warm(self, s):
        self.lib.ow_structure_warm(self.h, int(s))

    def structure_frame(self, frame, dt, active):
        """One frame of the load-path schedule; returns (sweeps, warm_sweeps, live, joints, over, failed, crushed,
        max_ratio) of the frame."""
        a = np.ascontiguousarray(active, np.int32)
        out = np.zeros(8, np.uint32)
        self.lib.ow_structure_frame(self.h, int(frame), float(dt), _p(a, C.c_int32), len(a), _p(out, C.c_uint32))
        return tuple(int(x) for x in out[:7]) + (float(out[7:8].view(np.float32)[0]),)

    def structure_state(self, n):
        warm = np.zeros(n, np.int32); solved = np.zeros(n, np.uint8); settle = np.zeros(n, np.float32)
        resid = np.zeros(n, np.float64)
        self.lib.ow_structure_state(self.h, _p(warm, C.c_int32), _p(solved, C.c_uint8), _p(settle, C.c_float),
                                    resid.ctypes.data_as(C.POINTER(C.c_double)))
        return warm, solved, settle, resid

    def phi(self):
        p = np.zeros(self.ns, np.float32)
        self.lib.ow_get_phi(self.h, _p(p, C.c_float))
        return p

    def phi64(self):
        p = np.zeros(self.ns, np.float64)
        self.lib.ow_get_phi64(self.h, _p(p, C.c_double))
        return p

    def set_phi(self, phi):
        p = np.ascontiguousarray(phi, np.float32)
        self.lib.ow_set_phi(self.h, _p(p, C.c_float))

    def set_ext(self, ext):
        e = np.ascontiguousarray(ext, np.float32)
        self.lib.ow_set_ext(self.h, _p(e, C.c_float))

    def stress(self, structure, dt=1.0 / 60.0, live=True, cap=None):
        cap = cap or self.ns * 4 + 16
        ids = np.zeros((cap, 5), np.uint32)
        vals = np.zeros((cap, 2), np.float32)
        mr = C.c_float()
        n = self.lib.ow_stress(self.h, int(structure), float(dt), 1 if live else 0, cap, _p(ids, C.c_uint32),
                               _p(vals, C.c_float), C.byref(mr))
        return ids[:n], vals[:n], mr.value

    def structure_loads(self, structures):
        s = np.ascontiguousarray(structures, np.int32)
        self.lib.ow_structure_loads(self.h, _p(s, C.c_int32), len(s))

    def ext(self):
        e = np.zeros(self.ns, np.float32)
        self.lib.ow_get_ext(self.h, _p(e, C.c_float))
        return e

    def remove_static(self, i):
        self.lib.ow_remove_static(self.h, int(i))

    def set_capacity(self, spare_bodies, spare_bricks):
        """Room for detached pieces beyond the bodies and bricks the scene was created with."""
        self.lib.ow_set_capacity(self.h, int(spare_bodies), int(spare_bricks))

    def _conn_out(self):
        n = max(self.n_struct, 1)
        return np.zeros(3, np.uint32), np.zeros(n, np.uint32), np.zeros(n, np.int32)

    def connect(self, structures):
        """conn_struct of the listed structures in order; returns ((pieces, detached, pending), now, top)."""
        ids = np.ascontiguousarray(structures, np.int32)
        c, now, top = self._conn_out()
        self.lib.ow_connect(self.h, _p(ids, C.c_int32), len(ids), _p(c, C.c_uint32), _p(now, C.c_uint32),
                            _p(top, C.c_int32))
        return tuple(int(x) for x in c), now, top

    def connectivity(self):
        """connectivity(): every pending structure in structure order; returns as connect."""
        c, now, top = self._conn_out()
        self.lib.ow_connectivity(self.h, _p(c, C.c_uint32), _p(now, C.c_uint32), _p(top, C.c_int32))
        return tuple(int(x) for x in c), now, top

    def remove_bricks(self, statics=(), body_bricks=()):
        """remove_brick of static bricks (static ids) and body bricks (ids counted from the first body brick)."""
        a = np.ascontiguousarray(statics, np.uint32)
        b = np.ascontiguousarray(body_bricks, np.uint32)
        self.lib.ow_remove_bricks(self.h, _p(a, C.c_uint32), len(a), _p(b, C.c_uint32), len(b))

    def rebuild_bodies(self):
        """rebuild_body of every marked body; returns (bodies, pieces, removed, dissolved, lone)."""
        c = np.zeros(5, np.uint32)
        self.lib.ow_rebuild_bodies(self.h, _p(c, C.c_uint32))
        return tuple(int(x) for x in c)

    def body_bonds(self):
        nd = self.nd
        b = np.zeros((nd, 4), np.float32)
        nb = np.zeros((nd, 6), np.uint32)
        self.lib.ow_body_bonds(self.h, _p(b, C.c_float), _p(nb, C.c_uint32))
        return b, nb

    def crush_at(self, start, e, p, cap=2500):
        """crush_at on brick `start` (static id, or n_static + body-brick id); returns the bricks crushed."""
        return int(self.lib.ow_crush_at(self.h, int(start), float(e), float(p[0]), float(p[1]), float(p[2]), int(cap)))

    def body_frame(self, dt=1.0 / 60.0, crushes_used=0):
        """structural's debris-body part; returns (bodies swept, sweeps, brick updates, joints, over, failed, crushed,
        max ratio, crushes after the pass)."""
        c = np.zeros(9, np.uint32)
        self.lib.ow_body_frame(self.h, float(dt), int(crushes_used), _p(c, C.c_uint32))
        return tuple(int(x) for x in c[:7]) + (float(c[7:8].view(np.float32)[0]), int(c[8]))

    def body_state(self):
        nb = self.nb
        r = np.zeros(nb, np.float64); n = np.zeros(nb, np.float32); lt = np.zeros(nb, np.float32); mr = np.zeros(nb, np.float32)
        self.lib.ow_body_state(self.h, _p(r, C.c_double), _p(n, C.c_float), _p(lt, C.c_float), _p(mr, C.c_float))
        return r, n, lt, mr

    def body_phi(self):
        nd = self.nd
        p = np.zeros(nd, np.float64); e = np.zeros(nd, np.float32)
        self.lib.ow_body_phi(self.h, _p(p, C.c_double), _p(e, C.c_float))
        return p, e

    def read_damage(self, plough=False):
        """(candidates, crushed, removed, severed, cracked) since the last read (with plough: + ploughed loose,
        scraped), and per structure the hit flags."""
        c = np.zeros(7, np.uint64)
        h = np.zeros(max(self.n_struct, 1), np.uint8)
        self.lib.ow_read_damage(self.h, _p(c, C.c_uint64), _p(h, C.c_uint8))
        return tuple(int(x) for x in c[:7 if plough else 5]), h[:self.n_struct]

    def pending(self):
        f = np.zeros(max(self.n_struct, 1), np.uint8)
        self.lib.ow_conn_pending(self.h, _p(f, C.c_uint8))
        return f[:self.n_struct]


def collide_hulls(hull_data, a, b, margin=0.02, reduce=False):
    """hull_hull / hull_ground (gpu/gpu_world.js:421-530) for one pair; returns (count, normal, points[count, 4])."""
    lib = load()
    h = np.ascontiguousarray(hull_data, np.float32)
    a = np.ascontiguousarray(a, np.float32); b = np.ascontiguousarray(b, np.float32)
    out = np.zeros(36, np.float32)
    n = lib.ow_collide_hulls(_p(h, C.c_float), _p(a, C.c_float), _p(b, C.c_float), float(margin), 1 if reduce else 0,
                             _p(out, C.c_float))
    return n, out[:3].copy(), out[4:4 + 4 * n].reshape(n, 4).copy()


def collide_boxes(a, b, margin=0.02, reduce=True):
    lib = load()
    out = np.zeros(3 + 8 * 4, np.float32)
    a = np.ascontiguousarray(a, np.float32); b = np.ascontiguousarray(b, np.float32)
    n = lib.ow_collide_boxes(_p(a, C.c_float), _p(b, C.c_float), float(margin), 1 if reduce else 0, _p(out, C.c_float))
    return n, out[:3].copy(), out[3:3 + 4 * n].reshape(n, 4).copy()


def collide_batch_hits(a, b, hull_data=None, margin=0.02):
    """Box pairs (hull_data None) or hull pairs, all in one call of the restatement; returns the touching count."""
    lib = load()
    if hull_data is None:
        a = np.ascontiguousarray(a, np.float32).reshape(-1, 10); b = np.ascontiguousarray(b, np.float32).reshape(-1, 10)
        return int(lib.ow_collide_boxes_batch(_p(a, C.c_float), _p(b, C.c_float), len(a), float(margin), 1))
    h = np.ascontiguousarray(hull_data, np.float32)
    a = np.ascontiguousarray(a, np.float32).reshape(-1, 11); b = np.ascontiguousarray(b, np.float32).reshape(-1, 11)
    return int(lib.ow_collide_hulls_batch(_p(h, C.c_float), _p(a, C.c_float), _p(b, C.c_float), len(a), float(margin), 0))


def ref_colouring(a, b, a_awake, b_awake, n_bodies, color_limit=16, rounds_s=2, rounds_a=4):
    """The reference's round-based manifold colouring (gpu/gpu_world.js:922-1038) on a manifold graph; returns
    (colour per manifold, colours used, overflow manifolds). b = 0xFFFFFFFF marks the static side."""
    lib = load()
    a = np.ascontiguousarray(a, np.uint32); b = np.ascontiguousarray(b, np.uint32)
    aa = np.ascontiguousarray(a_awake, np.uint8); bb = np.ascontiguousarray(b_awake, np.uint8)
    # salt = the manifold's index among the manifolds of the same body pair (chunks of one pair)
    pair = a.astype(np.uint64) << np.uint64(32) | b.astype(np.uint64)
    order = np.argsort(pair, kind="stable")
    sp = pair[order]
    start = np.r_[0, np.nonzero(sp[1:] != sp[:-1])[0] + 1]
    run = np.repeat(start, np.diff(np.r_[start, len(sp)]))
    salt = np.zeros(len(a), np.uint32)
    salt[order] = (np.arange(len(sp)) - run).astype(np.uint32)
    col = np.zeros(len(a), np.uint32)
    st = np.zeros(2, np.uint32)
    lib.ow_ref_colouring(len(a), _p(a, C.c_uint32), _p(b, C.c_uint32), _p(salt, C.c_uint32), _p(aa, C.c_uint8), _p(bb, C.c_uint8), int(n_bodies),
                         int(color_limit), int(rounds_s), int(rounds_a), _p(col, C.c_uint32), _p(st, C.c_uint32))
    return col, int(st[0]), int(st[1])


class OracleBoxWorld:
    """The engine crate's box world (engine/src/phys.rs World) restated: `boxes` is an (n, 11) array of
    p3 q4 h3 density records (World::add_box), `params` a ctypes structure with the layout of sf_box_params, `order`
    ORDER_LIST (the reference's manifold list order) or ORDER_COLOR (key order solved colour by colour)."""

    def __init__(self, boxes, params, order=ORDER_LIST):
        self._lib = load()
        b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 11)
        self.n = len(b)
        self._h = self._lib.obx_create(_p(b, C.c_float), self.n, C.cast(C.pointer(params), C.c_void_p), int(order))

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.obx_destroy(self._h)
            self._h = None

    def set_hulls(self, hull_data, hull_ids):
        """The convex-cell library (hulls.library().packed()) and a cell per box (0 = a plain box)."""
        d = np.ascontiguousarray(hull_data, np.float32).reshape(-1, 320)
        ids = np.ascontiguousarray(hull_ids, np.uint32).reshape(-1)
        assert len(ids) == self.n
        self._hulls = d
        self._lib.obx_set_hulls(self._h, _p(d, C.c_float), len(d), _p(ids, C.c_uint32))

    def step(self, dt, n=1):
        self._lib.obx_step(self._h, float(dt), int(n))

    def state(self):
        """(n, 22): p3 q4 v3 w3 sleep_t sleep_p3 sleep_q4 awake."""
        out = np.zeros((self.n, 22), np.float32)
        self._lib.obx_read(self._h, _p(out, C.c_float))
        return out

    def stats(self):
        """awake, pairs, manifolds, points, colours of the last step."""
        out = np.zeros(5, np.uint32)
        self._lib.obx_stats(self._h, _p(out, C.c_uint32))
        return tuple(int(x) for x in out)

    def manifolds(self):
        """(m, 16) words a manifold in the solver's list: a, b, cnt, stick, n3, jn4, jt1, jt2, jtw (f32 bits), colour."""
        m = self._lib.obx_manifolds(self._h, None, 0)
        out = np.zeros((m, 16), np.uint32)
        self._lib.obx_manifolds(self._h, _p(out, C.c_uint32), m)
        return out

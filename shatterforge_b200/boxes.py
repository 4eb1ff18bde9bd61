"""The engine crate's box world on the GPU (engine/src/phys.rs `World`): oriented boxes, the hashed-grid broadphase,
box SAT with face clipping, the soft-step solver with anchored patch friction and island sleep, many scenes in one
launch. Scenes are (n, 11) float32 arrays of p3 q4 h3 density records, as `World::add_box` takes them (density 0 is
a static box).

The scene builders restate the reference's own scenarios bit for bit, including its float32 sine polynomial
(engine/src/math.rs:85-93) inside `Quat::from_axis_angle` (engine/src/math.rs:35):

  * `pile(n)`: the throughput scenario (engine/src/phys.rs:631-646), brick-sized boxes in a loose grid;
  * `stack(n)`: the 20-high gate stack (engine/src/phys.rs:654-662);
  * `tilted_box()`: `single_box_rests` (engine/src/phys.rs:664-671);
  * `offset_column()`: `tilted_stack_falls_and_settles` (engine/src/phys.rs:686-697).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

F = np.float32
TAU, PI, HALF_PI = F(6.2831855), F(3.1415927), F(1.5707964)


class BoxParams(C.Structure):
    """sf_box_params: the fields of the box world's `Params` (engine/src/phys.rs:74-98)."""
    _fields_ = [("gravity", C.c_float * 3), ("substeps", C.c_uint32), ("contact_hertz", C.c_float),
                ("damping_ratio", C.c_float), ("max_push", C.c_float), ("friction", C.c_float),
                ("speculative", C.c_float), ("sleep_lin", C.c_float), ("sleep_ang", C.c_float),
                ("sleep_time", C.c_float), ("sleep_dist", C.c_float), ("sleep_rot", C.c_float),
                ("allow_sleep", C.c_int32), ("cell", C.c_float), ("leak", C.c_float), ("anchor", C.c_int32),
                ("anchor_push", C.c_float), ("anchor_slop", C.c_float), ("reserved", C.c_uint32 * 4)]


def box_params(**kw) -> BoxParams:
    """`Params::default()` (engine/src/phys.rs:99-106), with any field overridden by keyword."""
    p = BoxParams()
    p.gravity[:] = (0.0, -9.81, 0.0)
    vals = dict(substeps=12, contact_hertz=0.0, damping_ratio=10.0, max_push=3.0, friction=0.6, speculative=0.02,
                sleep_lin=0.05, sleep_ang=0.08, sleep_time=0.5, sleep_dist=0.01, sleep_rot=0.02, allow_sleep=1,
                cell=1.0, leak=1.0, anchor=1, anchor_push=3.0, anchor_slop=0.0)
    vals.update(kw)
    for k, v in vals.items():
        if k == "gravity":
            p.gravity[:] = v
        else:
            setattr(p, k, int(v) if k in ("substeps", "allow_sleep", "anchor") else float(v))
    return p


def _floor(x):
    t = F(int(x))                    # `as i32` truncates toward zero
    return t - F(1) if t > x else t


def _sin(x):
    """The crate's sine: range-reduce to [-pi, pi], fold to [-pi/2, pi/2], then the odd Taylor polynomial to x^9."""
    x = F(x)
    a = F(x - TAU * _floor(x / TAU + F(0.5)))
    if a > PI * F(0.5):
        a = PI - a
    elif a < -PI * F(0.5):
        a = -PI - a
    a2 = a * a
    t = F(1) - a2 / F(72)
    t = F(1) - a2 / F(42) * t
    t = F(1) - a2 / F(20) * t
    t = F(1) - a2 / F(6) * t
    return F(a * t)


def from_axis_angle(axis, ang):
    ax = [F(v) for v in axis]
    l2 = ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]
    l = F(np.sqrt(l2)) if l2 > 0 else F(0)
    ax = [v * (F(1) / l) for v in ax] if l > F(1e-12) else [F(0)] * 3
    h = F(ang) * F(0.5)
    s, c = _sin(h), _sin(h + HALF_PI)
    return [ax[0] * s, ax[1] * s, ax[2] * s, c]


def _rec(p, q, h, density):
    return [F(v) for v in (*p, *q, *h, density)]


def pile(n: int) -> np.ndarray:
    side = max(int(np.sqrt(F(n) / F(20))), 1)
    h = (0.25, 0.125, 0.125)
    seed = 1

    def rnd():
        nonlocal seed
        seed = (seed * 1664525 + 1013904223) & 0xFFFFFFFF
        return F(seed >> 8) / F(16777216.0)

    out = []
    layer = 0
    while len(out) < n:
        for i in range(side):
            for j in range(side):
                if len(out) >= n:
                    break
                x = F(i) * F(0.62) + rnd() * F(0.05)
                y = F(0.2) + F(layer) * F(0.3)
                z = F(j) * F(0.36) + rnd() * F(0.05)
                axis = (rnd() - F(0.5), rnd() - F(0.5), rnd() - F(0.5))
                q = from_axis_angle(axis, rnd() * F(0.6))
                out.append(_rec((x, y, z), q, h, 1900.0))
        layer += 1
    return np.array(out, np.float32)


def stack(n: int = 20) -> np.ndarray:
    h = F(0.25)
    return np.array([_rec((0.0, h + F(2.0) * h * F(k), 0.0), (0, 0, 0, 1), (h, h, h), 1900.0) for k in range(n)], np.float32)


def tilted_box() -> np.ndarray:
    q = from_axis_angle((1.0, 0.3, 0.2), 0.7)
    return np.array([_rec((0.0, 1.0, 0.0), q, (0.25, 0.125, 0.5), 2000.0)], np.float32)


def offset_column(n: int = 10) -> np.ndarray:
    return np.array([_rec((F(0.06) * F(k), F(0.25) + F(0.5) * F(k), 0.0), (0, 0, 0, 1), (0.25, 0.25, 0.25), 1900.0)
                     for k in range(n)], np.float32)


class BoxStats(C.Structure):
    """sf_box_stats: the last step's counts of one scene."""
    _fields_ = [("awake", C.c_uint32), ("pairs", C.c_uint32), ("manifolds", C.c_uint32), ("points", C.c_uint32),
                ("colours", C.c_uint32), ("status", C.c_uint32), ("rounds", C.c_uint32), ("reserved", C.c_uint32),
                ("ms", C.c_float), ("steps", C.c_uint64), ("phase_ms", C.c_float * 5), ("reserved2", C.c_uint32)]


class BoxWorld:
    """Scenes of boxes stepped together on the GPU (sf_box_world_*). `scenes` is one (n, 11) record array or a list
    of them; every scene is an independent `World` with the same `params`."""

    def __init__(self, scenes, params: BoxParams | None = None):
        from . import _check, _ptr, load
        self._check, self._ptr = _check, _ptr
        if isinstance(scenes, np.ndarray):
            scenes = [scenes]
        recs = [np.ascontiguousarray(s, np.float32).reshape(-1, 11) for s in scenes]
        first = np.zeros(len(recs) + 1, np.uint32)
        first[1:] = np.cumsum([len(r) for r in recs])
        boxes = np.ascontiguousarray(np.concatenate(recs), np.float32)
        self.first = first
        self.n = int(first[-1])
        self.n_scenes = len(recs)
        self.params = params if params is not None else box_params()
        self._lib = load()
        h = C.c_void_p()
        _check(self._lib.sf_box_world_create(_ptr(boxes, C.c_float), _ptr(first, C.c_uint32), len(recs),
                                             C.byref(self.params), C.byref(h)), "sf_box_world_create")
        self._h = h

    def set_hulls(self, hull_data: np.ndarray, hull_ids: np.ndarray):
        """Convex cells (sf_box_world_set_hulls): hull_data the packed library (hulls.library().packed()), hull_ids a
        cell per box over all scenes (0 = a plain box)."""
        data = np.ascontiguousarray(hull_data, np.float32).reshape(-1, 320)
        ids = np.ascontiguousarray(hull_ids, np.uint32).reshape(-1)
        assert len(ids) == self.n
        self._check(self._lib.sf_box_world_set_hulls(self._h, self._ptr(data, C.c_float), len(data),
                                                     self._ptr(ids, C.c_uint32)), "sf_box_world_set_hulls")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sf_box_world_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def step(self, dt, n: int = 1):
        self._check(self._lib.sf_box_world_step(self._h, float(dt), int(n)), "sf_box_world_step")

    def state(self, scene: int | None = None) -> np.ndarray:
        """(n, 22): centre 3, quaternion 4, velocity 3, spin 3, sleep timer, rest centre 3, rest quaternion 4, awake."""
        out = np.zeros((self.n, 22), np.float32)
        self._check(self._lib.sf_box_world_read(self._h, self._ptr(out, C.c_float)), "sf_box_world_read")
        if scene is None:
            return out
        return out[self.first[scene]:self.first[scene + 1]]

    def stats(self, scene: int = 0) -> BoxStats:
        st = BoxStats()
        self._check(self._lib.sf_box_world_stats(self._h, scene, C.byref(st)), "sf_box_world_stats")
        return st

    def manifolds(self, scene: int = 0) -> np.ndarray:
        """(m, 16) words a manifold in key order: a, b, count, stick, normal 3, jn 4, jt1, jt2, jtw (f32 bits), colour."""
        cnt = C.c_uint32()
        self._check(self._lib.sf_box_world_manifolds(self._h, scene, None, 0, C.byref(cnt)), "sf_box_world_manifolds")
        out = np.zeros((cnt.value, 16), np.uint32)
        if cnt.value:
            self._check(self._lib.sf_box_world_manifolds(self._h, scene, self._ptr(out, C.c_uint32), cnt.value,
                                                         C.byref(cnt)), "sf_box_world_manifolds")
        return out


def main(argv=None) -> None:
    """Steps the reference's pile (or several copies of it, one scene each) and prints the device time a step:
    python -m shatterforge_b200.boxes --boxes 20000 --scenes 1 --warmup 60 --steps 20"""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--boxes", type=int, default=20000)
    ap.add_argument("--scenes", type=int, default=1)
    ap.add_argument("--substeps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=60)
    ap.add_argument("--steps", type=int, default=20)
    a = ap.parse_args(argv)
    dt = np.float32(1.0 / 60.0)
    w = BoxWorld([pile(a.boxes)] * a.scenes, box_params(allow_sleep=0, substeps=a.substeps))
    w.step(dt, a.warmup)
    w.step(dt, a.steps)
    st = w.stats(0)
    print(json.dumps({"boxes": a.boxes, "scenes": a.scenes, "substeps": a.substeps, "ms_per_step": st.ms / a.steps,
                      "box_steps_per_s": a.boxes * a.scenes * a.steps / (st.ms * 1e-3), "pairs": st.pairs,
                      "manifolds": st.manifolds, "colours": st.colours,
                      "phase_ms_per_step": [x / a.steps for x in st.phase_ms]}))
    w.close()


if __name__ == "__main__":
    main()

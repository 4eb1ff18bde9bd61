"""The library of convex fracture cells the hull narrow phase collides.

A restatement of the reference's hull library (gpu/gpu_world.js:2112-2209 `hullLibrary`, engine/src/hull.rs:83-149
`build`): 16 patterns, seed 7, each pattern the Voronoi cells of 2-6 random seeds in the cube [-1, 1]^3, every cell a
convex polytope within the GPU's limits (16 vertices, 12 faces of at most 8 vertices, 24 edges, 12 edge directions,
half size at least 0.15 on every axis). Hull 0 is the whole cube. Each cell is stored in its own bounding box mapped
to [-1, 1]^3, so a shape is a cell stretched by its half extents h.

Packed layout, 80 float4 per hull (the reference's HULL.STRIDE):
    [0]       nv, nf, nseg, ndir
    [1..16]   vertices (x, y, z, 0)
    [17..28]  face planes (n, d) with n.x <= d inside, n of unit length
    [29..52]  per face two float4 of vertex indices (8 slots, counter-clockwise about n)
    [53..64]  edges, two (i, j) pairs per float4
    [65..76]  distinct edge directions (unit)
    [77..79]  vertex count of each face (12 slots)
"""
from __future__ import annotations

import math

import numpy as np

LIMITS = dict(V=16, F=12, FV=8, S=24, D=12)
STRIDE = 80


def _rng(seed: int):
    a = seed & 0xFFFFFFFF

    def rnd() -> float:
        nonlocal a
        a = (a + 0x6D2B79F5) & 0xFFFFFFFF
        t = a
        t = ((t ^ (t >> 15)) * (t | 1)) & 0xFFFFFFFF
        t ^= (t + (((t ^ (t >> 7)) * (t | 61)) & 0xFFFFFFFF)) & 0xFFFFFFFF
        return ((t ^ (t >> 14)) & 0xFFFFFFFF) / 4294967296.0

    return rnd


def _sub(p, q):
    return (p[0] - q[0], p[1] - q[1], p[2] - q[2])


def _dot(p, q):
    return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]


def _cross(p, q):
    return (p[1] * q[2] - p[2] * q[1], p[2] * q[0] - p[0] * q[2], p[0] * q[1] - p[1] * q[0])


def _len(p):
    return math.sqrt(_dot(p, p))


def _nrm(p):
    l = _len(p)
    return (p[0] / l, p[1] / l, p[2] / l)


def polytope(planes):
    """Vertices (from triples of planes), faces (vertex loops), edges and distinct edge directions of the convex
    polytope {x : n.x <= d for every plane}."""
    V = []
    np_ = len(planes)
    for i in range(np_):
        for j in range(i + 1, np_):
            for k in range(j + 1, np_):
                (a, da), (b, db), (c, dc) = planes[i], planes[j], planes[k]
                bc = _cross(b, c)
                det = _dot(a, bc)
                if abs(det) < 1e-9:
                    continue
                ca, ab = _cross(c, a), _cross(a, b)
                x = tuple((da * bc[q] + db * ca[q] + dc * ab[q]) / det for q in range(3))
                if all(_dot(n, x) <= d + 1e-7 for n, d in planes) and not any(_len(_sub(v, x)) < 1e-6 for v in V):
                    V.append(x)
    faces = []
    for n, d in planes:
        idx = [i for i, v in enumerate(V) if abs(_dot(n, v) - d) < 1e-6]
        if len(idx) < 3:
            continue
        c = tuple(sum(V[i][q] for i in idx) / len(idx) for q in range(3))
        u = _nrm(_sub(V[idx[0]], c))
        w = _cross(n, u)
        idx.sort(key=lambda i: math.atan2(_dot(_sub(V[i], c), w), _dot(_sub(V[i], c), u)))
        faces.append((n, d, idx))
    seg = []
    for _, _, f in faces:
        for k in range(len(f)):
            i, j = f[k], f[(k + 1) % len(f)]
            if not any((x == i and y == j) or (x == j and y == i) for x, y in seg):
                seg.append((i, j))
    dirs = []
    for i, j in seg:
        dd = _nrm(_sub(V[j], V[i]))
        if not any(abs(_dot(e, dd)) > 0.9995 for e in dirs):
            dirs.append(dd)
    return V, faces, seg, dirs


def mass_props(V, faces):
    """Volume and centroid from tetrahedra (the vertices' mean, a face triangle)."""
    o = tuple(sum(v[q] for v in V) / len(V) for q in range(3))
    vol, m1 = 0.0, [0.0, 0.0, 0.0]
    for _, _, f in faces:
        for t in range(1, len(f) - 1):
            a, b, c = V[f[0]], V[f[t]], V[f[t + 1]]
            tv = abs(_dot(_sub(a, o), _cross(_sub(b, o), _sub(c, o)))) / 6.0
            vol += tv
            for q in range(3):
                m1[q] += tv * (o[q] + a[q] + b[q] + c[q]) / 4.0
    return vol, tuple(x / vol for x in m1)


class HullLibrary:
    def __init__(self, n_patterns: int = 16, seed: int = 7):
        rnd = _rng(seed)
        cube = [((1.0, 0.0, 0.0), 1.0), ((-1.0, 0.0, 0.0), 1.0), ((0.0, 1.0, 0.0), 1.0), ((0.0, -1.0, 0.0), 1.0),
                ((0.0, 0.0, 1.0), 1.0), ((0.0, 0.0, -1.0), 1.0)]
        V, faces, seg, dirs = polytope(cube)
        self.cells = [dict(V=V, faces=faces, seg=seg, dirs=dirs, box_c=(0.0, 0.0, 0.0), box_h=(1.0, 1.0, 1.0), vol=1.0,
                           pattern=-1)]
        self.patterns = []
        p = tries = 0
        while p < n_patterns and tries < 40000:
            tries += 1
            k = 2 + (p % 5)
            seeds = [tuple(rnd() * 1.6 - 0.8 for _ in range(3)) for _ in range(k)]
            out, ok = [], True
            for i in range(k):
                planes = list(cube)
                for j in range(k):
                    if j != i:
                        n = _nrm(_sub(seeds[j], seeds[i]))
                        m = tuple((seeds[i][q] + seeds[j][q]) / 2.0 for q in range(3))
                        planes.append((n, _dot(n, m)))
                V, faces, seg, dirs = polytope(planes)
                lo = [min(v[q] for v in V) for q in range(3)]
                hi = [max(v[q] for v in V) for q in range(3)]
                c = tuple((lo[q] + hi[q]) / 2.0 for q in range(3))
                h = tuple((hi[q] - lo[q]) / 2.0 for q in range(3))
                if (len(V) > LIMITS["V"] or len(faces) > LIMITS["F"] or len(seg) > LIMITS["S"] or len(dirs) > LIMITS["D"]
                        or any(len(f) > LIMITS["FV"] for _, _, f in faces) or any(x < 0.15 for x in h)):
                    ok = False
                    break
                Vb = [tuple((v[q] - c[q]) / h[q] for q in range(3)) for v in V]
                fb = []
                for n, d, f in faces:
                    n0 = tuple(n[q] * h[q] for q in range(3))
                    l = _len(n0)
                    fb.append((tuple(x / l for x in n0), (d - _dot(n, c)) / l, f))
                db = [_nrm(tuple(dd[q] / h[q] for q in range(3))) for dd in dirs]
                # the share of the cube (volume 8), on the cube-space polytope (engine/src/hull.rs:143)
                vol, _ = mass_props(V, faces)
                out.append(dict(V=Vb, faces=fb, seg=seg, dirs=db, box_c=c, box_h=h, vol=vol / 8.0, pattern=p))
            if not ok:
                continue
            ids = []
            for cell in out:
                self.cells.append(cell)
                ids.append(len(self.cells) - 1)
            self.patterns.append(ids)
            p += 1

    def __len__(self):
        return len(self.cells)

    def packed(self) -> np.ndarray:
        """float32 [n_hulls, 80, 4] in the reference's GPU layout."""
        data = np.zeros((len(self.cells), STRIDE, 4), np.float32)
        for i, H in enumerate(self.cells):
            data[i, 0] = [len(H["V"]), len(H["faces"]), len(H["seg"]), len(H["dirs"])]
            for k, v in enumerate(H["V"]):
                data[i, 1 + k, :3] = v
            for k, (n, d, f) in enumerate(H["faces"]):
                data[i, 17 + k] = [n[0], n[1], n[2], d]
                ix = list(f) + [0] * (8 - len(f))
                data[i, 29 + 2 * k] = ix[:4]
                data[i, 30 + 2 * k] = ix[4:8]
                data[i, 77 + k // 4, k % 4] = len(f)
            for k, (x, y) in enumerate(H["seg"]):
                data[i, 53 + (k >> 1), 2 * (k & 1)] = x
                data[i, 53 + (k >> 1), 2 * (k & 1) + 1] = y
            for k, dd in enumerate(H["dirs"]):
                data[i, 65 + k, :3] = dd
        return data


_LIB = None


def library() -> HullLibrary:
    global _LIB
    if _LIB is None:
        _LIB = HullLibrary()
    return _LIB

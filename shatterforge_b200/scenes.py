"""Seeded synthetic scenes for the Shatterforge physics path.

A *scene* is one independent world in the 640 x 136 x 640 lattice of 0.5 m cells (src/lib.rs:110-120): static
bricks on lattice cells (structures and obstacles) plus compound rigid bodies, each a set of bricks given in local
lattice coordinates and a parent pose.  Arrays use the layout of ``sf_scene_desc`` in include/sf.h:

    static_xyz   int32 [n, 3]   lattice cell of each static brick
    static_mat   uint8 [n]      material 1..5 (concrete, masonry, steel, glass, timber; src/lib.rs:163)
    static_sid   int32 [n]      structure id, -1 for loose static geometry
    static_infill uint8 [n]     1 = infill brick (glass always is; src/lib.rs:632)
    body_first   uint32 [nb+1]  prefix offsets of each body's bricks
    body_brick_xyz int32 [nd,3] local lattice cell of each body brick
    body_brick_mat uint8 [nd]
    body_pose    float32 [nb,13] parent position, quaternion (x, y, z, w), velocity, angular velocity

setup_body (src/lib.rs:844-891) turns a body's lattice cells into its mass, centre and inertia; the parent pose
is applied about the lattice origin exactly as the reference does.

Random numbers: small scenes draw from the reference's own xorshift32 stream (src/lib.rs:324-329); bulk scenes
(tens of thousands of bodies) draw from numpy's PCG64 seeded from that stream, so every scene is a pure function
of its seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

CONC, MASON, STEEL, GLASS, WOOD = 1, 2, 3, 4, 5
NX, NY, NZ = 640, 136, 640
ORIGIN = (NX // 2, 0, NZ // 2)   # lattice cell whose centre is (0.25, 0.25, 0.25) m


class XorShift32:
    """src/lib.rs:324-329: x ^= x << 13; x ^= x >> 17; x ^= x << 5; value = (x >> 8) / 2^24."""

    def __init__(self, seed: int):
        self.x = (seed or 0x9E3779B9) & 0xFFFFFFFF

    def u32(self) -> int:
        x = self.x
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        self.x = x
        return x

    def rnd(self) -> float:
        return (self.u32() >> 8) / 16777216.0


@dataclass
class Scene:
    static_xyz: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    static_mat: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint8))
    static_sid: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    static_infill: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint8))
    body_first: np.ndarray = field(default_factory=lambda: np.zeros(1, np.uint32))
    body_brick_xyz: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    body_brick_mat: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint8))
    body_pose: np.ndarray = field(default_factory=lambda: np.zeros((0, 13), np.float32))
    name: str = ""

    @property
    def n_static(self) -> int:
        return int(self.static_mat.shape[0])

    @property
    def n_bodies(self) -> int:
        return int(self.body_pose.shape[0])

    @property
    def n_body_bricks(self) -> int:
        return int(self.body_brick_mat.shape[0])

    def contiguous(self) -> "Scene":
        self.static_xyz = np.ascontiguousarray(self.static_xyz, np.int32).reshape(-1, 3)
        self.static_mat = np.ascontiguousarray(self.static_mat, np.uint8)
        self.static_sid = np.ascontiguousarray(self.static_sid, np.int32)
        self.static_infill = np.ascontiguousarray(self.static_infill, np.uint8)
        self.body_first = np.ascontiguousarray(self.body_first, np.uint32)
        self.body_brick_xyz = np.ascontiguousarray(self.body_brick_xyz, np.int32).reshape(-1, 3)
        self.body_brick_mat = np.ascontiguousarray(self.body_brick_mat, np.uint8)
        self.body_pose = np.ascontiguousarray(self.body_pose, np.float32).reshape(-1, 13)
        return self

    def structure_ids(self) -> list[int]:
        return sorted(int(s) for s in np.unique(self.static_sid) if s >= 0)

    def without_static(self, mask: np.ndarray) -> "Scene":
        keep = ~mask
        return Scene(self.static_xyz[keep], self.static_mat[keep], self.static_sid[keep], self.static_infill[keep],
                     self.body_first, self.body_brick_xyz, self.body_brick_mat, self.body_pose, self.name).contiguous()


def _concat_static(parts):
    if not parts:
        return (np.zeros((0, 3), np.int32), np.zeros(0, np.uint8), np.zeros(0, np.int32), np.zeros(0, np.uint8))
    xyz = np.concatenate([p[0] for p in parts]).astype(np.int32)
    mat = np.concatenate([p[1] for p in parts]).astype(np.uint8)
    sid = np.concatenate([p[2] for p in parts]).astype(np.int32)
    inf = np.concatenate([p[3] for p in parts]).astype(np.uint8)
    return xyz, mat, sid, inf


def frame_structure(x0: int, z0: int, wx: int, wz: int, storeys: int, storey_h: int, col_xs, col_zs, sid: int,
                    mat_of=None, y0: int = 0):
    """A column/slab frame: per storey, (storey_h - 1)-cell columns at (col_xs x col_zs) and a full slab on top."""
    cells = []
    for s in range(storeys):
        yb = y0 + s * storey_h
        for cx in col_xs:
            for cz in col_zs:
                for y in range(yb, yb + storey_h - 1):
                    cells.append((x0 + cx, y, z0 + cz))
        ys = yb + storey_h - 1
        xs, zs = np.meshgrid(np.arange(wx), np.arange(wz), indexing="ij")
        slab = np.stack([x0 + xs.ravel(), np.full(xs.size, ys), z0 + zs.ravel()], 1)
        cells.extend(map(tuple, slab))
    xyz = np.array(cells, np.int32).reshape(-1, 3)
    if mat_of is None:
        mat = np.full(len(xyz), CONC, np.uint8)
    else:
        mat = mat_of(xyz)
    infill = (mat == GLASS).astype(np.uint8)
    return xyz, mat, np.full(len(xyz), sid, np.int32), infill


def _quat_uniform(u1, u2, u3):
    """Shoemake's uniform random unit quaternion (x, y, z, w) from three uniforms."""
    a = np.sqrt(1.0 - u1)
    b = np.sqrt(u1)
    t1 = 2.0 * math.pi * u2
    t2 = 2.0 * math.pi * u3
    return np.stack([a * np.sin(t1), a * np.cos(t1), b * np.sin(t2), b * np.cos(t2)], -1)


def frame5_structure(seed: int = 1, remove_columns: int = 2):
    """5-storey concrete frame on 24 x 24 cells; storeys of 7 cells (6-cell 1 x 1 columns on a 3 x 3 grid, then a
    full 24 x 24 slab): 5 * (9 * 6 + 576) = 3150 bricks, structure 0, centred on the lattice origin.
    Returns (scene, removed_mask) where removed_mask marks the bricks of `remove_columns` seed-chosen ground columns."""
    rng = XorShift32(seed)
    x0, z0 = ORIGIN[0] - 12, ORIGIN[2] - 12
    cols = [0, 11, 23]
    xyz, mat, sid, inf = frame_structure(x0, z0, 24, 24, 5, 7, cols, cols, 0)
    sc = Scene(xyz, mat, sid, inf, name="frame5").contiguous()
    ground_cols = [(x0 + cx, z0 + cz) for cx in cols for cz in cols]
    chosen = []
    while len(chosen) < remove_columns:
        k = int(rng.rnd() * len(ground_cols)) % len(ground_cols)
        if k not in chosen:
            chosen.append(k)
    removed = np.zeros(sc.n_static, bool)
    for k in chosen:
        cx, cz = ground_cols[k]
        removed |= (xyz[:, 0] == cx) & (xyz[:, 2] == cz) & (xyz[:, 1] < 6)
    return sc, removed


def loose_debris(n: int, seed: int, box_lo=(8.0, 2.0, -5.0), box_hi=(18.0, 12.0, 5.0),
                 mats=(CONC, MASON, WOOD)):
    """n single-brick bodies at xorshift32-uniform positions in an axis-aligned box, at rest (the debris beside the 5-storey frame)."""
    rng = XorShift32(seed)
    pose = np.zeros((n, 13), np.float32)
    mat = np.zeros(n, np.uint8)
    for b in range(n):
        p = [box_lo[k] + (box_hi[k] - box_lo[k]) * rng.rnd() for k in range(3)]
        # the brick's lattice centre is (0.25, 0.25, 0.25) about the parent origin
        pose[b, 0:3] = [p[0] - 0.25, p[1] - 0.25, p[2] - 0.25]
        pose[b, 6] = 1.0
        mat[b] = mats[int(rng.rnd() * len(mats)) % len(mats)]
    xyz = np.tile(np.array(ORIGIN, np.int32), (n, 1))
    return np.arange(n + 1, dtype=np.uint32), xyz, mat, pose


def body_blocks(n: int = 3, wx: int = 20, wz: int = 25, h: int = 8, gap: int = 4, mat: int = CONC) -> Scene:
    """n rectangular concrete blocks of wx x h x wz bricks as bodies standing on the ground in a row along x, gap
    cells apart, at rest: bodies whose load fields need many sweeps, for the frame's shared sweep budget."""
    first, xyz = [0], []
    for k in range(n):
        x0 = k * (wx + gap)
        c = np.array([[ORIGIN[0] + x0 + x, y, ORIGIN[2] + z] for y in range(h) for z in range(wz) for x in range(wx)],
                     np.int32)
        xyz.append(c)
        first.append(first[-1] + len(c))
    pose = np.zeros((n, 13), np.float32)
    pose[:, 6] = 1.0
    allx = np.concatenate(xyz)
    return Scene(body_first=np.array(first, np.uint32), body_brick_xyz=allx,
                 body_brick_mat=np.full(len(allx), mat, np.uint8), body_pose=pose, name="body_blocks").contiguous()


def tilted_beam(length: int = 60, angle_deg: float = 45.0, height: int = 60, rows: int = 1, mat: int = CONC) -> Scene:
    """A concrete beam of length x rows x 1 bricks as one body, rotated angle_deg about z and dropped from height
    cells: it lands on one end, and the impact loads its joints past their strength."""
    c = np.array([[ORIGIN[0] + x, y, ORIGIN[2]] for y in range(rows) for x in range(length)], np.int32)
    pose = np.zeros((1, 13), np.float32)
    a = np.float32(np.radians(angle_deg) / 2.0)
    pose[0, 3:7] = [0.0, 0.0, np.sin(a), np.cos(a)]
    pose[0, 1] = height * 0.5
    return Scene(body_first=np.array([0, len(c)], np.uint32), body_brick_xyz=c,
                 body_brick_mat=np.full(len(c), mat, np.uint8), body_pose=pose, name="tilted_beam").contiguous()


def plough_scene(n_bricks: int = 12, speed: float = 8.0, block_speed: float = 8.0) -> Scene:
    """Bodies driven into static bricks: a glass pane (structure 0, 10 x 6 bricks, one layer) with n_bricks single
    concrete bricks flying at it at `speed` m/s, and a timber wall (structure 1, 10 x 8 x 2 bricks) with a 54-brick
    concrete block driven at it at `block_speed` m/s: the bricks knock glass loose, the block scrapes the timber."""
    ox, oz = ORIGIN[0], ORIGIN[2]
    pane = [(ox + 10 + x, y, oz) for y in range(6) for x in range(10)]
    wall = [(ox + 30 + x, y, oz + 10 + z) for z in range(2) for y in range(8) for x in range(10)]
    sxyz = np.array(pane + wall, np.int32)
    smat = np.array([GLASS] * len(pane) + [WOOD] * len(wall), np.uint8)
    ssid = np.array([0] * len(pane) + [1] * len(wall), np.int32)
    sinf = np.zeros(len(sxyz), np.uint8)
    first, xyz, mat, pose = [0], [], [], []
    for k in range(n_bricks):
        xyz.append([ORIGIN[0], 0, ORIGIN[2]])
        mat.append(CONC)
        first.append(first[-1] + 1)
        p = np.zeros(13, np.float32)
        # the brick's lattice centre is (0.25, 0.25, 0.25) about the parent origin
        p[0:3] = [5.25 + (k % 6) * 0.8 - 0.25, 0.8 + (k // 6) * 0.9 - 0.25, -3.0 - 0.25]
        p[6] = 1.0
        p[9] = speed
        pose.append(p)
    blk = [[ORIGIN[0] + x, y, ORIGIN[2] + z] for y in range(3) for z in range(3) for x in range(6)]
    xyz.extend(blk)
    mat.extend([CONC] * len(blk))
    first.append(first[-1] + len(blk))
    p = np.zeros(13, np.float32)
    p[0:3] = [16.0, 0.6, 2.5]
    p[6] = 1.0
    p[9] = block_speed
    pose.append(p)
    return Scene(sxyz, smat, ssid, sinf, np.array(first, np.uint32), np.array(xyz, np.int32),
                 np.array(mat, np.uint8), np.array(pose, np.float32), name="plough").contiguous()


def frame5_debris_scene(seed: int = 1, n_debris: int = 1024, removed: bool = False) -> Scene:
    """The 5-storey frame plus 1,024 loose single-brick bodies 2 m above the ground beside it."""
    frame, rm = frame5_structure(seed)
    if removed:
        frame = frame.without_static(rm)
    bf, bxyz, bmat, pose = loose_debris(n_debris, seed + 101)
    frame.body_first, frame.body_brick_xyz, frame.body_brick_mat, frame.body_pose = bf, bxyz, bmat, pose
    frame.name = "frame5_debris"
    return frame.contiguous()


def tower16_structure(seed: int = 2, remove_columns: int = 8):
    """A 16-storey tower on 48 x 48 cells, storeys of 7 cells. Per storey: 6-cell concrete columns on a
    5 x 5 grid at 12-cell spacing, glass infill panels (6 cells high, non-bearing) in alternate 2-cell bays of the
    perimeter, and a 48 x 48 slab whose outer ring is masonry (the 1-brick perimeter) and whose inside is concrete.
    16 * (25 * 6 + 534 + 2304) = 47,808 bricks, structure 0. Returns (scene, removed_mask) where removed_mask marks
    the bricks of `remove_columns` seed-chosen ground-storey columns."""
    rng = XorShift32(seed)
    W, H, storeys = 48, 7, 16
    x0, z0 = ORIGIN[0] - W // 2, ORIGIN[2] - W // 2
    cols = [0, 12, 24, 36, 47]
    ring = [(x, 0) for x in range(W)] + [(W - 1, z) for z in range(1, W)] + \
           [(x, W - 1) for x in range(W - 2, -1, -1)] + [(0, z) for z in range(W - 2, 0, -1)]
    colset = {(cx, cz) for cx in cols for cz in cols}
    bays = [c for k, c in enumerate(ring) if (k // 2) % 2 == 1 and c not in colset]
    xyz, mat = [], []
    for s in range(storeys):
        yb = s * H
        for cx in cols:
            for cz in cols:
                for y in range(yb, yb + H - 1):
                    xyz.append((x0 + cx, y, z0 + cz)); mat.append(CONC)
        for (bx, bz) in bays:
            for y in range(yb, yb + H - 1):
                xyz.append((x0 + bx, y, z0 + bz)); mat.append(GLASS)
        ys = yb + H - 1
        for x in range(W):
            for z in range(W):
                edge = x == 0 or z == 0 or x == W - 1 or z == W - 1
                xyz.append((x0 + x, ys, z0 + z)); mat.append(MASON if edge else CONC)
    xyz = np.array(xyz, np.int32)
    mat = np.array(mat, np.uint8)
    inf = (mat == GLASS).astype(np.uint8)
    sc = Scene(xyz, mat, np.zeros(len(mat), np.int32), inf, name="tower16").contiguous()
    ground_cols = [(x0 + cx, z0 + cz) for cx in cols for cz in cols]
    chosen = []
    while len(chosen) < remove_columns:
        k = int(rng.rnd() * len(ground_cols)) % len(ground_cols)
        if k not in chosen:
            chosen.append(k)
    removed = np.zeros(sc.n_static, bool)
    for k in chosen:
        cx, cz = ground_cols[k]
        removed |= (xyz[:, 0] == cx) & (xyz[:, 2] == cz) & (xyz[:, 1] < H - 1)
    return sc, removed


def tower16_debris_scene(seed: int = 2, n_bodies: int = 30000, removed: bool = True, kmax: int = 512,
                  lift: float = 60.0) -> Scene:
    """The 16-storey tower with its debris: the tower (ground columns removed) plus a pre-fragmented body set of n compound
    bodies of 1-512 bricks (k ~ Geometric(0.3), a few large slabs) falling beside and onto it from `lift` m above
    the debris mix's spawn layers (the roof is at 56 m)."""
    tower, rm = tower16_structure(seed)
    if removed:
        tower = tower.without_static(rm)
    lib = ClusterLibrary(seed ^ 0x1B873593, kmax=kmax)
    deb = debris_scene(n_bodies, seed * 7919 + 1, lib=lib, kmax=kmax, obstacles=(0, 0), spacing=2.0)
    big = max(1, n_bodies // 500)
    ks = np.diff(deb.body_first.astype(np.int64))
    # a few large fragments (slab pieces of up to kmax bricks) stand for the bodies a collapse sheds
    rng = np.random.default_rng(seed + 17)
    sel = rng.choice(n_bodies, big, replace=False)
    ks[sel] = rng.integers(kmax // 4, kmax + 1, big)
    picks = rng.integers(0, 1 << 30, n_bodies)
    cl, _ = lib.gather(ks, picks)
    first = np.zeros(n_bodies + 1, np.uint32)
    first[1:] = np.cumsum(ks)
    bmat = np.repeat(np.array((CONC, MASON, WOOD), np.uint8)[rng.integers(0, 3, n_bodies)], ks)
    pose = deb.body_pose.copy()
    pose[:, 1] += lift
    tower.body_first, tower.body_brick_xyz = first, (cl + np.array(ORIGIN, np.int32)).astype(np.int32)
    tower.body_brick_mat, tower.body_pose = bmat, pose
    tower.name = "tower16_debris"
    return tower.contiguous()


# ---------------------------------------------------------------- compound debris
_NBR = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.int32)


def random_cluster(k: int, rng: np.random.Generator) -> np.ndarray:
    """A connected random lattice cluster of k cells: grow from one cell by attaching a random free face
    neighbour of a random member."""
    cells = [(0, 0, 0)]
    seen = {(0, 0, 0)}
    while len(cells) < k:
        c = cells[int(rng.integers(len(cells)))]
        d = _NBR[int(rng.integers(6))]
        nc = (c[0] + int(d[0]), c[1] + int(d[1]), c[2] + int(d[2]))
        if nc not in seen:
            seen.add(nc)
            cells.append(nc)
    return np.array(cells, np.int32)


class ClusterLibrary:
    """Random connected clusters, `variants` per brick count, reused across bodies of the same count."""

    def __init__(self, seed: int, variants: int = 6, kmax: int = 256):
        self.rng = np.random.default_rng(seed)
        self.variants = variants
        self.kmax = kmax
        self.cache: dict[int, list[np.ndarray]] = {}

    def get(self, k: int, pick: int) -> np.ndarray:
        if k not in self.cache:
            self.cache[k] = [random_cluster(k, self.rng) for _ in range(self.variants if k > 1 else 1)]
        lst = self.cache[k]
        return lst[pick % len(lst)]

    def gather(self, ks: np.ndarray, picks: np.ndarray):
        """Vectorised get() for many bodies: (concatenated cells, per-body extent in cells)."""
        for k in sorted(set(int(k) for k in np.unique(ks))):
            self.get(k, 0)
        keys = sorted(self.cache)
        flat, off, ext, vstart, vcount = [], [0], [], np.zeros(self.kmax + 2, np.int64), np.zeros(self.kmax + 2, np.int64)
        for k in keys:
            vstart[k] = len(ext)
            vcount[k] = len(self.cache[k])
            for c in self.cache[k]:
                flat.append(c)
                off.append(off[-1] + len(c))
                ext.append(float(np.abs(c).max()))
        flat = np.concatenate(flat, 0)
        off = np.array(off[:-1], np.int64)
        ext = np.array(ext)
        lid = vstart[ks] + picks % vcount[ks]
        first = np.concatenate([[0], np.cumsum(ks)])
        idx = np.repeat(off[lid] - first[:-1], ks) + np.arange(first[-1])
        return flat[idx], ext[lid]


def debris_scene(n_bodies: int, seed: int, lib: ClusterLibrary | None = None, p_geom: float = 0.3, kmax: int = 256,
                 obstacles: tuple[int, int] = (4, 16), spacing: float = 2.5, v_sigma: float = 3.0,
                 mats=(CONC, MASON, WOOD), name: str = "debris") -> Scene:
    """A debris scene: n compound bodies of k ~ Geometric(p) bricks (capped at kmax) in connected random lattice
    clusters, uniform random orientation, N(0, v_sigma) velocities, falling onto the ground plane among 4-16
    static box obstacles (static bricks, no structure)."""
    rng = np.random.default_rng(seed)
    lib = lib or ClusterLibrary(seed ^ 0x5F3759DF)
    ks = np.minimum(rng.geometric(p_geom, n_bodies), kmax).astype(np.int64)
    picks = rng.integers(0, 1 << 30, n_bodies)
    cl, ext_cells = lib.gather(ks, picks)
    first = np.zeros(n_bodies + 1, np.uint32)
    first[1:] = np.cumsum(ks)
    # spread bricks of a body over lattice cells about the origin cell
    bxyz = (cl + np.array(ORIGIN, np.int32)).astype(np.int32)
    bmat = np.array(mats, np.uint8)[rng.integers(0, len(mats), n_bodies)]
    bmat = np.repeat(bmat, ks)
    # spawn slots: a jittered grid, at most 60 per side, layers above 2 m
    side = int(min(60, math.ceil(math.sqrt(n_bodies))))
    layers = int(math.ceil(n_bodies / (side * side)))
    slot = np.arange(n_bodies)
    rng.shuffle(slot)
    sx = slot % side
    sz = (slot // side) % side
    sy = slot // (side * side)
    jitter = rng.uniform(-0.25, 0.25, (n_bodies, 3))
    # big bodies take more room: shift by their extent in the layer above
    ext = ext_cells * 0.5 + 0.5
    half = (side - 1) * spacing * 0.5
    px = sx * spacing - half + jitter[:, 0]
    pz = sz * spacing - half + jitter[:, 2]
    py = 2.5 + sy * (spacing + 0.5) + ext + jitter[:, 1]
    q = _quat_uniform(rng.random(n_bodies), rng.random(n_bodies), rng.random(n_bodies))
    v = rng.normal(0.0, v_sigma, (n_bodies, 3))
    pose = np.zeros((n_bodies, 13), np.float32)
    pose[:, 0], pose[:, 1], pose[:, 2] = px - 0.25, py - 0.25, pz - 0.25
    pose[:, 3:7] = q
    pose[:, 7:10] = v
    # static box obstacles on the ground inside the spawn footprint
    nob = int(rng.integers(obstacles[0], obstacles[1] + 1)) if obstacles[1] > 0 else 0
    parts = []
    for _ in range(nob):
        w = rng.integers(2, 9, 3)
        w[1] = rng.integers(2, 7)
        cx = int(rng.uniform(-half, half) / 0.5) + ORIGIN[0]
        cz = int(rng.uniform(-half, half) / 0.5) + ORIGIN[2]
        xs, ys, zs = np.meshgrid(np.arange(w[0]), np.arange(w[1]), np.arange(w[2]), indexing="ij")
        xyz = np.stack([cx + xs.ravel(), ys.ravel(), cz + zs.ravel()], 1)
        m = np.full(len(xyz), CONC, np.uint8)
        parts.append((xyz, m, np.full(len(xyz), -1, np.int32), np.zeros(len(xyz), np.uint8)))
    sxyz, smat, ssid, sinf = _concat_static(parts)
    if len(sxyz):
        key = sxyz[:, 0].astype(np.int64) * (NY * NZ) + sxyz[:, 1].astype(np.int64) * NZ + sxyz[:, 2]
        _, uniq = np.unique(key, return_index=True)
        uniq.sort()
        sxyz, smat, ssid, sinf = sxyz[uniq], smat[uniq], ssid[uniq], sinf[uniq]
    return Scene(sxyz, smat, ssid, sinf, first, bxyz, bmat, pose, name).contiguous()


def debris_mix(seed: int = 3, n_scenes: int = 256, lo: int = 500, hi: int = 20000, scale: float = 1.0,
                   **kw) -> list[Scene]:
    """The debris mix: n_scenes independent debris scenes, body counts log-uniform in [lo, hi] (times `scale`)."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(math.log(lo), math.log(hi), n_scenes)) * scale
    counts = np.maximum(1, counts.astype(np.int64))
    lib = ClusterLibrary(seed ^ 0x2545F491)
    return [debris_scene(int(c), seed * 1000003 + s, lib=lib, name=f"debris{s}", **kw) for s, c in enumerate(counts)]


# ---------------------------------------------------------------- the structure lattice
def structure_lattice(seed: int = 2, n_struct: int = 37, lo: int = 1000, hi: int = 40000, cap: int = 500000,
                  scale: float = 1.0, total: float = 378000.0) -> Scene:
    """The structure lattice: n_struct column/slab frames in one 640 x 136 x 640 lattice; brick counts log-uniform in [lo, hi],
    scaled together so that 37 structures hold `total` bricks (capped at `cap`), storey height 6-8 cells, footprints
    8-60 cells a side, materials 50 % concrete, 25 % masonry, 10 % steel, 10 % timber, 5 % glass.

    Glass is non-bearing infill: under finalize_brick's rules (src/lib.rs:668-690) an infill brick bonds to nothing
    sideways and to no structural brick above it, so glass can only stand on a structural brick. It is placed as
    window panels standing on a slab's perimeter (storey height - 1 cells tall, under the next slab, which they do
    not bond to), never inside a column or a slab, where it would cut a load path. Each footprint is drawn wide
    enough that the target fits under the lattice's 136-cell height."""
    rng = np.random.default_rng(seed)
    targets = np.exp(rng.uniform(math.log(lo), math.log(hi), n_struct))
    targets *= total * n_struct / 37.0 / targets.sum()
    if targets.sum() > cap:
        targets *= cap / targets.sum()
    targets *= scale
    slots_x, slots_z = 7, 6
    parts = []
    for s in range(n_struct):
        target = float(targets[s])
        h = int(rng.integers(6, 9))
        max_storeys = (NY - 1) // h
        # the smallest square footprint that holds the target in max_storeys slabs, and the largest the target allows
        wmin = int(min(60, max(8, math.ceil(math.sqrt(target / max_storeys)))))
        wmax = int(min(60, max(wmin, math.sqrt(target / 2.0))))
        wx = int(rng.integers(wmin, wmax + 1))
        wz = int(rng.integers(wmin, wmax + 1))
        spacing = int(rng.integers(5, 13))
        col_xs = sorted(set(list(range(0, wx, spacing)) + [wx - 1]))
        col_zs = sorted(set(list(range(0, wz, spacing)) + [wz - 1]))
        structural = wx * wz + len(col_xs) * len(col_zs) * (h - 1)
        panels = int(round(0.05 / 0.95 * structural / (h - 1)))     # glass panels per storey
        per = structural + panels * (h - 1)
        storeys = int(max(1, min(max_storeys, round(target / per))))
        gx, gz = s % slots_x, s // slots_x
        x0 = 8 + gx * (NX - 16) // slots_x
        z0 = 8 + gz * (NZ - 16) // slots_z

        def mat_of(xyz, _rng=rng):
            # structural bricks: 50 / 25 / 10 / 10 of the structure's 95 % that is not glass
            u = _rng.random(len(xyz)) * 0.95
            m = np.full(len(xyz), CONC, np.uint8)
            m[u >= 0.50] = MASON
            m[u >= 0.75] = STEEL
            m[u >= 0.85] = WOOD
            return m

        parts.append(frame_structure(x0, z0, wx, wz, storeys, h, col_xs, col_zs, s, mat_of))
        # window panels on the perimeter of each slab that has a storey above it, away from the columns
        ring = [(x, 0) for x in range(wx)] + [(x, wz - 1) for x in range(wx)] + \
               [(0, z) for z in range(1, wz - 1)] + [(wx - 1, z) for z in range(1, wz - 1)]
        ring = [c for c in ring if not (c[0] in col_xs and c[1] in col_zs)]
        cells = []
        for st in range(storeys - 1):
            ys = st * h + h - 1
            pick = rng.choice(len(ring), min(panels, len(ring)), replace=False)
            for k in pick:
                cx, cz = ring[int(k)]
                for y in range(ys + 1, ys + h):
                    cells.append((x0 + cx, y, z0 + cz))
        if cells:
            g = np.array(cells, np.int32)
            parts.append((g, np.full(len(g), GLASS, np.uint8), np.full(len(g), s, np.int32), np.ones(len(g), np.uint8)))
    xyz, mat, sid, inf = _concat_static(parts)
    keep = grounded_mask(xyz, mat, sid, inf)
    return Scene(xyz[keep], mat[keep], sid[keep], inf[keep], name="structures").contiguous()


def bond_edges(xyz, mat, sid, infill):
    """Bonded + axis neighbour pairs (i, j) under finalize_brick's rules (src/lib.rs:668-690): same structure,
    both bricks present, and no infill gap (infill bonds to nothing sideways and to no structural brick above)."""
    key = (xyz[:, 0].astype(np.int64) * NY + xyz[:, 1]) * NZ + xyz[:, 2]
    order = np.argsort(key)
    skey = key[order]
    inf = ((mat == GLASS) | (infill != 0)).astype(np.uint8)
    out_i, out_j = [], []
    for a, d in enumerate(((1, 0, 0), (0, 1, 0), (0, 0, 1))):
        nk = ((xyz[:, 0].astype(np.int64) + d[0]) * NY + (xyz[:, 1] + d[1])) * NZ + (xyz[:, 2] + d[2])
        pos = np.searchsorted(skey, nk)
        pos = np.minimum(pos, len(skey) - 1)
        hit = skey[pos] == nk
        i = np.nonzero(hit)[0]
        j = order[pos[hit]]
        gap = (inf[i] != inf[j]) & ((a != 1) | (inf[i] == 1))
        ok = ~gap & (sid[i] == sid[j])
        out_i.append(i[ok]); out_j.append(j[ok])
    return np.concatenate(out_i), np.concatenate(out_j)


def grounded_mask(xyz, mat, sid, infill):
    """Bricks whose bond network reaches the ground (y = 0): an ungrounded piece would be detached as debris by
    the reference's connectivity pass (src/lib.rs:1085-1141) and has no finite load potential."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    n = len(mat)
    if n == 0:
        return np.zeros(0, bool)
    i, j = bond_edges(xyz, mat, sid, infill)
    g = coo_matrix((np.ones(len(i), np.int8), (i, j)), shape=(n, n))
    _, lab = connected_components(g, directed=False)
    good = np.zeros(lab.max() + 1, bool)
    good[lab[xyz[:, 1] == 0]] = True
    return good[lab]


# ---------------------------------------------------------------- long-horizon statistics
HEIGHT_BINS = (-1e9, 0.5, 1.0, 1.5, 2.0, 3.0, 5.0, 1e9)
SIZE_BINS = (1, 2, 4, 8, 16, 1 << 30)      # fragment size classes in bricks: 1, 2-3, 4-7, 8-15, 16+


def horizon_stats(scene: Scene, state13: np.ndarray, flags: np.ndarray) -> dict:
    """Statistics by which trajectories of a chaotic pile are compared after many steps, when bit-level agreement of
    different impulse orders is lost: the centre-of-mass height of the surviving bodies; per material, the
    histogram of their heights (HEIGHT_BINS, metres) and the surviving fraction of each fragment size class
    (SIZE_BINS, bricks per body; bodies leave by pinch removal or by falling out of the world)."""
    first = scene.body_first.astype(np.int64)
    size = np.diff(first)
    mat = scene.body_brick_mat[first[:-1]] if len(size) else np.zeros(0, np.uint8)
    alive = (flags & 1) == 1
    y = state13[:, 1].astype(np.float64)
    out = {"com_y": float(y[alive].mean()) if alive.any() else float("nan"), "alive": int(alive.sum()),
           "asleep": int(((flags & 3) == 3).sum()), "materials": {}}
    cls = np.searchsorted(np.array(SIZE_BINS), size, side="right") - 1
    for m in np.unique(mat):
        sel = mat == m
        live = sel & alive
        hist, _ = np.histogram(y[live], bins=HEIGHT_BINS)
        surv = []
        for c in range(len(SIZE_BINS) - 1):
            n0 = int((sel & (cls == c)).sum())
            surv.append((n0, int((live & (cls == c)).sum())))
        out["materials"][int(m)] = {"alive": int(live.sum()), "mean_y": float(y[live].mean()) if live.any() else float("nan"),
                                    "height_hist": (hist / max(int(live.sum()), 1)).tolist(), "survivors": surv}
    return out


def horizon_distance(a: dict, b: dict, min_class: int = 20) -> dict:
    """Largest differences between two horizon_stats: COM height (m), a material's mean height (m), the total
    variation distance of a material's height histograms, and a size class's surviving fraction (classes of at
    least min_class bodies)."""
    d = {"com_y": abs(a["com_y"] - b["com_y"]), "mean_y": 0.0, "height_tv": 0.0, "survival": 0.0}
    for m, x in a["materials"].items():
        y = b["materials"][m]
        d["mean_y"] = max(d["mean_y"], abs(x["mean_y"] - y["mean_y"]))
        d["height_tv"] = max(d["height_tv"], 0.5 * float(np.abs(np.array(x["height_hist"]) - np.array(y["height_hist"])).sum()))
        for (n0, s0), (_, s1) in zip(x["survivors"], y["survivors"]):
            if n0 >= min_class:
                d["survival"] = max(d["survival"], abs(s0 - s1) / n0)
    return d

"""Seeded synthetic scenes for the beam pipeline (positions float32, triangles uint32).

Every scene is generated from a PCG32 stream with a fixed seed, so the same
geometry is fed to the GPU tracer and to the CPU oracle.  Coordinates are
float32 from the start: both sides see exactly the same vertices.

Scenes (sizes are the workloads the benchmark and the tests use):

    room        864 triangles: 10 x 8 x 3 m box, each face an 8 x 8 quad grid,
                plus 8 seeded boxes on the floor; z is up.
    plant       ~5.4K triangles: a 24-segment stem, 400 leaves of 13 triangles
                (random yaw/pitch, length U[0.05, 0.15] m) and a ground quad;
                y is up; square area light of side 0.5 m at 3 m.
    building    ~2.1M triangles: 7 floors of 40 x 40 m, 10 x 10 rooms, walls
                tessellated into 0.5 m quads with random door gaps, desks and
                chairs as seeded boxes of 12-48 triangles; y is up.
    icosphere   20 * 4^k triangles, optional seeded fractal displacement.
    torus       any size (2 * nu * nv triangles).
    meeting     ~125K triangles: a box room with 12 tables and 120 chairs made
                of tessellated boxes and cylinders.
    analytic    floor + square occluder (closed-form soft shadows).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MASK64 = (1 << 64) - 1


class Pcg32:
    """PCG32 (O'Neill), the generator the reference seeds its scenes with
    (src/util/misc.h:24-46): same state update, output permutation and
    [0, 1) mapping, so a seed names the same stream on both sides."""

    def __init__(self, seed: int = 0x853C49E6748FEA9B, seq: int = 0xDA3E39CB94B95BDB):
        self.state = 0
        self.inc = ((seq << 1) | 1) & MASK64
        self.next()
        self.state = (self.state + seed) & MASK64
        self.next()

    def next(self) -> int:
        old = self.state
        self.state = (old * 6364136223846793005 + self.inc) & MASK64
        xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xs >> rot) | (xs << ((-rot) & 31))) & 0xFFFFFFFF

    def uniform(self, a: float = 0.0, b: float = 1.0) -> float:
        u = (self.next() >> 5) * (1.0 / 134217728.0)
        return a + (b - a) * u


@dataclass
class View:
    eye: tuple
    target: tuple
    fov: float


@dataclass
class SceneData:
    name: str
    pos: np.ndarray            # (nv, 3) float32
    tris: np.ndarray           # (nt, 3) uint32
    up: tuple = (0.0, 1.0, 0.0)
    views: list = field(default_factory=list)
    point_light: tuple | None = None
    area_light: tuple | None = None   # (c, U, V): centre and full edge vectors

    @property
    def num_tris(self) -> int:
        return int(len(self.tris))

    def light_array(self, scale: float = 1.0) -> np.ndarray:
        """Area light as 9 doubles (c, U*scale, V*scale); the scale is applied
        in float32 as the reference CLI does (apps/bt_render.cpp:288-290)."""
        c, U, V = (np.asarray(v, np.float32) for v in self.area_light)
        s = np.float32(scale)
        return np.concatenate([c, U * s, V * s]).astype(np.float64)


class _Builder:
    """Accumulates vertices and triangles (float32 / uint32)."""

    def __init__(self):
        self.pos: list = []
        self.tris: list = []
        self.nv = 0

    def verts(self, p) -> np.ndarray:
        p = np.asarray(p, np.float32).reshape(-1, 3)
        idx = np.arange(self.nv, self.nv + len(p), dtype=np.uint32)
        self.pos.append(p)
        self.nv += len(p)
        return idx

    def add(self, t):
        self.tris.append(np.asarray(t, np.uint32).reshape(-1, 3))

    def grid(self, o, du, dv, nu, nv_, flip=False):
        """A planar grid of nu x nv quads spanning o + [0,1]du + [0,1]dv."""
        o, du, dv = (np.asarray(v, np.float64) for v in (o, du, dv))
        s = np.arange(nu + 1) / nu
        t = np.arange(nv_ + 1) / nv_
        P = o[None, None, :] + s[:, None, None] * du[None, None, :] + t[None, :, None] * dv[None, None, :]
        idx = self.verts(P.reshape(-1, 3)).reshape(nu + 1, nv_ + 1)
        a = idx[:-1, :-1].ravel()
        b = idx[1:, :-1].ravel()
        c = idx[1:, 1:].ravel()
        d = idx[:-1, 1:].ravel()
        if flip:
            self.add(np.stack([a, c, b], 1))
            self.add(np.stack([a, d, c], 1))
        else:
            self.add(np.stack([a, b, c], 1))
            self.add(np.stack([a, c, d], 1))

    def box(self, lo, hi, sub=1):
        """Axis-aligned box, outward faces, each face a sub x sub grid
        (12 * sub^2 triangles); corners shared within a face."""
        lo = np.asarray(lo, np.float64)
        hi = np.asarray(hi, np.float64)
        d = hi - lo
        ex, ey, ez = np.array([d[0], 0, 0]), np.array([0, d[1], 0]), np.array([0, 0, d[2]])
        # (origin, du, dv) with du x dv pointing outward
        faces = [(lo, ey, ex), (lo + ez, ex, ey),      # -z, +z
                 (lo, ex, ez), (lo + ey, ez, ex),      # -y, +y
                 (lo, ez, ey), (lo + ex, ey, ez)]      # -x, +x
        for o, du, dv in faces:
            self.grid(o, du, dv, sub, sub)

    def cylinder(self, base, axis, r, h, seg, rings=1, cap_top=True, cap_bottom=False):
        base = np.asarray(base, np.float64)
        axis = np.asarray(axis, np.float64)
        axis = axis / np.linalg.norm(axis)
        a = np.array([1.0, 0, 0]) if abs(axis[0]) < 0.6 else np.array([0, 1.0, 0])
        u = np.cross(axis, a)
        u /= np.linalg.norm(u)
        v = np.cross(axis, u)
        ang = 2 * np.pi * np.arange(seg) / seg
        ring = np.cos(ang)[:, None] * u + np.sin(ang)[:, None] * v
        P = base[None, None, :] + (np.arange(rings + 1) / rings * h)[:, None, None] * axis + r * ring[None]
        idx = self.verts(P.reshape(-1, 3)).reshape(rings + 1, seg)
        j = np.roll(np.arange(seg), -1)
        for k in range(rings):
            i0, i1 = idx[k], idx[k + 1]
            self.add(np.stack([i0, i1[j], i1], 1))
            self.add(np.stack([i0, i0[j], i1[j]], 1))
        if cap_top:
            c = self.verts(base + axis * h)[0]
            top = idx[rings]
            self.add(np.stack([np.full(seg, c), top, top[j]], 1))
        if cap_bottom:
            c = self.verts(base)[0]
            bot = idx[0]
            self.add(np.stack([np.full(seg, c), bot[j], bot], 1))

    def build(self):
        pos = np.concatenate(self.pos).astype(np.float32)
        tris = np.concatenate(self.tris).astype(np.uint32)
        return pos, tris


def weld(pos: np.ndarray, tris: np.ndarray):
    """Merges vertices with identical float32 coordinates (shared edges then
    share vertex indices, which fixes their canonical orientation)."""
    keys = np.ascontiguousarray(pos).view(np.dtype((np.void, 12))).ravel()
    _, first, inv = np.unique(keys, return_index=True, return_inverse=True)
    order = np.argsort(first)
    remap = np.empty(len(order), np.int64)
    remap[order] = np.arange(len(order))
    new_pos = pos[first[order]]
    return new_pos, remap[inv][tris].astype(np.uint32)


# ---------------------------------------------------------------- scenes

def room(seed: int = 1) -> SceneData:
    """864 triangles: the box's 6 faces as 8 x 8 quad grids (768), inward,
    plus 8 boxes (12 triangles each) with edges U[0.3, 1.5] m, uniform on the floor."""
    b = _Builder()
    X, Y, Z = 10.0, 8.0, 3.0
    n = 8
    # inward-facing faces: du x dv points into the room
    b.grid((0, 0, 0), (X, 0, 0), (0, Y, 0), n, n)          # floor, +z
    b.grid((0, 0, Z), (0, Y, 0), (X, 0, 0), n, n)          # ceiling, -z
    b.grid((0, 0, 0), (0, 0, Z), (X, 0, 0), n, n)          # y = 0 wall, +y
    b.grid((0, Y, 0), (X, 0, 0), (0, 0, Z), n, n)          # y = Y wall, -y
    b.grid((0, 0, 0), (0, Y, 0), (0, 0, Z), n, n)          # x = 0 wall, +x
    b.grid((X, 0, 0), (0, 0, Z), (0, Y, 0), n, n)          # x = X wall, -x
    rng = Pcg32(seed)
    for _ in range(8):
        e = [rng.uniform(0.3, 1.5) for _ in range(3)]
        x0 = rng.uniform(0.0, X - e[0])
        y0 = rng.uniform(0.0, Y - e[1])
        b.box((x0, y0, 0.0), (x0 + e[0], y0 + e[1], e[2]))
    pos, tris = weld(*b.build())
    return SceneData("room", pos, tris, up=(0.0, 0.0, 1.0),
                     views=[View((1.0, 1.0, 1.6), (5.0, 4.0, 1.5), 60.0)],
                     point_light=(5.0, 4.0, 2.7),
                     area_light=((5.0, 4.0, 2.95), (1.0, 0.0, 0.0), (0.0, -1.0, 0.0)))


def _leaf(b: _Builder, base, a, w, nn, L):
    """13 triangles: a strip of 6 quads along the midrib plus a tip triangle,
    folded along the midrib."""
    s = np.arange(7) / 7.0
    half = 0.45 * L * np.sin(np.pi * (0.08 + 0.84 * s)) * (0.35 + 0.65 * s)
    fold = 0.25 * half
    mid = base[None, :] + (s * L)[:, None] * a[None, :]
    left = mid - half[:, None] * w + fold[:, None] * nn
    right = mid + half[:, None] * w + fold[:, None] * nn
    tip = base + L * a
    li = b.verts(left)
    ri = b.verts(right)
    ti = b.verts(tip)[0]
    for i in range(6):
        b.add([[li[i], ri[i], ri[i + 1]], [li[i], ri[i + 1], li[i + 1]]])
    b.add([[li[6], ri[6], ti]])


def plant(seed: int = 7, leaves: int = 400) -> SceneData:
    """24-segment stem (4 rings + top cap: 216 triangles), `leaves` leaves of
    13 triangles, 2-triangle ground quad: 5418 triangles at 400 leaves."""
    b = _Builder()
    G = 2.0
    b.grid((-G, 0, -G), (0, 0, 2 * G), (2 * G, 0, 0), 1, 1)   # ground, normal +y
    H = 0.8
    b.cylinder((0, 0, 0), (0, 1, 0), 0.02, H, 24, rings=4, cap_top=True)
    rng = Pcg32(seed)
    for _ in range(leaves):
        h = H * rng.uniform(0.25, 1.0)
        az = rng.uniform(0.0, 2 * math.pi)
        r = rng.uniform(0.02, 0.3)
        base = np.array([r * math.cos(az), h, r * math.sin(az)])
        yaw = az + rng.uniform(-0.8, 0.8)
        pitch = rng.uniform(-0.6, 0.9)
        a = np.array([math.cos(yaw) * math.cos(pitch), math.sin(pitch), math.sin(yaw) * math.cos(pitch)])
        w = np.cross(a, np.array([0.0, 1.0, 0.0]))
        w /= np.linalg.norm(w)
        roll = rng.uniform(-0.7, 0.7)
        nn = np.cross(w, a)
        w, nn = math.cos(roll) * w + math.sin(roll) * nn, -math.sin(roll) * w + math.cos(roll) * nn
        L = rng.uniform(0.05, 0.15)
        _leaf(b, base, a, w, nn, L)
    pos, tris = b.build()
    return SceneData("plant", pos, tris, up=(0.0, 1.0, 0.0),
                     views=[View((1.1, 1.05, 1.35), (0.0, 0.35, 0.0), 50.0)],
                     point_light=(0.8, 3.0, 0.6),
                     area_light=((0.3, 3.0, 0.2), (0.5, 0.0, 0.0), (0.0, 0.0, 0.5)))


def analytic(h: float = 1.0, occ: float = 1.0, F: float = 10.0) -> SceneData:
    """Floor (side 2F) and a square occluder of side `occ` at height `h` under
    a unit square light at height 3: visibility on the floor has a closed form."""
    b = _Builder()
    b.grid((-F, 0, -F), (0, 0, 2 * F), (2 * F, 0, 0), 1, 1)
    a = occ / 2
    b.grid((-a, h, -a), (0, 0, occ), (occ, 0, 0), 1, 1)
    pos, tris = b.build()
    return SceneData("analytic", pos, tris, up=(0.0, 1.0, 0.0), views=[View((0.0, 5.0, 5.0), (0.0, 0.0, 0.0), 60.0)],
                     point_light=(0.3, 3.0, 0.2),
                     area_light=((0.0, 3.0, 0.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0)))


def icosphere(subdiv: int, radius: float = 1.0, center=(0.0, 0.0, 0.0), displace: float = 0.0,
              seed: int = 3) -> SceneData:
    """Icosahedron subdivided `subdiv` times (20 * 4^subdiv triangles).  With
    `displace` > 0 every vertex moves along its normal by a seeded fractal
    (sum of octaves of random plane waves) of that amplitude."""
    t = (1.0 + 5 ** 0.5) / 2
    V = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(subdiv):
        edges = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        e = np.sort(edges, axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.ravel()
        mid = V[uniq[:, 0]] + V[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = len(V) + inv.reshape(3, -1).T   # (nf, 3): midpoints of edges 01, 12, 20
        V = np.concatenate([V, mid])
        a, b_, c = F[:, 0], F[:, 1], F[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        F = np.concatenate([np.stack([a, m01, m20], 1), np.stack([b_, m12, m01], 1),
                            np.stack([c, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    r = np.full(len(V), radius)
    if displace > 0:
        rng = Pcg32(seed)
        disp = np.zeros(len(V))
        amp, freq = 1.0, 2.0
        total = 0.0
        for _ in range(5):
            for _ in range(4):
                d = np.array([rng.uniform(-1, 1) for _ in range(3)])
                d /= np.linalg.norm(d) + 1e-12
                ph = rng.uniform(0, 2 * math.pi)
                disp += amp * np.sin(freq * (V @ d) * math.pi + ph)
                total += amp
            amp *= 0.5
            freq *= 2.0
        r = r + displace * disp / (total / 4.0)
    P = np.asarray(center)[None, :] + V * r[:, None]
    return SceneData(f"icosphere{subdiv}", P.astype(np.float32), F.astype(np.uint32))


def displaced_sphere(subdiv: int = 7, seed: int = 3) -> SceneData:
    """The served sphere: icosahedron subdivided `subdiv` times (7: 327,680
    triangles), radius 1, seeded fractal displacement of amplitude 0.1; the
    relief shadows itself.  Camera at 3 m, lights above and to the side."""
    s = icosphere(subdiv, 1.0, displace=0.1, seed=seed)
    s.up = (0.0, 1.0, 0.0)
    s.views = [View((1.8, 1.2, 2.2), (0.0, 0.0, 0.0), 45.0)]
    s.point_light = (2.5, 3.0, 1.0)
    s.area_light = ((2.0, 3.0, 1.5), (0.6, 0.0, 0.0), (0.0, 0.0, 0.6))
    return s


def torus(nu: int, nv: int, R: float = 1.0, r: float = 0.35, center=(0.0, 0.0, 0.0)) -> SceneData:
    """Torus around +y with nu x nv quads (2 * nu * nv triangles)."""
    u = 2 * np.pi * np.arange(nu) / nu
    v = 2 * np.pi * np.arange(nv) / nv
    U, Vv = np.meshgrid(u, v, indexing="ij")
    x = (R + r * np.cos(Vv)) * np.cos(U)
    z = (R + r * np.cos(Vv)) * np.sin(U)
    y = r * np.sin(Vv)
    P = np.stack([x, y, z], -1).reshape(-1, 3) + np.asarray(center)[None, :]
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    i1, j1 = (i + 1) % nu, (j + 1) % nv
    a = (i * nv + j).ravel()
    b_ = (i1 * nv + j).ravel()
    c = (i1 * nv + j1).ravel()
    d = (i * nv + j1).ravel()
    T = np.concatenate([np.stack([a, c, b_], 1), np.stack([a, d, c], 1)])
    return SceneData("torus", P.astype(np.float32), T.astype(np.uint32))


def merge(name: str, parts, **kw) -> SceneData:
    pos, tris, off = [], [], 0
    for p in parts:
        pos.append(p.pos)
        tris.append(p.tris.astype(np.int64) + off)
        off += len(p.pos)
    return SceneData(name, np.concatenate(pos).astype(np.float32), np.concatenate(tris).astype(np.uint32), **kw)


def _ground(size: float, y: float = 0.0) -> SceneData:
    b = _Builder()
    b.grid((-size, y, -size), (0, 0, 2 * size), (2 * size, 0, 0), 1, 1)
    pos, tris = b.build()
    return SceneData("ground", pos, tris)


def shadow_job(seed: int, tris_target: int) -> SceneData:
    """A receiver/occluder pair over a ground plane: a torus (any size) or an
    icosphere (20 * 4^k) with about `tris_target` triangles in total, the
    occluder hovering over the receiver, plus a 2-triangle ground."""
    rng = Pcg32(seed)
    use_torus = rng.uniform() < 0.5
    half = max(tris_target // 2, 20)
    if use_torus:
        k = max(3, int(round((half / 2) ** 0.5)))
        occ = torus(k, k, R=0.6, r=0.2, center=(0.0, 1.6, 0.0))
        rec = torus(k, k, R=1.0, r=0.35, center=(0.0, 0.4, 0.0))
    else:
        sub = max(1, min(7, int(round(math.log(half / 20.0, 4)))))
        occ = icosphere(sub, 0.45, center=(0.1, 1.7, 0.0))
        rec = icosphere(sub, 0.8, center=(0.0, 0.8, 0.0))
    return merge(f"job{seed}", [_ground(3.0), rec, occ], up=(0.0, 1.0, 0.0),
                 views=[View((2.4, 2.6, 3.0), (0.0, 0.6, 0.0), 50.0)],
                 area_light=((0.2, 3.0, 0.1), (0.5, 0.0, 0.0), (0.0, 0.0, 0.5)))


def building(floors: int = 7, rooms: int = 10, seed: int = 11, furniture: int = 31) -> SceneData:
    """Office building: `floors` slabs of 40 x 40 m, `rooms` x `rooms` rooms
    per floor, walls tessellated into 0.5 m quads (both faces) with seeded
    door gaps, and `furniture` seeded desks/chairs per room built from boxes
    of 12 or 48 triangles (the defaults give about 2.1M triangles)."""
    b = _Builder()
    S = 40.0
    cell = S / rooms
    Hf = 3.5            # floor-to-floor height
    Hw = 3.0            # wall height
    q = 0.5             # wall / slab tessellation
    nq = int(round(S / q))
    rng = Pcg32(seed)
    for f in range(floors):
        y0 = f * Hf
        # slab: top (floor of this storey) and bottom (ceiling of the one below)
        b.grid((0, y0, 0), (0, 0, S), (S, 0, 0), nq, nq)
        b.grid((0, y0 - 0.2, 0), (S, 0, 0), (0, 0, S), nq, nq)
        # walls along x at z = k * cell and along z at x = k * cell, as segments per room edge
        nseg = int(round(cell / q))
        nh = int(round(Hw / q))
        for k in range(rooms + 1):
            for r_ in range(rooms):
                door = 0 < k < rooms and rng.uniform() < 0.6
                d0 = int(rng.uniform(1, nseg - 3)) if door else -1
                for s in range(nseg):
                    if door and d0 <= s < d0 + 2:
                        # door gap: keep only the lintel quad row above 2.5 m
                        lo = int(2.5 / q)
                    else:
                        lo = 0
                    a0 = r_ * cell + s * q
                    # wall along x at z = k*cell (two faces)
                    z = k * cell
                    b.grid((a0, y0 + lo * q, z), (q, 0, 0), (0, (nh - lo) * q, 0), 1, nh - lo)
                    b.grid((a0, y0 + lo * q, z), (0, (nh - lo) * q, 0), (q, 0, 0), nh - lo, 1)
                    # wall along z at x = k*cell
                    x = k * cell
                    b.grid((x, y0 + lo * q, a0), (0, (nh - lo) * q, 0), (0, 0, q), nh - lo, 1)
                    b.grid((x, y0 + lo * q, a0), (0, 0, q), (0, (nh - lo) * q, 0), 1, nh - lo)
        for i in range(rooms):
            for j in range(rooms):
                ox, oz = i * cell + 0.3, j * cell + 0.3
                for _ in range(furniture):
                    kind = rng.uniform()
                    px = ox + rng.uniform(0.0, cell - 1.6)
                    pz = oz + rng.uniform(0.0, cell - 1.6)
                    sub = 2 if rng.uniform() < 0.35 else 1
                    if kind < 0.4:   # desk: top + 2 side panels
                        w, d = rng.uniform(0.8, 1.4), rng.uniform(0.5, 0.8)
                        b.box((px, y0 + 0.70, pz), (px + w, y0 + 0.75, pz + d), sub)
                        b.box((px, y0, pz), (px + 0.04, y0 + 0.70, pz + d), 1)
                        b.box((px + w - 0.04, y0, pz), (px + w, y0 + 0.70, pz + d), 1)
                    else:            # chair: seat, back, 4 legs
                        s_ = rng.uniform(0.4, 0.5)
                        b.box((px, y0 + 0.42, pz), (px + s_, y0 + 0.46, pz + s_), sub)
                        b.box((px, y0 + 0.46, pz + s_ - 0.04), (px + s_, y0 + 0.95, pz + s_), sub)
                        for lx in (0.0, s_ - 0.04):
                            for lz in (0.0, s_ - 0.04):
                                b.box((px + lx, y0, pz + lz), (px + lx + 0.04, y0 + 0.42, pz + lz + 0.04), 1)
    pos, tris = b.build()
    mid = 1 * Hf + 1.6
    return SceneData("building", pos, tris, up=(0.0, 1.0, 0.0),
                     views=[View((1.0, mid, 2.0), (12.0, mid - 0.4, 14.0), 70.0)],
                     point_light=(2.0, 1 * Hf + 2.7, 2.5),
                     area_light=((2.0, 1 * Hf + 2.9, 2.0), (0.8, 0.0, 0.0), (0.0, 0.0, 0.8)))


def meeting_room(seed: int = 5, tables: int = 12, chairs: int = 120) -> SceneData:
    """~125K triangles: a 20 x 14 x 3.5 m box room (tessellated walls), 12
    tables (top + cylindrical legs) and 120 chairs of tessellated boxes."""
    b = _Builder()
    X, Y, Z = 20.0, 3.5, 14.0
    b.grid((0, 0, 0), (0, 0, Z), (X, 0, 0), 80, 56)          # floor
    b.grid((0, Y, 0), (X, 0, 0), (0, 0, Z), 80, 56)          # ceiling
    b.grid((0, 0, 0), (X, 0, 0), (0, Y, 0), 80, 14)          # walls
    b.grid((0, 0, Z), (0, Y, 0), (X, 0, 0), 14, 80)
    b.grid((0, 0, 0), (0, Y, 0), (0, 0, Z), 14, 56)
    b.grid((X, 0, 0), (0, 0, Z), (0, Y, 0), 56, 14)
    rng = Pcg32(seed)
    for t in range(tables):
        cx = 2.5 + (t % 4) * 5.0 + rng.uniform(-0.3, 0.3)
        cz = 2.5 + (t // 4) * 4.5 + rng.uniform(-0.3, 0.3)
        b.box((cx - 1.4, 0.72, cz - 0.7), (cx + 1.4, 0.76, cz + 0.7), 6)
        for lx in (-1.2, 1.2):
            for lz in (-0.5, 0.5):
                b.cylinder((cx + lx, 0.0, cz + lz), (0, 1, 0), 0.04, 0.72, 24, rings=6)
    for c in range(chairs):
        t = c % tables
        cx = 2.5 + (t % 4) * 5.0 + rng.uniform(-1.6, 1.6)
        cz = 2.5 + (t // 4) * 4.5 + (1.0 if rng.uniform() < 0.5 else -1.5)
        s = 0.45
        b.box((cx, 0.44, cz), (cx + s, 0.48, cz + s), 6)
        b.box((cx, 0.48, cz + s - 0.05), (cx + s, 0.95, cz + s), 6)
        for lx in (0.0, s - 0.04):
            for lz in (0.0, s - 0.04):
                b.cylinder((cx + lx + 0.02, 0.0, cz + lz + 0.02), (0, 1, 0), 0.02, 0.44, 12, rings=2)
    pos, tris = b.build()
    return SceneData("meeting", pos, tris, up=(0.0, 1.0, 0.0),
                     views=[View((1.0, 2.2, 1.0), (10.0, 0.8, 7.0), 65.0)],
                     point_light=(10.0, 3.2, 7.0),
                     area_light=((10.0, 3.4, 7.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0)))


SCENES = {"room": room, "plant": plant, "analytic": analytic, "building": building, "meeting": meeting_room,
          "sphere": displaced_sphere}

"""Serving: resident scenes, continuous batching, admission by a device
memory budget, p50/p99 latency -- a thin Python front over the library's
own request loop (bt_gpu_serve_start / bt_gpu_submit / bt_gpu_poll in
include/bt_gpu.h; no counterpart in the reference).

Requests -- primary visibility (per-pixel hit-triangle ids), point shadows
(per-pixel shadow mask) or exact area-light soft shadows, each for a camera
and resolution on one resident scene -- arrive at any time through
`Server.submit`.  All scenes live in one context's scene pool with their
kd-trees for the server's lifetime.  Inside the library:

* soft-shadow requests share a streaming engine run on the soft lane:
  those that arrive while the run is young are folded into the rounds in
  flight, and each is handed back as soon as its own roots are done;
* primary and point requests run on `vis_lanes` lanes (engine buffers and a
  CUDA stream each), overlapping each other and the soft run on the GPU;
* admission refuses a request (BT_ERR_BUSY) while the resident scenes, the
  lanes' sub-beam queue high-water mark and the admitted requests would
  exceed the memory budget; refused requests wait here, in arrival order,
  and are submitted again as completions free memory.

Results do not depend on what else is in flight: the engine accumulates in
fixed point and a job gives bitwise the same result alone or in a run.

Scenes are given as generated scenes, prepared scenes, or paths of the
reference's scene configs; configs go through a SceneCache
(beamtrace2007_b200.ingest), so a scene ingested and prepared once -- its
kd-tree build is the host work that gates admission -- is admitted again
from the cache directory.
"""
from __future__ import annotations

import collections
import ctypes as C
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

KINDS = ("primary", "point", "soft")
_KIND_CODE = {"primary": N.BT_REQ_PRIMARY_IDS, "point": N.BT_REQ_POINT_MASK, "soft": N.BT_REQ_SOFT}
BT_ERR_BUSY = -7


@dataclass
class Request:
    kind: str                 # "primary" | "point" | "soft"
    scene: str
    W: int
    H: int
    view: int = 0
    light_scale: float = 1.0  # soft: area light scale
    exact: bool = True        # soft: Lambert integral over the visible light
    tile: int = 0             # primary / point: the tile it ran with (set by the server)
    arrival: float = 0.0      # perf_counter seconds, set by submit
    done: float = 0.0
    ms_queued: float = 0.0    # in the library: submit to start (soft: to joining a run)
    result: object = None
    error: str | None = None
    event: threading.Event = field(default_factory=threading.Event)

    @property
    def pixels(self) -> int:
        return self.W * self.H

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def primary_tile(r: Request) -> int:
    """Pixels per side of a primary root when the scene and size were not
    tuned: 4 from 512 pixels up, 2 below.  The reference's 16 leaves too few
    roots to fill the GPU on dense meshes, and a smaller root beam splits
    fewer times in sequence: the displaced sphere's primary ids at 256^2 in
    20 ms at tile 1, 24 at 2, 33 at 4 and 124 at 16; at 1024^2 in 18.5 ms at
    2 and 20 at 4."""
    return 4 if min(r.W, r.H) >= 512 else 2


class _Scene:
    def __init__(self, name, data, prepared, sid):
        self.name = name
        self.data = data
        self.prepared = prepared
        self.id = sid


class Server:
    """Resident scenes on one GPU behind the library's request loop."""

    def __init__(self, scenes: dict, memory_budget_gb: float = 8.0, device: int = 0, queue_records: int = 1 << 25,
                 cache=None, kd_on_gpu: bool = True, vis_lanes: int = 4, fold_ms: float = 100.0,
                 soft_pixels: int = 8 << 20, soft_blocks_per_sm: int = 0):
        from .ingest import SceneCache
        from .renderer import GpuRenderer, PreparedScene
        kd_device = device if kd_on_gpu else None
        self.cache = cache if cache is not None else SceneCache(kd_device=kd_device)
        self.prep_ms: dict = {}   # scene -> ms to admit it (ingest, finalise, kd-tree)
        self.budget = int(memory_budget_gb * (1 << 30))
        self.device = device
        self.scenes: dict[str, _Scene] = {}
        self.engine = None
        for name, sd in scenes.items():
            t0 = time.perf_counter()
            if isinstance(sd, str):  # a scene config: ingested and prepared through the cache
                sd, ps = self.cache.get(sd)
            else:
                ps = sd if isinstance(sd, PreparedScene) else PreparedScene(sd.pos, sd.tris, kd_device=kd_device)
            if self.engine is None:
                self.engine = GpuRenderer(ps, device=device, capacity=queue_records)
                sid = 0
            else:
                sid = self.engine.add_scene(ps)
            self.prep_ms[name] = (time.perf_counter() - t0) * 1e3
            self.scenes[name] = _Scene(name, sd, ps, sid)
        cfg = N.ServeConfig(vis_lanes=vis_lanes, soft_jobs=256, soft_pixels=soft_pixels, capacity=queue_records,
                            fold_ms=fold_ms, memory_budget=self.budget, soft_blocks_per_sm=soft_blocks_per_sm)
        N.check(N.lib().bt_gpu_serve_start(self.engine._h, C.byref(cfg)))
        self.tiles: dict = {}   # (kind, scene, W, H) -> root tile chosen by `tune`
        self.lock = threading.Lock()
        self.inflight: dict[int, tuple] = {}   # ticket -> (request, its C struct and output arrays)
        self.waiting: collections.deque[Request] = collections.deque()  # refused for memory, in arrival order
        self.refusals = 0
        self.running = True
        self.poller = threading.Thread(target=self._poll, daemon=True)
        self.poller.start()

    @property
    def slots(self):
        return self.scenes

    def tune(self, sizes=(256, 512, 1024), tiles=(1, 2, 4, 8, 16), reps: int = 2, max_roots: int = 1 << 18,
             kinds=("primary", "point")):
        """Autotunes the root tile of every resident scene at each square
        size, for primary-id and for point-mask requests (a point request
        also traces a point-shadow root per primary polygon, and smaller
        tiles make more polygons): each candidate request is timed through
        the serving lanes (the fastest of `reps` after a warm-up); tiles that
        would make more than `max_roots` roots are not tried.  Call before
        the stream starts.  Untuned sizes use `primary_tile`."""
        out = {}
        for kind in kinds:
            for name in self.scenes:
                for W in sizes:
                    ms = {}
                    for tile in [t for t in tiles if (-(-W // t)) ** 2 <= max_roots] or [max(tiles)]:
                        t = []
                        for _ in range(reps + 1):
                            r = self.submit(Request(kind, name, W, W, tile=tile))
                            r.event.wait()
                            t.append(r.latency * 1e3)
                        ms[tile] = float(np.min(t[1:]))
                    best = min(ms, key=ms.get)
                    self.tiles[(kind, name, W, W)] = best
                    key = f"{name}/{W}" if kind == "primary" else f"{kind}:{name}/{W}"
                    out[key] = {"tile": best, "ms": {k: round(v, 2) for k, v in ms.items()}}
        return out

    def camera(self, r: Request):
        from .renderer import make_camera
        sc = self.scenes[r.scene]
        v = sc.data.views[r.view]
        return make_camera(v.eye, v.target, v.fov, sc.data.up, r.W, r.H)

    _camera = camera

    # ---- requests ----
    def submit(self, r: Request) -> Request:
        if r.kind not in KINDS or r.scene not in self.scenes:
            raise ValueError(f"bad request {r.kind} / {r.scene}")
        r.arrival = time.perf_counter()
        if r.kind != "soft" and not r.tile:
            r.tile = (self.tiles.get((r.kind, r.scene, r.W, r.H)) or self.tiles.get(("primary", r.scene, r.W, r.H))
                      or primary_tile(r))
        with self.lock:
            if self.waiting or not self._submit(r):
                self.waiting.append(r)
        return r

    def _submit(self, r: Request) -> bool:
        """Hands a request to the library (called with self.lock held);
        False when it is refused for memory now."""
        sc = self.scenes[r.scene]
        q = N.Request()
        q.kind = _KIND_CODE[r.kind]
        q.scene = sc.id
        q.cam = self.camera(r)
        n = r.W * r.H
        keep = []
        if r.kind == "soft":
            L = N.AreaLight.from_array(sc.data.light_array(r.light_scale))
            q.light = L
            q.opts = N.SoftOpts(int(r.exact), 0.0)
            keep = [np.zeros(n, np.int32)] + [np.zeros(n, np.float32) for _ in range(3)]
            q.tri, q.vis, q.E, q.Eu = (N.ptr(a) for a in keep)
        else:
            q.cull = 0
            q.tile = r.tile
            q.point_light[:] = [float(x) for x in sc.data.point_light] if r.kind == "point" else [0.0, 0.0, 0.0]
            keep = [np.zeros(n, np.int32), np.zeros(n, np.uint8)]
            q.tri = N.ptr(keep[0])
            q.mask = N.ptr(keep[1]) if r.kind == "point" else None
        ticket = C.c_uint64()
        rc = N.lib().bt_gpu_submit(self.engine._h, C.byref(q), C.byref(ticket))
        if rc == BT_ERR_BUSY:
            self.refusals += 1
            return False
        if rc != N.BT_OK:
            r.error = N.lib().bt_gpu_last_error().decode(errors="replace")
            r.done = time.perf_counter()
            r.event.set()
            return True
        self.inflight[ticket.value] = (r, q, keep)
        return True

    def _poll(self):
        comps = (N.Completion * 64)()
        count = C.c_int32()
        while self.running:
            N.lib().bt_gpu_poll(self.engine._h, comps, 64, C.byref(count), 50)
            now = time.perf_counter()
            with self.lock:
                for k in range(count.value):
                    c = comps[k]
                    r, q, keep = self.inflight.pop(c.ticket)
                    r.ms_queued = c.ms_queued
                    if c.status != N.BT_OK:
                        r.error = c.error.decode(errors="replace")
                    elif r.kind == "soft":
                        from .renderer import SoftResult
                        r.result = SoftResult(*keep)
                    elif r.kind == "primary":
                        r.result = keep[0].reshape(r.H, r.W)
                    else:
                        r.result = keep[1].reshape(r.H, r.W)
                    r.done = now
                    r.event.set()
                # refused requests again, in arrival order, while they are admitted
                while self.waiting and self._submit(self.waiting[0]):
                    self.waiting.popleft()

    def stats(self) -> dict:
        st = N.ServeStats()
        N.check(N.lib().bt_gpu_serve_stats(self.engine._h, C.byref(st)))
        d = st.as_dict()
        d["waiting_here"] = len(self.waiting)
        d["refusals"] = self.refusals
        return d

    def close(self):
        if not self.running:
            return
        deadline = time.perf_counter() + 600
        while (self.inflight or self.waiting) and time.perf_counter() < deadline:
            time.sleep(0.01)
        self.running = False
        self.poller.join(timeout=60)
        self.engine.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def poisson_stream(server: Server, rate: float, n: int, mix=(0.60, 0.25, 0.15), sizes=(256, 512, 1024),
                   scenes=None, seed: int = 1, light_scales=(0.5, 1.0, 2.0)):
    """Submits n requests with exponential inter-arrival times (rate per
    second), kinds drawn from `mix` (primary, point, soft), square
    resolutions from `sizes`, scenes uniformly; waits for all and returns
    (requests, summary).  `offered_s` is the submission window; a rate is
    sustained when the requests finish within about that window."""
    rng = np.random.default_rng(seed)
    names = list(scenes or server.scenes.keys())
    reqs = []
    t0 = time.perf_counter()
    t_next = t0
    for _ in range(n):
        t_next += rng.exponential(1.0 / rate)
        kind = KINDS[int(rng.choice(3, p=np.asarray(mix) / np.sum(mix)))]
        s = int(rng.choice(sizes))
        r = Request(kind, names[int(rng.integers(len(names)))], s, s,
                    light_scale=float(rng.choice(light_scales)))
        delay = t_next - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        reqs.append(server.submit(r))
    t_sub = time.perf_counter()
    for r in reqs:
        r.event.wait()
    t_end = max(r.done for r in reqs)
    lat = np.array([r.latency for r in reqs])
    px = sum(r.pixels for r in reqs)
    summary = {"requests": n, "rate_req_s": rate, "p50_ms": float(np.percentile(lat, 50) * 1e3),
               "p99_ms": float(np.percentile(lat, 99) * 1e3), "max_ms": float(lat.max() * 1e3),
               "px_per_s": px / (t_end - t0), "req_per_s": n / (t_end - t0), "offered_s": t_sub - t0,
               "span_s": t_end - t0, "errors": sum(r.error is not None for r in reqs),
               "by_kind": {k: int(sum(r.kind == k for r in reqs)) for k in KINDS},
               "p50_ms_by_kind": {k: float(np.percentile([r.latency for r in reqs if r.kind == k], 50) * 1e3)
                                  for k in KINDS if any(r.kind == k for r in reqs)}}
    return reqs, summary

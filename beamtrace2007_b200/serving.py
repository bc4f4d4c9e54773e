"""Serving loop: resident scenes, continuous batching, admission by a device
memory budget, p50/p99 latency (no counterpart in the reference).

Requests -- primary visibility (per-pixel hit-triangle ids), point shadows
(per-pixel shadow mask) or exact area-light soft shadows, each for a camera
and resolution on one resident scene -- arrive at any time through
`Server.submit`.  Every resident scene keeps its kd-tree and
`workers_per_scene` engine contexts on the GPU for the server's lifetime;
each context has its own CUDA stream and worker thread, so requests of
different scenes, and of one scene, run on the device at the same time.  A
free worker takes its scene's oldest admitted request: if that is a soft-
shadow request, together with every other soft-shadow request waiting for
the scene, in one batched engine run (bt_gpu_batch_soft, whose roots share
the rounds); otherwise that request alone.  So a short primary request does
not wait behind a long soft-shadow batch while another worker is free.

Admission: the resident scenes and their sub-beam queues are charged to the
budget at start; a request is admitted, in arrival order, when its own
device memory (outputs, per-pixel scratch, roots) fits in what is left, and
released when it completes.

Results do not depend on what else is in flight: the engine accumulates in
fixed point and the batch path is bitwise the single-job path.

Scenes are given as generated scenes, prepared scenes, or paths of the
reference's scene configs; configs go through a SceneCache
(beamtrace2007_b200.ingest), so a scene ingested and prepared once -- its
kd-tree build is the host work that gates admission -- is admitted again
from the cache directory.
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass, field

import numpy as np

KINDS = ("primary", "point", "soft")


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
    result: object = None
    error: str | None = None
    event: threading.Event = field(default_factory=threading.Event)

    @property
    def pixels(self) -> int:
        return self.W * self.H

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def request_bytes(r: Request) -> int:
    """Device memory a request holds while it runs: outputs and per-pixel
    scratch (tri, X, N, vis, E, Eu) and, per root, the engine's root state
    (soft: one root per pixel; primary and point: polygon lists)."""
    px = r.W * r.H
    if r.kind == "soft":
        return px * (4 + 12 + 12 + 12 + 164)
    return px * (2 * 44 + 16) + (px // 256 + 1) * 164


def primary_tile(r: Request) -> int:
    """Pixels per side of a primary root: 16 (the reference's tile) from 512
    pixels up; 8 below, where 16 leaves too few roots to fill the GPU
    (measured on the served scenes: 69 vs 142 ms at 256^2)."""
    return 16 if min(r.W, r.H) >= 512 else 8


class _SceneSlot:
    def __init__(self, name, scene_data, engines):
        self.name = name
        self.data = scene_data
        self.engines = engines
        self.pending: collections.deque[Request] = collections.deque()
        self.cv = threading.Condition()
        self.threads: list[threading.Thread] = []

    @property
    def engine(self):
        return self.engines[0]

    def take(self) -> list:
        """The oldest pending request, with every other pending soft-shadow
        request when it is one (called with cv held)."""
        head = self.pending.popleft()
        if head.kind != "soft":
            return [head]
        batch = [head] + [r for r in self.pending if r.kind == "soft"]
        self.pending = collections.deque(r for r in self.pending if r.kind != "soft")
        return batch


class Server:
    """Resident scenes on one GPU.  `engine_factory(prepared_scene, capacity)`
    builds a context (GpuRenderer by default; tests may pass a stand-in)."""

    def __init__(self, scenes: dict, memory_budget_gb: float = 8.0, device: int = 0, queue_records: int = 1 << 21,
                 engine_factory=None, cache=None, kd_on_gpu: bool = True, workers_per_scene: int = 2):
        from .ingest import SceneCache
        from .renderer import GpuRenderer, PreparedScene
        kd_device = device if kd_on_gpu else None
        self.cache = cache if cache is not None else SceneCache(kd_device=kd_device)
        self.prep_ms: dict = {}   # scene -> ms to admit it (ingest, finalise, kd-tree)
        self.budget = int(memory_budget_gb * (1 << 30))
        self.device = device
        if engine_factory is None:
            def engine_factory(ps, capacity):
                return GpuRenderer(ps, device=device, capacity=capacity)
        self.slots: dict[str, _SceneSlot] = {}
        self.resident = 0
        for name, sd in scenes.items():
            t0 = time.perf_counter()
            if isinstance(sd, str):  # a scene config: ingested and prepared through the cache
                sd, ps = self.cache.get(sd)
            else:
                ps = sd if isinstance(sd, PreparedScene) else PreparedScene(sd.pos, sd.tris, kd_device=kd_device)
            self.prep_ms[name] = (time.perf_counter() - t0) * 1e3
            # each context holds the scene, its tree and its queues
            per = 44 * len(ps.kd_split) + 64 * len(ps.kd_tri_indices) + 32 * ps.num_tris + 3 * 64 * queue_records
            self.resident += per * workers_per_scene
            slot = _SceneSlot(name, sd, [engine_factory(ps, queue_records) for _ in range(workers_per_scene)])
            self.slots[name] = slot
        if self.resident > self.budget:
            raise ValueError(f"resident scenes and queues need {self.resident / 2**30:.2f} GiB, "
                             f"over the {memory_budget_gb} GiB budget")
        self.tiles: dict = {}   # (scene, W, H) -> primary tile chosen by `tune`
        self.in_use = 0
        self.lock = threading.Lock()
        self.waiting: collections.deque[Request] = collections.deque()
        self.running = True
        for slot in self.slots.values():
            for eng in slot.engines:
                t = threading.Thread(target=self._worker, args=(slot, eng), daemon=True)
                slot.threads.append(t)
                t.start()

    def tune(self, sizes=(256, 512, 1024), tiles=(8, 16, 32)):
        """Autotunes the primary tile of every resident scene at each square
        size (autotune.tune_tile); call before the stream starts (it uses the
        scenes' contexts).  Untuned sizes use `primary_tile`."""
        from .autotune import tune_tile
        out = {}
        for name, slot in self.slots.items():
            for W in sizes:
                r = Request("primary", name, W, W)
                best, t = tune_tile(slot.engine, self._camera(slot, r), tiles)
                self.tiles[(name, W, W)] = best
                out[f"{name}/{W}"] = {"tile": best, "ms": {k: round(v * 1e3, 2) for k, v in t.items()}}
        return out

    # ---- admission ----
    def submit(self, r: Request) -> Request:
        if r.kind not in KINDS or r.scene not in self.slots:
            raise ValueError(f"bad request {r.kind} / {r.scene}")
        if request_bytes(r) > self.budget - self.resident:
            raise ValueError("request larger than the memory budget")
        r.arrival = time.perf_counter()
        with self.lock:
            self.waiting.append(r)
            self._admit()
        return r

    def _admit(self):
        # in arrival order, while the head fits (called with self.lock held)
        while self.waiting:
            r = self.waiting[0]
            need = request_bytes(r)
            if self.resident + self.in_use + need > self.budget:
                break
            self.waiting.popleft()
            self.in_use += need
            slot = self.slots[r.scene]
            with slot.cv:
                slot.pending.append(r)
                slot.cv.notify()

    def _release(self, reqs):
        with self.lock:
            for r in reqs:
                self.in_use -= request_bytes(r)
            self._admit()

    # ---- execution ----
    def _worker(self, slot: _SceneSlot, engine):
        while True:
            with slot.cv:
                while self.running and not slot.pending:
                    slot.cv.wait(0.05)
                if not self.running and not slot.pending:
                    return
                batch = slot.take()
            try:
                self._run(slot, engine, batch)
            except Exception as e:  # a failed run fails its requests, not the server
                for r in batch:
                    if r.result is None:
                        r.error = f"{type(e).__name__}: {e}"
            now = time.perf_counter()
            for r in batch:
                r.done = now if r.done == 0.0 else r.done
            self._release(batch)
            for r in batch:
                r.event.set()

    def _camera(self, slot, r):
        from .renderer import make_camera
        v = slot.data.views[r.view]
        return make_camera(v.eye, v.target, v.fov, slot.data.up, r.W, r.H)

    def _run(self, slot: _SceneSlot, engine, batch):
        soft = [r for r in batch if r.kind == "soft"]
        if soft:
            cams = [self._camera(slot, r) for r in soft]
            lights = [slot.data.light_array(r.light_scale) for r in soft]
            res = engine.batch_soft(cams, lights, exact=soft[0].exact) if all(
                r.exact == soft[0].exact for r in soft) else None
            if res is None:
                res = [engine.soft_shadows(c, L, exact=r.exact) for c, L, r in zip(cams, lights, soft)]
            now = time.perf_counter()
            for r, x in zip(soft, res):
                r.result = x
                r.done = now
        for r in batch:
            if r.kind == "soft":
                continue
            cam = self._camera(slot, r)
            tile = r.tile = self.tiles.get((r.scene, r.W, r.H)) or primary_tile(r)
            if r.kind == "primary":
                r.result = engine.primary_ids(cam, tile=tile)
            else:
                r.result = engine.point_mask(cam, np.asarray(slot.data.point_light, np.float32), tile=tile)[1]
            r.done = time.perf_counter()

    def close(self):
        self.running = False
        for slot in self.slots.values():
            with slot.cv:
                slot.cv.notify_all()
            for t in slot.threads:
                t.join(timeout=60)
            for eng in slot.engines:
                close = getattr(eng, "close", None)
                if close:
                    close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def poisson_stream(server: Server, rate: float, n: int, mix=(0.60, 0.25, 0.15), sizes=(256, 512, 1024),
                   scenes=None, seed: int = 1, light_scales=(0.5, 1.0, 2.0)):
    """Submits n requests with exponential inter-arrival times (rate per
    second), kinds drawn from `mix` (primary, point, soft), square
    resolutions from `sizes`, scenes uniformly; waits for all and returns
    (requests, summary)."""
    rng = np.random.default_rng(seed)
    names = list(scenes or server.slots.keys())
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
    for r in reqs:
        r.event.wait()
    t_end = max(r.done for r in reqs)
    lat = np.array([r.latency for r in reqs])
    px = sum(r.pixels for r in reqs)
    summary = {"requests": n, "rate_req_s": rate, "p50_ms": float(np.percentile(lat, 50) * 1e3),
               "p99_ms": float(np.percentile(lat, 99) * 1e3), "px_per_s": px / (t_end - t0),
               "errors": sum(r.error is not None for r in reqs),
               "by_kind": {k: int(sum(r.kind == k for r in reqs)) for k in KINDS}}
    return reqs, summary

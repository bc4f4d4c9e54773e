"""The serving loop (beamtrace2007_b200/serving.py): admission by memory
budget and continuous batching (CPU, with a stand-in engine), and on the
GPU a mixed Poisson stream over three resident scenes whose every result is
bitwise the result of the same request run alone."""
import threading
import time

import numpy as np
import pytest

from conftest import scene


class FakeEngine:
    """Stands in for a GpuRenderer: records what ran together."""
    log = []
    lock = threading.Lock()

    def __init__(self, ps, capacity):
        self.ps = ps

    def _note(self, what):
        with FakeEngine.lock:
            FakeEngine.log.append(what)
        time.sleep(0.02)

    def batch_soft(self, cams, lights, exact=True):
        self._note(("batch", len(cams)))
        from beamtrace2007_b200.renderer import SoftResult
        return [SoftResult(np.zeros(c.W * c.H, np.int32), np.full(c.W * c.H, float(L[0]), np.float32),
                           np.zeros(c.W * c.H, np.float32), np.zeros(c.W * c.H, np.float32)) for c, L in
                zip(cams, lights)]

    def soft_shadows(self, cam, L, exact=True):
        return self.batch_soft([cam], [L], exact)[0]

    def primary(self, cam, tile=16):
        self._note(("primary", cam.W))
        return None

    def primary_ids(self, cam, tile=16):
        self._note(("primary", cam.W))
        return np.full((cam.H, cam.W), cam.W, np.int32)

    def point_mask(self, cam, light, tile=16):
        self._note(("point", cam.W))
        return np.full((cam.H, cam.W), cam.W, np.int32), np.zeros((cam.H, cam.W), np.uint8)

    def point_shadows(self, cam, prim, light):
        return None

    def raster(self, cam, prim, sh):
        return np.full(cam.W * cam.H, cam.W, np.int32), np.zeros(cam.W * cam.H, np.uint8)

    def close(self):
        pass


def test_admission_and_batching(native_lib):
    from beamtrace2007_b200.serving import Request, Server, request_bytes
    s, ps = scene("room")
    scenes = {"a": s, "b": s}
    FakeEngine.log = []
    # a budget that holds the resident part and about eight 128^2 soft requests
    probe = Request("soft", "a", 128, 128)
    with Server(scenes, memory_budget_gb=1.0, queue_records=1 << 10, engine_factory=FakeEngine,
                kd_on_gpu=False) as srv:
        srv.budget = srv.resident + 8 * request_bytes(probe)
        peak = [0]
        reqs = []
        for i in range(24):
            r = Request("soft" if i % 3 else "primary", "ab"[i % 2], 128, 128, light_scale=1.0 + i)
            reqs.append(srv.submit(r))
            peak[0] = max(peak[0], srv.in_use)
        for r in reqs:
            assert r.event.wait(30)
        assert srv.in_use == 0
    assert peak[0] <= 8 * request_bytes(probe)
    assert all(r.error is None and r.done >= r.arrival for r in reqs)
    # soft requests that waited together ran as one batch at least once
    assert any(k == "batch" and n > 1 for k, n in FakeEngine.log)
    for r in reqs:
        if r.kind == "soft":
            assert r.result.vis[0] == np.float32(r.result.vis[0])


class SlowSoftEngine(FakeEngine):
    """A stand-in whose soft-shadow batches take 0.3 s."""

    def batch_soft(self, cams, lights, exact=True):
        time.sleep(0.3)
        return super().batch_soft(cams, lights, exact)


@pytest.mark.parametrize("workers", [1, 2])
def test_primary_does_not_wait_behind_a_soft_batch(native_lib, workers):
    """With two workers per scene, a primary request that arrives while a
    long soft-shadow batch runs on the same scene is served by the other
    worker; with one it waits for the batch."""
    from beamtrace2007_b200.serving import Request, Server
    s, _ = scene("room")
    with Server({"a": s}, memory_budget_gb=1.0, queue_records=1 << 10, engine_factory=SlowSoftEngine,
                kd_on_gpu=False, workers_per_scene=workers) as srv:
        soft = srv.submit(Request("soft", "a", 64, 64))
        time.sleep(0.05)
        prim = srv.submit(Request("primary", "a", 64, 64))
        assert soft.event.wait(30) and prim.event.wait(30)
    assert soft.error is None and prim.error is None
    if workers == 2:
        assert prim.done < soft.done and prim.latency < 0.2
    else:
        assert prim.done >= soft.done


def test_config_scenes_through_the_cache(native_lib, tmp_path):
    """Scenes given as the reference's configs are ingested and prepared
    once; a second server on the same cache directory admits them from the
    stored arrays.  Requests use the config's views and lights."""
    from beamtrace2007_b200.ingest import SceneCache
    from beamtrace2007_b200.serving import Request, Server
    cfg = tmp_path / "room.cfg"
    cfg.write_text("name room\nmesh procedural room\nup 0 1 0\norbit 4 1.2 4  2.8 0.7 8 70\n"
                   "point_light 5.5 2.6 2.5\narea_light 4 2.95 4  1 0 0  0 0 1\n")
    store = str(tmp_path / "cache")
    results = []
    for run in range(2):
        cache = SceneCache(store)
        with Server({"room": str(cfg)}, memory_budget_gb=1.0, queue_records=1 << 10, engine_factory=FakeEngine,
                    cache=cache, kd_on_gpu=False) as srv:
            slot = srv.slots["room"]
            assert len(slot.data.views) == 8
            assert np.array_equal(np.float32(slot.data.point_light), np.float32([5.5, 2.6, 2.5]))
            reqs = [srv.submit(Request(k, "room", 64, 48, view=3)) for k in ("primary", "point", "soft")]
            for r in reqs:
                assert r.event.wait(30) and r.error is None
            results.append([r.result for r in reqs])
        assert (cache.misses, cache.disk_hits) == ((1, 0) if run == 0 else (0, 1))
    assert np.array_equal(results[0][0], results[1][0])


@pytest.mark.gpu
def test_mixed_stream_same_as_alone(gpu):
    from beamtrace2007_b200.serving import Server, poisson_stream
    scenes = {"room": scene("room")[0], "plant": scene("plant")[0],
              "building": scene("building", floors=1, furniture=2)[0]}
    with Server(scenes, memory_budget_gb=8.0) as srv:
        tuned = srv.tune(sizes=(64, 128), tiles=(8, 16))
        assert set(tuned) == {f"{s}/{w}" for s in scenes for w in (64, 128)}
        reqs, summary = poisson_stream(srv, rate=200.0, n=30, sizes=(64, 96, 128), seed=3)
        assert summary["errors"] == 0, [r.error for r in reqs if r.error]
        assert summary["p99_ms"] >= summary["p50_ms"] > 0
        # each request again, alone, on the same resident scene
        for r in reqs:
            slot = srv.slots[r.scene]
            cam = srv._camera(slot, r)
            if r.kind == "soft":
                alone = slot.engine.soft_shadows(cam, slot.data.light_array(r.light_scale), exact=r.exact)
                for k in ("tri", "vis", "E", "Eu"):
                    assert np.array_equal(getattr(r.result, k), getattr(alone, k)), (r.kind, k)
            else:
                # alone, and through the host polygon path
                prim = slot.engine.primary(cam, tile=r.tile)
                if r.kind == "primary":
                    tri, _ = slot.engine.raster(cam, prim, None)
                    assert np.array_equal(r.result, tri)
                else:
                    sh = slot.engine.point_shadows(cam, prim, np.asarray(slot.data.point_light, np.float32))
                    _, flag = slot.engine.raster(cam, prim, sh)
                    assert np.array_equal(r.result, flag)


@pytest.mark.gpu
def test_autotune_engine_settings(gpu):
    """tune_engine times each candidate context and returns the fastest; the
    frame it renders is the same for every candidate."""
    from beamtrace2007_b200.autotune import tune_engine
    from beamtrace2007_b200.renderer import GpuRenderer, make_camera
    s, ps = scene("plant")
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, 96, 96)
    best, timings = tune_engine(ps, cam, s.light_array(), blocks_per_sm=(0, 1), tail_records=(0, -1),
                                yield_pcts=(0, -1), reps=1)
    assert len(timings) == 8 and all(t > 0 for t in timings.values())
    assert (best["blocks_per_sm"], best["tail_records"], best["capacity"], best["yield_pct"]) == min(
        timings, key=timings.get)
    with GpuRenderer(ps, **best) as g1, GpuRenderer(ps, blocks_per_sm=1, tail_records=-1, yield_pct=-1) as g2:
        a = g1.soft_shadows(cam, s.light_array(), exact=True)
        b = g2.soft_shadows(cam, s.light_array(), exact=True)
    assert np.array_equal(a.vis, b.vis) and np.array_equal(a.E, b.E)

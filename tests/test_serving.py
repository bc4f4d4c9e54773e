"""Serving (bt_gpu_serve_start / bt_gpu_submit / bt_gpu_poll and the Python
front, beamtrace2007_b200/serving.py): continuous batching with soft
requests folded into a running engine run, lanes that overlap, admission by
a memory budget, and every result bitwise the result of the same request
run alone.  The argument checks run without a GPU; the rest on the GPU,
including a C host (tests/native/serve_c_test.c) that submits and polls
three mixed requests."""
import ctypes as C
import os
import subprocess
import time

import numpy as np
import pytest

from conftest import ROOT, scene


def test_serving_arguments_without_a_gpu(native_lib):
    """Bad calls return status codes (no context here: nothing to serve)."""
    from beamtrace2007_b200 import _native as N
    q = N.Request()
    t = C.c_uint64()
    assert native_lib.bt_gpu_submit(None, C.byref(q), C.byref(t)) == -1
    assert native_lib.bt_gpu_serve_start(None, None) == -1
    cnt = C.c_int32(5)
    assert native_lib.bt_gpu_poll(None, None, 0, C.byref(cnt), 0) == -1 and cnt.value == 0
    assert native_lib.bt_gpu_serve_stats(None, None) == -1


def _alone(srv, r):
    """The request alone: soft shadows as a one-job batch on the server's
    own context (bitwise the single-job path), primary ids and point masks
    on a fresh context whose only scene is the request's."""
    from beamtrace2007_b200.renderer import GpuRenderer
    sc = srv.scenes[r.scene]
    cam = srv.camera(r)
    if r.kind == "soft":
        [res] = [x for x in srv.engine.batch_soft([cam], [sc.data.light_array(r.light_scale)], exact=r.exact,
                                                  scenes=[sc.id])]
        return res
    with GpuRenderer(sc.prepared, capacity=1 << 20) as g:
        if r.kind == "primary":
            return g.primary_ids(cam, tile=r.tile)
        return g.point_mask(cam, np.asarray(sc.data.point_light, np.float32), tile=r.tile)[1]


def _same(r, alone):
    if r.kind == "soft":
        return all(np.array_equal(getattr(r.result, k), getattr(alone, k)) for k in ("tri", "vis", "E", "Eu"))
    return np.array_equal(r.result, alone)


@pytest.mark.gpu
def test_mixed_stream_same_as_alone(gpu):
    from beamtrace2007_b200.serving import Server, poisson_stream
    scenes = {"room": scene("room")[0], "plant": scene("plant")[0],
              "building": scene("building", floors=1, furniture=2)[0]}
    with Server(scenes, memory_budget_gb=8.0) as srv:
        tuned = srv.tune(sizes=(64, 128), tiles=(8, 16), reps=1)
        assert set(tuned) == ({f"{s}/{w}" for s in scenes for w in (64, 128)}
                              | {f"point:{s}/{w}" for s in scenes for w in (64, 128)})
        reqs, summary = poisson_stream(srv, rate=200.0, n=40, sizes=(64, 96, 128), seed=3)
        assert summary["errors"] == 0, [r.error for r in reqs if r.error]
        assert summary["p99_ms"] >= summary["p50_ms"] > 0
        for r in reqs:
            assert _same(r, _alone(srv, r)), (r.kind, r.scene, r.W)


@pytest.mark.gpu
def test_soft_requests_fold_into_a_running_run(gpu):
    """Soft requests submitted while a long soft run is going join it (the
    library counts them as folded) and are handed back before it ends; each
    equals the request alone."""
    from beamtrace2007_b200.serving import Request, Server
    with Server({"plant": scene("plant")[0]}, memory_budget_gb=8.0, fold_ms=10_000.0) as srv:
        big = srv.submit(Request("soft", "plant", 512, 512, light_scale=4.0))
        time.sleep(0.004)
        small = [srv.submit(Request("soft", "plant", 48, 48, view=0, light_scale=0.5 + 0.25 * i)) for i in range(6)]
        for r in [big] + small:
            assert r.event.wait(120) and r.error is None, r.error
        st = srv.stats()
        assert st["soft_folded"] >= 1, st
        assert st["soft_runs"] < 1 + len(small), st
        # the small requests that joined the big run came back before it
        assert min(r.done for r in small) < big.done
        for r in [big] + small:
            assert _same(r, _alone(srv, r))


@pytest.mark.gpu
def test_primary_does_not_wait_behind_a_soft_run(gpu):
    """A primary request that arrives while a long soft run is going runs on
    a visibility lane at the same time and comes back first."""
    from beamtrace2007_b200.serving import Request, Server
    with Server({"plant": scene("plant")[0]}, memory_budget_gb=8.0, fold_ms=1.0) as srv:
        # every lane has served a request (its buffers allocated) before the race
        warm = [srv.submit(Request("primary", "plant", 64, 64)) for _ in range(16)]
        warm.append(srv.submit(Request("soft", "plant", 32, 32)))
        assert all(r.event.wait(60) for r in warm)
        soft = srv.submit(Request("soft", "plant", 512, 512, light_scale=4.0))
        time.sleep(0.004)
        prim = srv.submit(Request("primary", "plant", 64, 64))
        assert soft.event.wait(120) and prim.event.wait(120)
        assert soft.error is None and prim.error is None
        assert prim.done < soft.done
        assert _same(prim, _alone(srv, prim))


@pytest.mark.gpu
def test_admission_by_memory_budget(gpu):
    """A budget that holds the resident scene and a few requests: the
    library refuses the rest for a while (BT_ERR_BUSY), the front submits
    them again as memory frees, every request completes and equals the
    request alone, and the memory charged to admitted requests never exceeds
    what the budget leaves."""
    from beamtrace2007_b200.serving import Request, Server
    s, ps = scene("room")
    with Server({"room": s}, memory_budget_gb=8.0, queue_records=1 << 16) as srv:
        scene_bytes = srv.stats()["scene_bytes"]
    one = 128 * 128 * 40 + 128 * 128 * 72   # what admission charges a 128^2 soft request
    budget = scene_bytes + 3 * one + one // 2
    with Server({"room": s}, memory_budget_gb=budget / (1 << 30), queue_records=1 << 16) as srv:
        reqs = [srv.submit(Request("soft" if i % 3 else "primary", "room", 128, 128, light_scale=0.5 + 0.1 * i))
                for i in range(18)]
        peak = 0
        while not all(r.event.is_set() for r in reqs):
            peak = max(peak, srv.stats()["admitted_bytes"])
            time.sleep(0.001)
        assert all(r.error is None for r in reqs), [r.error for r in reqs if r.error]
        st = srv.stats()
        assert st["refused"] > 0 and st["completed"] == len(reqs), st
        assert peak <= budget - scene_bytes, (peak, st)
        for r in reqs:
            assert _same(r, _alone(srv, r))


@pytest.mark.gpu
def test_config_scenes_through_the_cache(gpu, tmp_path):
    """Scenes given as the reference's configs are ingested and prepared
    once; a second server on the same cache directory admits them from the
    stored arrays.  Requests use the config's views and lights and give the
    same results from both."""
    from beamtrace2007_b200.ingest import SceneCache
    from beamtrace2007_b200.serving import Request, Server
    cfg = tmp_path / "room.cfg"
    cfg.write_text("name room\nmesh procedural room\nup 0 1 0\norbit 4 1.2 4  2.8 0.7 8 70\n"
                   "point_light 5.5 2.6 2.5\narea_light 4 2.95 4  1 0 0  0 0 1\n")
    store = str(tmp_path / "cache")
    results = []
    for run in range(2):
        cache = SceneCache(store)
        with Server({"room": str(cfg)}, memory_budget_gb=1.0, queue_records=1 << 16, cache=cache) as srv:
            sc = srv.scenes["room"]
            assert len(sc.data.views) == 8
            assert np.array_equal(np.float32(sc.data.point_light), np.float32([5.5, 2.6, 2.5]))
            reqs = [srv.submit(Request(k, "room", 64, 48, view=3)) for k in ("primary", "point", "soft")]
            for r in reqs:
                assert r.event.wait(60) and r.error is None
            results.append([r.result for r in reqs])
        assert (cache.misses, cache.disk_hits) == ((1, 0) if run == 0 else (0, 1))
    assert np.array_equal(results[0][0], results[1][0]) and np.array_equal(results[0][1], results[1][1])
    assert np.array_equal(results[0][2].vis, results[1][2].vis)


@pytest.mark.gpu
def test_c_host_submits_and_polls(gpu):
    """tests/native/serve_c_test.c, built here against libbt_gpu.so: three
    mixed requests through bt_gpu_submit / bt_gpu_poll, each bitwise the
    synchronous call's result."""
    out = os.path.join(ROOT, "tests", "native", "_serve_c_test")
    src = os.path.join(ROOT, "tests", "native", "serve_c_test.c")
    lib = os.path.join(ROOT, "beamtrace2007_b200")
    subprocess.run(["gcc", "-std=c11", "-O2", "-I" + os.path.join(ROOT, "include"), src, "-L" + lib, "-lbt_gpu",
                    "-Wl,-rpath," + lib, "-o", out], check=True)
    r = subprocess.run([out, "96"], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "serve_c_test: ok" in r.stdout


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


@pytest.mark.gpu
def test_soft_lane_cta_cap_same_results(gpu):
    """soft_blocks_per_sm caps the soft lane's persistent CTAs per SM (room
    for the visibility lanes); results stay bitwise those of the request
    alone."""
    from beamtrace2007_b200.serving import Request, Server
    with Server({"plant": scene("plant")[0]}, memory_budget_gb=8.0, soft_blocks_per_sm=1) as srv:
        reqs = [srv.submit(Request("soft", "plant", 96, 72, light_scale=s)) for s in (0.5, 2.0)]
        reqs.append(srv.submit(Request("primary", "plant", 96, 72)))
        for r in reqs:
            assert r.event.wait(120) and r.error is None, r.error
            assert _same(r, _alone(srv, r))


@pytest.mark.gpu
def test_autotune_trace_ctas(gpu):
    """tune_engine with trace_ctas candidates times each and reports the
    fastest; the frame is the same for 3 and 4 trace CTAs per SM."""
    from beamtrace2007_b200.autotune import tune_engine
    from beamtrace2007_b200.renderer import GpuRenderer, make_camera
    s, ps = scene("plant")
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, 96, 96)
    best, timings = tune_engine(ps, cam, s.light_array(), blocks_per_sm=(0,), tail_records=(0,), trace_ctas=(3, 4),
                                reps=1)
    assert set(timings) == {(0, 0, 0, 0, 3), (0, 0, 0, 0, 4)}
    assert best["trace_ctas"] == min(timings, key=timings.get)[4]
    frames = []
    for tc in (3, 4):
        with GpuRenderer(ps, trace_ctas=tc) as g:
            frames.append(g.soft_shadows(cam, s.light_array(), exact=True))
    assert np.array_equal(frames[0].vis, frames[1].vis) and np.array_equal(frames[0].E, frames[1].E)

"""Benchmark: exact area-light soft shadows at 512x512, pixels per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step = one frame): the seeded plant scene (5418 triangles: a
24-segment stem, 400 leaves of 13 triangles, ground quad), square area light
of side 0.5 m at 3 m, 512x512 pixels, exact Lambert integral (--exact): GPU
primary rays at the pixel centres, then one shadow-beam tree per covered
pixel through the persistent-warp engine.  Synthetic, seeded data.

`value`: pixels/s with the scene resident in HBM, outputs in device memory,
each frame timed with CUDA events on the engine's stream; L2 is flushed
(a 256 MiB write) between timed frames because the scene fits in L2.
`roofline`: the trace kernel (the dominant one), algorithmic bytes per
launch over its launch time from CUDA events recorded between the round
kernels on the engine's stream inside the timed frames (kernel_timing);
`traffic` is the DRAM bytes per launch of the committed ncu capture.
`e2e`: the same frames through bt_gpu_soft with host output buffers (the
GpuRenderer::softShadows contract), wall-clocked per call, device-to-host
copies of tri/vis/E/Eu inside.
`accuracy`: the last timed frame's visibility against the reference's FP64
build on its own shading points (max, mean, histogram of the error), and
the reference's 256-ray sampled visibility's error beside it, computed
after the timed region.
`cpu_baseline` / `--impl reference`: the reference's own CPU tracer
(compiled from its sources, oracle/_ref) on the host's cores; the
reference arm also times the reference's own GPU engine built for sm_100a
(`reference_gpu`) when oracle/_ref/libbtref_gpu.so is present.

Multi-GPU: the frames of different GPUs are independent (replicas only):
each rank renders the workload on its own GPU, `value` = all ranks' pixels /
max-over-ranks time (weak scaling).
"""
from __future__ import annotations

import argparse
import faulthandler
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "soft-shadow px/s at 512² (batched vs plain GPU, ≤1e-4 err); p50/p99 latency"
W = H = 512


def workload_config():
    return {"workload": "plant 5418 tris, exact area-light soft shadows 512x512, plain single-job GPU path",
            "scene": "plant(seed=7, leaves=400)", "resolution": [W, H], "light_side_m": 0.5, "exact": True,
            "l2": "flushed between timed frames (256 MiB write)"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def dist_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_reference(scene, steps: int, warmup: int, min_seconds: float = 10.0, max_frames: int = 1000):
    """The reference CPU tracer (oracle/_ref) on the same frame, all host threads:
    at least `steps` frames and about `min_seconds` of work."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from ref import RefTracer, ref_available
    if not ref_available("f"):
        return None
    threads = os.cpu_count() or 1
    rf = RefTracer(scene.pos, scene.tris, "f")
    v = scene.views[0]
    cam = rf.camera_make(v.eye, v.target, v.fov, scene.up, W, H)  # the reference's Camera::make
    L = scene.light_array()
    for _ in range(warmup):
        rf.soft_image(cam, W, H, L, exact=True, threads=threads)
    times = []
    t_start = time.perf_counter()
    while len(times) < steps or time.perf_counter() - t_start < min_seconds:
        r = rf.soft_image(cam, W, H, L, exact=True, threads=threads)
        times.append(r["primary_s"] + r["trace_s"])
        if len(times) >= max_frames:
            break
    per = float(np.median(times))
    return {"value": W * H / per, "unit": "px/s", "cores": threads, "kind": "reference",
            "sample": f"{len(times)} full {W}x{H} frames (bt_render --mode softshadow --method beam --exact "
                      f"--threads {threads} pipeline: ray primary + beam soft shadows), median frame {per*1e3:.1f} ms",
            "ms_per_frame": per * 1e3}


def accuracy(scene, ps, cam, light, vis, ray_sample: int = 16384):
    """The timed frame's per-result error, outside the timed region: its
    visibility against the reference's FP64 build (bt_render_d --exact) on
    the frame's own shading points, every covered pixel (max, mean and a
    histogram of |vis - fp64|); and, beside it, the error of the reference's
    256-ray sampled visibility (--method ray --samples 256) on an even
    sample of the covered pixels, and the same frame with the opt-in FP64
    re-decision of band corners (eps_fp64): its error and frame time.  The
    FP64 run is timed on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from ref import RefTracer, ref_available
    if not (ref_available("f") and ref_available("d")):
        return None
    threads = os.cpu_count() or 1
    rf = RefTracer(scene.pos, scene.tris, "f")
    rd = RefTracer(scene.pos, scene.tris, "d")
    tri, X, N, _ = rf.primary_rays(cam.as_array(), cam.W, cam.H, threads=threads)
    t0 = time.perf_counter()
    vd, _, _, _ = rd.soft_points(light, ps.offset, tri, X, N, exact=True, threads=threads)
    fp64_s = time.perf_counter() - t0
    cov = np.nonzero(tri >= 0)[0]
    err = np.abs(vis[cov].astype(np.float64) - vd[cov])
    edges = [0.0, 1e-7, 1e-6, 1e-5, 1e-4, 1e-3, np.inf]
    hist, _ = np.histogram(err, bins=edges)
    pick = cov[np.linspace(0, len(cov) - 1, min(ray_sample, len(cov))).astype(np.int64)]
    t0 = time.perf_counter()
    vr = rf.soft_points_ray(light, ps.offset, tri[pick], X[pick], N[pick], pick % cam.W, pick // cam.W, samples=256,
                            threads=threads)
    ray_s = time.perf_counter() - t0
    er = np.abs(vr - vd[pick])
    # the opt-in FP64 re-decision of band corners on the same frame
    from beamtrace2007_b200.renderer import GpuRenderer
    with GpuRenderer(ps, eps_fp64=True) as g64:
        g64.soft_shadows(cam, light, exact=True)
        r64 = [g64.soft_shadows(cam, light, exact=True) for _ in range(3)]
    e64 = np.abs(r64[-1].vis[cov].astype(np.float64) - vd[cov])
    fp64_band = {"max_abs_err_vs_fp64": float(e64.max()), "mean_abs_err_vs_fp64": float(e64.mean()),
                 "pixels_over_1e-4": int((e64 > 1e-4).sum()),
                 "ms_per_frame": float(np.median([r.info["ms_total"] for r in r64])),
                 "band_corners": int(r64[-1].info["eps_band_corners"]),
                 "re_decided": int(r64[-1].info["eps_fp64_flips"]),
                 "pixels_changed": int((r64[-1].vis != vis).sum())}
    return {"pixels": int(len(cov)), "max_abs_err_vs_fp64": float(err.max()), "mean_abs_err_vs_fp64": float(err.mean()),
            "pixels_over_1e-4": int((err > 1e-4).sum()),
            "histogram": {"edges": ["0", "1e-7", "1e-6", "1e-5", "1e-4", "1e-3", "inf"],
                          "counts": [int(x) for x in hist]},
            "ray256": {"pixels": int(len(pick)), "max_abs_err_vs_fp64": float(er.max()),
                       "mean_abs_err_vs_fp64": float(er.mean()), "seconds": ray_s, "cores": threads},
            "fp64_oracle": {"seconds": fp64_s, "px_per_s": len(cov) / fp64_s, "cores": threads,
                            "what": "reference double build, exact, the frame's shading points"},
            "eps_fp64_mode": fp64_band,
            "oracle": "oracle/_ref (the reference compiled from its sources)"}


def reference_gpu(scene, steps: int, warmup: int):
    """The reference's own GPU engine (cuda/ built for sm_100a from its
    sources, oracle/_ref/libbtref_gpu.so) on the same frame, if built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from ref import RefGpu, RefTracer, ref_gpu_available
    if not ref_gpu_available():
        return None
    try:
        g = RefGpu(scene.pos, scene.tris)
    except OSError as e:
        return {"unavailable": str(e)[:200]}
    v = scene.views[0]
    cam = RefTracer(scene.pos, scene.tris, "f").camera_make(v.eye, v.target, v.fov, scene.up, W, H)
    L = scene.light_array()
    for _ in range(warmup):
        g.soft(cam, W, H, L, exact=True)
    ms, fb = [], 0
    for _ in range(steps):
        r = g.soft(cam, W, H, L, exact=True)
        ms.append((r["primary_s"] + r["trace_s"]) * 1e3)
        fb += r["overflow_px"]
    g.close()
    per = float(np.median(ms))
    return {"value": W * H / per * 1e3, "unit": "px/s", "ms_per_frame": per, "frames": steps,
            "cpu_fallback_pixels": fb,
            "build": "reference cuda/gpu_render.cu + cuda/wavefront.cu for sm_100a, --use_fast_math on wavefront.cu "
                     "as its cuda/CMakeLists.txt sets (wall-clocked GpuRenderer::softShadows)"}


# Primary visibility and point shadows (the other two paths of the engine):
# (scene, square size) at the reference's 16 x 16 tile, the hit polygons of
# the primary pass as the point-shadow roots.
VIS_WORKLOADS = (("building", 1024), ("sphere", 256), ("sphere", 1024), ("meeting", 256), ("meeting", 1024))


def _vis_scenes():
    from beamtrace2007_b200 import scenes
    return {"building": scenes.building(), "sphere": scenes.displaced_sphere(), "meeting": scenes.meeting_room()}


def visibility_measure(reps: int = 3):
    """This engine on VIS_WORKLOADS through bt_gpu_primary / bt_gpu_point
    (polygon lists to the host, the GpuRenderer::primary / pointShadows
    contract) and through bt_gpu_primary_ids / bt_gpu_point_mask (ids and
    mask rasterised on the GPU); wall-clocked per call, median of `reps`
    after a warm-up."""
    from beamtrace2007_b200.renderer import GpuRenderer, PreparedScene, make_camera
    out = {}
    sc = _vis_scenes()
    for name in sorted({n for n, _ in VIS_WORKLOADS}):
        s = sc[name]
        ps = PreparedScene(s.pos, s.tris, kd_device=0)
        light = np.asarray(s.point_light, np.float32)
        with GpuRenderer(ps) as g:
            for n_, W in VIS_WORKLOADS:
                if n_ != name:
                    continue
                v = s.views[0]
                cam = make_camera(v.eye, v.target, v.fov, s.up, W, W)
                tp, tq, tids, tmask = [], [], [], []
                for rep in range(reps + 1):
                    t0 = time.perf_counter()
                    prim = g.primary(cam, tile=16)
                    t1 = time.perf_counter()
                    sh = g.point_shadows(cam, prim, light)
                    t2 = time.perf_counter()
                    g.primary_ids(cam, tile=16)
                    t3 = time.perf_counter()
                    g.point_mask(cam, light, tile=16)
                    t4 = time.perf_counter()
                    if rep:
                        tp.append(t1 - t0)
                        tq.append(t2 - t1)
                        tids.append(t3 - t2)
                        tmask.append(t4 - t3)
                out[f"{name}/{W}"] = {"primary_ms": float(np.median(tp) * 1e3), "point_ms": float(np.median(tq) * 1e3),
                                      "hits": len(prim), "shadow_polys": len(sh),
                                      "primary_ids_ms": float(np.median(tids) * 1e3),
                                      "point_mask_ms": float(np.median(tmask) * 1e3)}
    return out


def reference_gpu_visibility(reps: int = 3):
    """The reference's own GPU engine (oracle/_ref/libbtref_gpu.so) on
    VIS_WORKLOADS: GpuRenderer::primary then pointShadows on its hit
    polygons, wall-clocked per call, median of `reps` after a warm-up."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from ref import RefGpu, RefTracer, ref_gpu_available
    if not ref_gpu_available():
        return None
    out = {}
    sc = _vis_scenes()
    for name in sorted({n for n, _ in VIS_WORKLOADS}):
        s = sc[name]
        g = RefGpu(s.pos, s.tris)
        rf = RefTracer(np.eye(3, dtype=np.float32), np.array([[0, 1, 2]], np.uint32), "f")  # Camera::make only
        for n_, W in VIS_WORKLOADS:
            if n_ != name:
                continue
            v = s.views[0]
            cam = rf.camera_make(v.eye, v.target, v.fov, s.up, W, W)
            rs = [g.primary_point(cam, W, W, np.asarray(s.point_light, np.float64), tile=16) for _ in range(reps + 1)]
            rs = rs[1:]
            out[f"{name}/{W}"] = {"primary_ms": float(np.median([r["primary_s"] for r in rs]) * 1e3),
                                  "point_ms": float(np.median([r["point_s"] for r in rs]) * 1e3),
                                  "hits": rs[-1]["hits"], "shadow_polys": rs[-1]["shadow_polys"],
                                  "cpu_fallback_ms": float(np.median([r["primary_fallback_s"] + r["point_fallback_s"]
                                                                      for r in rs]) * 1e3),
                                  "overflow_roots": rs[-1]["primary_overflow"] + rs[-1]["point_overflow"]}
        g.close()
    return out


def run_reference_arm(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from beamtrace2007_b200 import scenes
    s = scenes.plant()
    c = cpu_reference(s, args.steps, args.warmup, min_seconds=0.0, max_frames=args.steps)
    if c is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libbtref_f.so not built"}))
        return 0
    line = {"impl": "reference", "metric": METRIC, "value": c["value"], "unit": "px/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": c["ms_per_frame"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plant scene)",
            "config": workload_config(),
            "cpu_baseline": {"value": c["value"], "unit": "px/s", "cores": c["cores"], "kind": "reference",
                             "sample": c["sample"]},
            "e2e": {"value": c["value"], "unit": "px/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    try:
        import torch
        if torch.cuda.is_available():
            g = reference_gpu(s, max(args.steps, 5), args.warmup)
            if g is not None:
                line["reference_gpu"] = g
            if not args.no_extras:
                vis = reference_gpu_visibility()
                if vis is not None:
                    line["reference_gpu_visibility"] = vis
    except Exception as e:  # the CPU arm stands on its own
        line["reference_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"[:200]}
    print(json.dumps(line))
    return 0


def batched_measure(g, s, N, lib, C, steps):
    """A light-scale sweep of 8 frames (0.25-4x, the plant workload's sweep)
    as one batch (bt_gpu_batch_soft) against the same frames one by one
    (bt_gpu_soft_device); device time from the engine's CUDA events."""
    import torch
    from beamtrace2007_b200.renderer import make_camera
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    scales = [float(x) for x in np.geomspace(0.25, 4.0, 8)]
    lights = [s.light_array(k) for k in scales]
    npx = W * H
    outs = [(torch.empty(npx, dtype=torch.int32, device="cuda"),) +
            tuple(torch.empty(npx, dtype=torch.float32, device="cuda") for _ in range(3)) for _ in scales]
    info = N.RunInfo()
    opts = N.SoftOpts(1, 0.0)
    jobs = (N.SoftJob * len(scales))()
    for j, L in enumerate(lights):
        o = outs[j]
        jobs[j] = N.SoftJob(cam, N.AreaLight.from_array(L), opts, o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr(),
                            o[3].data_ptr())
    plain, batch = [], []
    for rep in range(steps + 1):
        t = 0.0
        for j, L in enumerate(lights):
            o = outs[j]
            N.check(lib.bt_gpu_soft_device(g._h, C.byref(cam), C.byref(N.AreaLight.from_array(L)), C.byref(opts),
                                           o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr(), o[3].data_ptr(),
                                           C.byref(info)))
            t += info.ms_total
        N.check(lib.bt_gpu_batch_soft(g._h, len(scales), jobs, C.byref(info)))
        if rep:  # the first pair warms up
            plain.append(t)
            batch.append(info.ms_total)
    px = npx * len(scales)
    pb, pp = float(np.median(batch)), float(np.median(plain))
    return {"value": px / pb * 1e3, "unit": "px/s", "plain_value": px / pp * 1e3, "ratio_vs_plain": pp / pb,
            "frames_per_batch": len(scales), "light_scales": [round(x, 3) for x in scales],
            "ms_per_batch": pb, "ms_frames_one_by_one": pp, "steps": steps}


def batched_jobs_measure(n_jobs: int = 64, sizes=(64, 128, 256, 512), max_tris: int = 200_000, reps: int = 1,
                         seed: int = 2024, tune: bool = True, plain_reps: int | None = None):
    """The batched-jobs workload: receiver/occluder pairs (icosphere or
    torus, meshes log-uniform between 100 and `max_tris` triangles, plus a
    ground quad), square resolutions from `sizes`, light scale U[0.25, 4],
    exact; all jobs in one engine run (scene pool, bt_gpu_batch_soft)
    against the same jobs one by one; device time from the engine's CUDA
    events.  kd-trees are built on the GPU.  With `tune`, the autotuner
    (autotune.tune_engine) picks the live sub-beam budget on the heaviest
    job at 64x64 before the runs.  The warm-up is one small job (a pass of
    the whole mix can take tens of seconds); `heaviest`: the two longest
    jobs alone, with their triangle tests (the algorithm's work: the engine's
    counters equal the reference's).  The batch is timed `reps` times and
    the jobs one by one the first `plain_reps` of them (default: all);
    medians of each."""
    from beamtrace2007_b200 import scenes
    from beamtrace2007_b200.autotune import tune_engine
    plain_reps = reps if plain_reps is None else plain_reps
    from beamtrace2007_b200.renderer import GpuRenderer, PreparedScene, make_camera
    rng = np.random.default_rng(seed)
    specs = [(int(np.exp(rng.uniform(np.log(100), np.log(max_tris)))), int(rng.choice(list(sizes))),
              float(rng.uniform(0.25, 4.0))) for _ in range(n_jobs)]
    t0 = time.perf_counter()
    jobs = []
    for i, (tris, res, scale) in enumerate(specs):
        sd = scenes.shadow_job(100 + i, tris)
        jobs.append((sd, PreparedScene(sd.pos, sd.tris, kd_device=0), res, scale))
    prep_s = time.perf_counter() - t0
    cams, lights = [], []
    for sd, ps, res, scale in jobs:
        v = sd.views[0]
        cams.append(make_camera(v.eye, v.target, v.fov, sd.up, res, res))
        lights.append(sd.light_array(scale))
    settings, tuned = {}, None
    if tune:
        h = max(range(len(jobs)), key=lambda k: jobs[k][1].num_tris * lights[k][3:6].dot(lights[k][3:6]))
        sd, ps, _, _ = jobs[h]
        v = sd.views[0]
        probe = make_camera(v.eye, v.target, v.fov, sd.up, 64, 64)
        settings, timings = tune_engine(ps, probe, lights[h], budgets=(128, 512, 2048), trace_ctas=(3, 4),
                                        blocks_per_sm=(0,), tail_records=(0,), reps=1)
        tuned = {"settings": settings, "probe": f"job {h} ({ps.num_tris} tris) at 64x64",
                 "ms": {str(k): round(t, 2) for k, t in timings.items()}}
    g = GpuRenderer(jobs[0][1], **settings)
    ids = [0] + [g.add_scene(ps) for _, ps, _, _ in jobs[1:]]
    px = sum(c.W * c.H for c in cams)
    small = min(range(len(jobs)), key=lambda k: cams[k].W * jobs[k][1].num_tris)
    g.batch_soft([cams[small]], [lights[small]], exact=True, scenes=[ids[small]], device_outputs=True)  # warm-up
    batch, plain, alone = [], [], {}
    for rep in range(reps):
        _, info = g.batch_soft(cams, lights, exact=True, scenes=ids, device_outputs=True)
        batch.append(info["ms_total"])
        if rep >= plain_reps:
            continue
        t = 0.0
        for k in range(len(cams)):
            _, i1 = g.batch_soft([cams[k]], [lights[k]], exact=True, scenes=[ids[k]], device_outputs=True)
            t += i1["ms_total"]
            alone[k] = (i1["ms_total"], i1["tri_tests"])
        plain.append(t)
    g.close()
    pb, pp = float(np.median(batch)), float(np.median(plain))
    top = sorted(alone, key=lambda k: -alone[k][0])[:2]
    return {"jobs": len(jobs), "triangles": int(sum(ps.num_tris for _, ps, _, _ in jobs)), "pixels": int(px),
            "sizes": list(sizes), "max_tris": max_tris, "reps": reps, "plain_reps": len(plain),
            "value": px / pb * 1e3, "unit": "px/s", "one_by_one_value": px / pp * 1e3, "ratio_vs_one_by_one": pp / pb,
            "ms_batch": pb, "ms_one_by_one": pp, "host_prep_s": prep_s, "autotuned": tuned,
            "heaviest": [{"job": k, "tris": jobs[k][1].num_tris, "res": cams[k].W, "light_scale": round(specs[k][2], 3),
                          "ms": round(alone[k][0], 1), "tri_tests": int(alone[k][1]),
                          "share_of_one_by_one": round(alone[k][0] / pp, 3)} for k in top]}


def serving_measure(n: int = 300):
    """The served stream through the library's request loop (bt_gpu_submit /
    bt_gpu_poll): three resident scenes (displaced sphere 327,680 triangles,
    meeting room 178,176, office building 2.1M; their kd-trees built on the
    GPU when the server admits them) in one context's pool, an 8 GB memory
    budget, Poisson arrivals, 60% primary / 25% point / 15% soft, 256-1024 px
    square; p50/p99 latency over `n` requests at the configured 50 req/s and
    px/s at a saturating 500 req/s."""
    from beamtrace2007_b200 import scenes
    from beamtrace2007_b200.serving import Server, poisson_stream
    sc = {"sphere": scenes.displaced_sphere(), "meeting": scenes.meeting_room(), "building": scenes.building()}
    out = {"scenes": {k: int(len(v.tris)) for k, v in sc.items()}, "memory_budget_gb": 8.0}
    with Server(sc, memory_budget_gb=8.0) as srv:
        # admitting a scene: finalise + kd-tree built on the GPU (bt_kd_build_gpu)
        out["scene_prep_ms"] = {k: round(v, 1) for k, v in srv.prep_ms.items()}
        out["tuned_tiles"] = srv.tune(sizes=(256, 512, 1024))  # the autotuner, before the stream
        poisson_stream(srv, rate=50.0, n=12, sizes=(256,), seed=11)  # warm-up
        for label, rate in (("configured_50", 50.0), ("saturated_500", 500.0)):
            _, summ = poisson_stream(srv, rate=rate, n=n, sizes=(256, 512, 1024), seed=7)
            out[label] = summ
        out["stats"] = srv.stats()
    return out


def trace_traffic():
    """DRAM bytes per trace-kernel launch from the committed ncu capture."""
    tp = os.path.join(ROOT, "profiles", "trace_kernel_plant512_traffic.json")
    if os.path.exists(tp):
        d = json.load(open(tp))
        return d.get("bytes_per_launch"), d.get("command")
    return None, None


def main():
    faulthandler.enable()  # a fatal signal prints the Python stack
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched and serving measurements")
    ap.add_argument("--capacity", type=int, default=0,
                    help="sub-beam records per queue (0: the engine's default); small values for profiler captures")
    ap.add_argument("--scene", default="plant", choices=["plant", "sphere"],
                    help="profiling only: 'sphere' renders the displaced icosphere (327,680 triangles, larger than "
                         "L2 with its tree) instead of the plant; the benchmark's workload is the plant")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference_arm(args)

    ws, rank, local = dist_setup()
    import ctypes as C

    import torch
    from beamtrace2007_b200 import _native as N
    from beamtrace2007_b200 import scenes
    from beamtrace2007_b200.renderer import GpuRenderer, PreparedScene, make_camera

    torch.cuda.set_device(local)
    s = scenes.plant() if args.scene == "plant" else scenes.displaced_sphere()
    ps = PreparedScene(s.pos, s.tris)
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    L = N.AreaLight.from_array(s.light_array())
    opts = N.SoftOpts(1, 0.0)
    g = GpuRenderer(ps, device=local, capacity=args.capacity, kernel_timing=True)
    lib = N.lib()
    npx = W * H
    dtri = torch.empty(npx, dtype=torch.int32, device="cuda")
    dvis, dE, dEu = (torch.empty(npx, dtype=torch.float32, device="cuda") for _ in range(3))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    info = N.RunInfo()

    def frame():
        N.check(lib.bt_gpu_soft_device(g._h, C.byref(cam), C.byref(L), C.byref(opts), dtri.data_ptr(),
                                       dvis.data_ptr(), dE.data_ptr(), dEu.data_ptr(), C.byref(info)))
        return info.as_dict()

    for _ in range(args.warmup):
        frame()
        flush.fill_(1)
    torch.cuda.synchronize()
    dist_barrier(ws)
    torch.cuda.synchronize()
    ms, infos = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            d = frame()
            ms.append(d["ms_total"])
            infos.append(d)
        torch.cuda.synchronize()
        dist_barrier(ws)
        torch.cuda.synchronize()
        # end to end: host output buffers through the reference-facing call
        e2e_t = []
        tri_h = np.zeros(npx, np.int32)
        vis_h, E_h, Eu_h = (np.zeros(npx, np.float32) for _ in range(3))
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            N.check(lib.bt_gpu_soft(g._h, C.byref(cam), C.byref(L), C.byref(opts), N.ptr(tri_h), N.ptr(vis_h),
                                    N.ptr(E_h), N.ptr(Eu_h), C.byref(info)))
            e2e_t.append(time.perf_counter() - t0)
    total_s = dist_max(sum(ms) * 1e-3, ws)
    e2e_s = dist_max(sum(e2e_t), ws)
    value = ws * npx * args.steps / total_s
    last = infos[-1]
    # Algorithmic bytes (counters are the reference's, bitwise): the frame
    # B_alg = 64 triTests + 12 kdSteps + 12 leafVisits + 128 beams + 40 px;
    # the trace kernel's share reads the triangle references, kd nodes and
    # each final sub-beam record once: 64 triTests + 12 kdSteps + 12 leafVisits + 64 beams.
    b_frame = (64 * last["tri_tests"] + 12 * last["kd_steps"] + 12 * last["leaf_visits"] + 128 * last["beams"]
               + 40 * npx)
    b_trace = 64 * last["tri_tests"] + 12 * last["kd_steps"] + 12 * last["leaf_visits"] + 64 * last["beams"]
    trace_ms = float(np.mean([d["ms_kernel_trace"] for d in infos]))
    launches_per_frame = float(np.mean([d["rounds"] for d in infos]))
    achieved = b_trace / (trace_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic, traffic_cmd = trace_traffic()
    if rank != 0:
        g.close()
        return 0
    line = {"metric": METRIC, "value": value, "unit": "px/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plant scene)",
            "config": dict(workload_config(), parallelism=f"replicas{ws}") if args.scene == "plant" else
            {"workload": "profiling run: displaced icosphere 327,680 tris, exact soft shadows 512x512 (not the "
                         "benchmark's workload)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "traceKernel<soft>",
                         "algorithmic_bytes_per_launch": b_trace / launches_per_frame,
                         "launches_per_frame": launches_per_frame,
                         "kernel_ms_per_launch": trace_ms / launches_per_frame,
                         "traffic_source": traffic_cmd,
                         "frame": {"algorithmic_bytes": b_frame, "achieved_gbs": b_frame / (total_s / args.steps) / 1e9,
                                   "frac": b_frame / (total_s / args.steps) / 1e9 / peak}},
            "e2e": {"value": ws * npx * args.steps / e2e_s, "unit": "px/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": npx * 16},
            "gpu_launches": int(sum(d["launches"] for d in infos)),
            "clocks": clk.summary(),
            "kernels_ms_per_frame": {"trace": trace_ms,
                                     "admit_clip_bookkeeping": float(np.mean([d["ms_round"] for d in infos])) - trace_ms},
            "counters": {k: last[k] for k in ("tri_tests", "kd_steps", "leaf_visits", "beams", "splits", "climbs",
                                               "rounds", "passes", "retried_roots", "max_spill")},
            "ms_primary": float(np.mean([d["ms_primary"] for d in infos])),
            "ms_trace": float(np.mean([d["ms_trace"] for d in infos]))}
    if not args.no_extras and ws == 1:  # (at N > 1 the other GPUs would wait on rank 0's extras)
        line["batched"] = batched_measure(g, s, N, lib, C, steps=3)
        # the batched-jobs workload as configured (64 jobs of up to 200K
        # triangles at up to 512^2), one repetition; and a mix of small jobs
        # (32 jobs of <= 20K triangles at 64-128^2) with three
        line["batched_jobs"] = batched_jobs_measure(reps=3, plain_reps=1)
        line["batched_jobs_small"] = batched_jobs_measure(n_jobs=32, max_tris=20_000, sizes=(64, 128), reps=3,
                                                          tune=False)
        line["visibility"] = visibility_measure()
        line["serving"] = serving_measure()
    if not args.no_cpu_baseline and ws == 1:
        c = cpu_reference(s, 3, 1)
        if c:
            line["cpu_baseline"] = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}
        # the last timed frame's results against the FP64 oracle
        acc = accuracy(s, ps, cam, s.light_array(), dvis.cpu().numpy())
        if acc:
            line["accuracy"] = acc
    print(json.dumps(line))
    g.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())

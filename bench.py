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
`e2e`: the same frames through bt_gpu_soft with host output buffers (the
GpuRenderer::softShadows contract), wall-clocked per call, device-to-host
copies of tri/vis/E/Eu inside.
`cpu_baseline` / `--impl reference`: the reference's own CPU tracer
(compiled from its sources, oracle/_ref) on the host's cores.

Multi-GPU: the frames of different GPUs are independent (replicas only):
each rank renders the workload on its own GPU, `value` = all ranks' pixels /
max-over-ranks time (weak scaling).
"""
from __future__ import annotations

import argparse
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


def cpu_reference(scene, steps: int, warmup: int, min_seconds: float = 3.0):
    """The reference CPU tracer (oracle/_ref) on the same frame, all host threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from ref import RefTracer, ref_available
    from beamtrace2007_b200.renderer import make_camera
    if not ref_available("f"):
        return None
    threads = os.cpu_count() or 1
    rf = RefTracer(scene.pos, scene.tris, "f")
    v = scene.views[0]
    cam = make_camera(v.eye, v.target, v.fov, scene.up, W, H).as_array()
    L = scene.light_array()
    for _ in range(warmup):
        rf.soft_image(cam, W, H, L, exact=True, threads=threads)
    times = []
    t_start = time.perf_counter()
    while len(times) < steps or time.perf_counter() - t_start < min_seconds:
        r = rf.soft_image(cam, W, H, L, exact=True, threads=threads)
        times.append(r["primary_s"] + r["trace_s"])
        if len(times) >= 1000:
            break
    per = float(np.median(times))
    return {"value": W * H / per, "unit": "px/s", "cores": threads, "kind": "reference",
            "sample": f"{len(times)} full {W}x{H} frames (bt_render --mode softshadow --method beam --exact "
                      f"--threads {threads} pipeline: ray primary + beam soft shadows), median frame {per*1e3:.1f} ms",
            "ms_per_frame": per * 1e3}


def run_reference_arm(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from beamtrace2007_b200 import scenes
    s = scenes.plant()
    c = cpu_reference(s, args.steps, args.warmup)
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
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    s = scenes.plant()
    ps = PreparedScene(s.pos, s.tris)
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    L = N.AreaLight.from_array(s.light_array())
    opts = N.SoftOpts(1, 0.0)
    g = GpuRenderer(ps, device=local)
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
    ms, round_ms, infos = [], [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            d = frame()
            ms.append(d["ms_total"])
            round_ms.append(d["ms_round"])
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
    # algorithmic bytes of one frame (counters are the oracle's, bitwise)
    b_alg = (64 * last["tri_tests"] + 12 * last["kd_steps"] + 12 * last["leaf_visits"] + 128 * last["beams"]
             + 40 * npx)
    rms = float(np.mean(round_ms))
    achieved = b_alg / (rms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "round_kernel_plant512_traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get("bytes_per_frame")
    if rank != 0:
        g.close()
        return 0
    line = {"metric": METRIC, "value": value, "unit": "px/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plant scene)",
            "config": dict(workload_config(), parallelism=f"replicas{ws}"),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "roundKernel<soft>", "algorithmic_bytes_per_frame": b_alg,
                         "kernel_ms_per_frame": rms},
            "e2e": {"value": ws * npx * args.steps / e2e_s, "unit": "px/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": npx * 16},
            "gpu_launches": int(sum(d["launches"] for d in infos)),
            "clocks": clk.summary(),
            "counters": {k: last[k] for k in ("tri_tests", "kd_steps", "leaf_visits", "beams", "splits",
                                               "round_launches", "passes", "retried_roots", "max_spill")},
            "ms_primary": float(np.mean([d["ms_primary"] for d in infos])),
            "ms_trace": float(np.mean([d["ms_trace"] for d in infos]))}
    if not args.no_cpu_baseline and ws == 1:
        c = cpu_reference(s, 3, 1)
        if c:
            line["cpu_baseline"] = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line))
    g.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())

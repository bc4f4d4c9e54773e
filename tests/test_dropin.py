"""The drop-in check: the reference's own command-line renderer
(apps/bt_render.cpp, built as bt_render_cuda by `make -C oracle shim`)
linked against beamtrace2007_b200/shim/gpu_render_shim.cpp, i.e. its
GpuRenderer running on libbt_gpu.so.  It loads the plant scene from an OBJ
file and a .cfg (the reference's scene format) and writes the visibility
image, which must be within 1e-4 of the reference's FP64 build on the same
shading points (bt_render_d, the FP64 oracle)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, scene

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "oracle", "_ref", "bt_render_cuda")
VIS_TOL = 1e-4


def _read_pfm(path):
    with open(path, "rb") as f:
        assert f.readline().strip() == b"PF"
        w, h = (int(x) for x in f.readline().split())
        scale = float(f.readline())
        data = np.frombuffer(f.read(), dtype="<f4" if scale < 0 else ">f4").reshape(h, w, 3)
    return data[::-1, :, 0]  # rows are stored bottom to top


def _write_scene(s, d):
    obj = os.path.join(d, "plant.obj")
    with open(obj, "w") as f:
        for p in np.asarray(s.pos, np.float32):
            f.write("v %.9g %.9g %.9g\n" % tuple(float(x) for x in p))
        for t in np.asarray(s.tris):
            f.write("f %d %d %d\n" % tuple(int(i) + 1 for i in t))
    v = s.views[0]
    L = np.asarray(s.light_array(), np.float64)
    cfg = os.path.join(d, "plant.cfg")
    with open(cfg, "w") as f:
        f.write("name plant\n")
        f.write(f"mesh obj {obj}\n")
        f.write("up %.9g %.9g %.9g\n" % tuple(float(x) for x in s.up))
        f.write("view " + " ".join("%.9g" % float(x) for x in (*v.eye, *v.target, v.fov)) + "\n")
        f.write("area_light " + " ".join("%.9g" % float(x) for x in L) + "\n")
    return cfg


def test_bt_render_cuda_soft_shadows(gpu, oracle_ready, tmp_path):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/bt_render_cuda not built")
    from ref import RefTracer
    s, ps = scene("plant")
    cfg = _write_scene(s, str(tmp_path))
    W, H = 96, 80
    out = os.path.join(str(tmp_path), "gpu")
    r = subprocess.run([EXE, "--config", cfg, "--mode", "softshadow", "--method", "beam", "--exact", "--res",
                        f"{W}x{H}", "--out", out, "--pfm"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "GPU:" in r.stderr
    vis = _read_pfm(out + "_vis.pfm").ravel()
    rf = RefTracer(s.pos, s.tris, "f")
    rd = RefTracer(s.pos, s.tris, "d")
    v = s.views[0]
    cam = rf.camera_make(v.eye, v.target, v.fov, s.up, W, H)
    tri, X, N, _ = rf.primary_rays(cam, W, H)
    vd, _, _, _ = rd.soft_points(s.light_array(), ps.offset, tri, X, N, exact=True, threads=4)
    m = tri >= 0
    assert m.sum() > W * H // 8
    assert np.all(vis[~m] == -1)
    err = np.abs(vis.astype(np.float64) - vd)[m]
    assert err.max() <= VIS_TOL, f"max |vis - fp64| {err.max():.3g}"


def test_reference_gpu_test_program_through_the_shim(gpu):
    """The reference's own GPU test program (cuda/test_cuda.cpp with its
    test runner, built unchanged by `make -C oracle shim_tests` as
    bt_tests_cuda) against the shim: soft shadows against its CPU tracer on
    its analytic, plant and room scenes; primary and point-shadow polygons
    rasterised at 384^2 with no interior pixel differing; two runs equal and
    a budget of 4 with 4096-record queues still exact, its over-budget
    pixels counted in lastOverflowPixels (retried on the GPU here, not on
    the CPU)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "bt_tests_cuda")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/bt_tests_cuda not built")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout + r.stderr)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "5/5 tests passed" in r.stdout + r.stderr
    assert "no CUDA device" not in r.stderr

"""CUDA engine vs the oracle, through the C-ABI (libbt_gpu.so).

Bars: pieces (primary hit polygons, point-shadow polygons) bitwise identical
to the reference float build per root; per-pixel ids and shadow flags
identical outside the band of pixel centres covered by two polygons (shared
edges, where the reference's own result depends on polygon order); soft
visibility within 1e-4 of the FP64 build (bt_render_d) on identical shading
points, exact E within 1e-5 of the image's largest E; primary rays (tri, X,
N) bitwise."""
import numpy as np
import pytest

from conftest import piece_keys, scene, to_f32

pytestmark = pytest.mark.gpu

VIS_TOL = 1e-4   # |vis - vis_fp64|, the soft-shadow parity bar
E_REL = 1e-5     # |E_exact - E_fp64| relative to the image's largest E


def _renderer(ps, **kw):
    from beamtrace2007_b200.renderer import GpuRenderer
    return GpuRenderer(ps, **kw)


@pytest.mark.parametrize("name,W,H", [("plant", 160, 120), ("room", 128, 128)])
def test_primary_rays_bitwise(name, W, H, gpu, oracle_ready):
    from ref import RefTracer
    from beamtrace2007_b200 import _native as N
    from beamtrace2007_b200.renderer import make_camera
    import ctypes as C
    s, ps = scene(name)
    rf = RefTracer(s.pos, s.tris, "f")
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    tr, Xr, Nr, _ = rf.primary_rays(cam.as_array(), W, H)
    with _renderer(ps) as g:
        tri = np.zeros(W * H, np.int32)
        X = np.zeros(3 * W * H, np.float32)
        Nn = np.zeros(3 * W * H, np.float32)
        N.check(N.lib().bt_gpu_primary_rays(g._h, C.byref(cam), N.ptr(tri), N.ptr(X), N.ptr(Nn)))
    assert np.array_equal(tri, tr)
    assert np.array_equal(X, Xr.astype(np.float32).ravel())
    assert np.array_equal(Nn, Nr.astype(np.float32).ravel())


@pytest.mark.parametrize("name,W,H,scale", [("plant", 160, 120, 1.0), ("plant", 96, 96, 4.0), ("room", 128, 96, 1.0)])
def test_soft_shadows_vs_fp64(name, W, H, scale, gpu, oracle_ready):
    from ref import RefTracer
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene(name)
    rf = RefTracer(s.pos, s.tris, "f")
    rd = RefTracer(s.pos, s.tris, "d")
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    L = s.light_array(scale)
    with _renderer(ps) as g:
        res = g.soft_shadows(cam, L, exact=True)
    tri, X, N, _ = rf.primary_rays(cam.as_array(), W, H)
    assert np.array_equal(res.tri, tri)
    vd, Ed, Eud, _ = rd.soft_points(L, ps.offset, tri, X, N, exact=True, threads=4)
    vf, Ef, Euf, _ = rf.soft_points(L, ps.offset, tri, X, N, exact=True, threads=4)
    m = tri >= 0
    assert m.sum() > W * H // 8
    err = np.abs(res.vis.astype(np.float64) - vd)[m]
    assert err.max() <= VIS_TOL, f"max |vis - fp64| {err.max():.3g}"
    assert np.abs(res.vis - vf.astype(np.float32))[m].max() <= 1e-6
    e_gpu = np.abs(res.E.astype(np.float64) - Ed)[m].max()
    assert e_gpu <= E_REL * np.abs(Ed).max(), f"max |E - fp64| {e_gpu:.3g}"
    # the FP64 accumulation is closer to the FP64 build than the float build is
    assert e_gpu <= np.abs(Ef - Ed)[m].max() + 1e-7
    assert np.array_equal(res.Eu, Euf.astype(np.float32))
    assert np.all(res.vis[~m] == -1)


def test_soft_points_closed_form(gpu):
    """Square occluder (side 1, height 1) under a unit square light at height
    3: visibility on the floor has a closed form (the reference's known-answer
    test, tests/test_tracing.cpp:255-312; 2e-3 in float there)."""
    from beamtrace2007_b200.scenes import Pcg32
    s, ps = scene("analytic")
    rng = Pcg32(17)
    pts = np.array([[rng.uniform(-1.5, 1.5), 0.0, rng.uniform(-1.5, 1.5)] for _ in range(400)], np.float32)
    floor = next(t for t in range(ps.num_tris) if np.all(ps.pos[ps.tris[t]][:, 1] == 0))
    tri = np.full(len(pts), floor, np.int32)
    Nn = np.tile(np.array([0, 1, 0], np.float32), (len(pts), 1))
    off = 1e-4
    with _renderer(ps) as g:
        res = g.soft_points(s.light_array(), tri, pts, Nn, offset=off)

    def closed(px, pz, H=3 - off, h=1 - off, occ=1.0):
        k = H / h
        cx, cz, half = px * (1 - k), pz * (1 - k), occ * k / 2
        ox = max(0.0, min(0.5, cx + half) - max(-0.5, cx - half))
        oz = max(0.0, min(0.5, cz + half) - max(-0.5, cz - half))
        return 1 - ox * oz

    ref = np.array([closed(float(p[0]), float(p[2])) for p in pts])
    assert np.abs(res.vis - ref).max() < 2e-3


@pytest.mark.parametrize("name", ["room", "plant"])
def test_primary_and_point_pieces_bitwise(name, gpu, oracle_ready):
    from ref import RefTracer
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene(name)
    rf = RefTracer(s.pos, s.tris, "f")
    v = s.views[0]
    W, H = 192, 160
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    camv = cam.as_array()
    with _renderer(ps) as g:
        prim = g.primary(cam, tile=16)
        pr, _ = rf.primary_tiles(camv, W, H, tile=16)
        pr = to_f32(pr)
        hits_ref = pr.select(pr.tri >= 0)
        assert np.array_equal(piece_keys(prim, True), piece_keys(hits_ref, True))
        light = np.array(s.point_light, np.float32)
        sh = g.point_shadows(cam, prim, light)
        pr2, _ = rf.point_shadows(camv, W, H, light.astype(np.float64), prim)
        assert np.array_equal(piece_keys(sh), piece_keys(to_f32(pr2)))
        tri_g, flag_g = g.raster(cam, prim, sh)
    tri_r, flag_r = rf.rasterize(camv, W, H, prim, to_f32(pr2))
    # pixel centres covered by two polygons (shared edges) depend on polygon
    # order in the reference; they are the band excluded from the comparison
    rev = lambda p: p.select(np.arange(len(p))[::-1])  # noqa: E731
    tri_r2, flag_r2 = rf.rasterize(camv, W, H, rev(prim), rev(to_f32(pr2)))
    band = (tri_r != tri_r2) | (flag_r != flag_r2)
    assert band.mean() <= 1e-2
    assert np.array_equal(tri_g[~band], tri_r[~band])
    assert np.array_equal(flag_g[~band], flag_r[~band])


def test_deterministic_and_budget_retry(gpu, oracle_ready):
    """Two runs are bitwise equal (fixed-point accumulation); tiny budgets and
    queues force roots into GPU retries, with the same result
    (cuda/test_cuda.cpp:155-192 checked the CPU fallback instead)."""
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene("plant")
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, 128, 128)
    L = s.light_array()
    with _renderer(ps) as g:
        a = g.soft_shadows(cam, L, exact=True)
        b = g.soft_shadows(cam, L, exact=True)
    assert np.array_equal(a.vis, b.vis) and np.array_equal(a.E, b.E)
    with _renderer(ps, budget=4, capacity=4096) as g:
        c = g.soft_shadows(cam, L, exact=True)
        info = c.info
    assert info["retried_roots"] > 100
    assert np.array_equal(a.vis, c.vis) and np.array_equal(a.E, c.E)


def test_primary_budget_retry(gpu, oracle_ready):
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene("plant")
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, 128, 128)
    with _renderer(ps) as g:
        a = g.primary(cam, tile=32)
    with _renderer(ps, primary_budget=8, capacity=2048) as g:
        b = g.primary(cam, tile=32)
        assert g.last_overflow_pixels > 0
    assert np.array_equal(piece_keys(a, True), piece_keys(b, True))


def test_batch_equals_jobs_alone(gpu):
    """Jobs of different sizes, cameras and light scales in one batch give
    bitwise the results each gives alone (the accumulation is fixed point,
    so the order in which pieces finish does not matter)."""
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene("plant")
    v = s.views[0]
    sizes = [(64, 48), (128, 128), (96, 160), (33, 17)]
    scales = [0.25, 1.0, 4.0, 2.0]
    cams = [make_camera(v.eye, v.target, v.fov + 5 * i, s.up, W, H) for i, (W, H) in enumerate(sizes)]
    lights = [s.light_array(k) for k in scales]
    with _renderer(ps) as g:
        batch = g.batch_soft(cams, lights, exact=True)
        for cam, L, b in zip(cams, lights, batch):
            alone = g.soft_shadows(cam, L, exact=True)
            assert np.array_equal(b.tri, alone.tri)
            assert np.array_equal(b.vis, alone.vis)
            assert np.array_equal(b.E, alone.E)
            assert np.array_equal(b.Eu, alone.Eu)


@pytest.mark.parametrize("k", [0, 1])
def test_soft_points_vs_golden_and_restatement(gpu, k):
    """Supplied shading points (the committed fixture: the reference's own
    primary-ray points and its FP64 results, light scales 1 and 4): the GPU
    within 1e-4 of the reference's double build and of the independent FP64
    restatement (oracle/restate_soft.py)."""
    import os
    from conftest import ROOT
    from restate_soft import soft_points
    g = np.load(os.path.join(ROOT, "tests", "golden", "plant_soft_points.npz"))
    s, ps = scene("plant")
    L = g[f"light{k}"]
    with _renderer(ps) as r:
        res = r.soft_points(L, g["tri"], g["X"], g["N"], exact=True, offset=float(g["offset"]))
    assert np.abs(res.vis.astype(np.float64) - g[f"vis{k}"]).max() <= VIS_TOL
    vr, Er = soft_points(ps.pos, ps.tris, L, float(g["offset"]), g["tri"], g["X"].astype(np.float64),
                         g["N"].astype(np.float64))
    assert np.abs(res.vis.astype(np.float64) - vr).max() <= VIS_TOL
    assert np.abs(res.E.astype(np.float64) - Er).max() <= E_REL * np.abs(Er).max()


@pytest.mark.parametrize("name,kw", [("room", {}), ("plant", {}), ("building", dict(floors=1, furniture=3))])
def test_device_ids_and_masks_equal_host_path(name, kw, gpu):
    """bt_gpu_primary_ids / bt_gpu_point_mask (polygons never leave the GPU)
    give bitwise the ids and masks of the host polygon path (bt_gpu_primary,
    bt_gpu_point, bt_gpu_raster), which the tests above pin to the reference."""
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene(name, **kw)
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, 200, 150)
    light = np.array(s.point_light, np.float32)
    with _renderer(ps) as g:
        ids = g.primary_ids(cam)
        ids2, mask = g.point_mask(cam, light)
        prim = g.primary(cam, tile=16)
        sh = g.point_shadows(cam, prim, light)
        tri_h, flag_h = g.raster(cam, prim, sh)
    assert np.array_equal(ids, tri_h)
    assert np.array_equal(ids2, tri_h)
    assert np.array_equal(mask, flag_h)


def test_eps_band_logging(gpu):
    """eps_stats: the trace kernels that count the edge votes inside the
    fuzzy band and how many of them an FP64 re-evaluation places outside it.
    Decisions stay the float ones, so the results are bitwise those of the
    plain kernels; the counts are per record, so they repeat exactly as long
    as no root is abandoned over its budget and retried (whether one is
    depends on timing): the budget here is one that no root reaches."""
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene("plant")
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, 160, 120)
    L = s.light_array(2.0)
    with _renderer(ps, budget=2048) as g:
        plain = g.soft_shadows(cam, L, exact=True)
    with _renderer(ps, eps_stats=True, budget=2048) as g:
        a = g.soft_shadows(cam, L, exact=True)
        b = g.soft_shadows(cam, L, exact=True)
    assert plain.info["retried_roots"] == a.info["retried_roots"] == b.info["retried_roots"] == 0
    for f in ("tri", "vis", "E", "Eu"):
        assert np.array_equal(getattr(a, f), getattr(plain, f))
    assert plain.info["eps_band_corners"] == 0
    band, flips = a.info["eps_band_corners"], a.info["eps_fp64_flips"]
    assert (band, flips) == (b.info["eps_band_corners"], b.info["eps_fp64_flips"])
    assert band > 0 and 0 <= flips <= band
    assert a.info["tri_tests"] == plain.info["tri_tests"]


@pytest.mark.parametrize("name,kw,budget", [("plant", {}, 128), ("plant", {}, 4),
                                            ("building", dict(floors=1, furniture=3), 128)])
def test_fused_primary_rays_same_as_separate(name, kw, budget, gpu):
    """fuse_primary: each shadow root's admission traces its pixel's eye ray
    instead of a separate primary-ray pass.  Bitwise the same tri, vis, E and
    Eu, exact and not (the non-exact E reads the fused X and N), also when
    roots over a tiny budget are re-admitted and retried; and through the
    device-buffer entry point."""
    import torch
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene(name, **kw)
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, 160, 120)
    L = s.light_array(2.0)
    with _renderer(ps, budget=budget) as g:
        sep = [g.soft_shadows(cam, L, exact=e) for e in (True, False)]
    with _renderer(ps, budget=budget, fuse_primary=True) as g:
        fus = [g.soft_shadows(cam, L, exact=e) for e in (True, False)]
        # the device-buffer entry point, fused
        import ctypes as C
        from beamtrace2007_b200 import _native as N
        n = cam.W * cam.H
        out = [torch.full((n,), 7, dtype=t, device="cuda:0") for t in (torch.int32, torch.float32, torch.float32,
                                                                         torch.float32)]
        torch.cuda.synchronize()
        N.check(N.lib().bt_gpu_soft_device(g._h, C.byref(cam), C.byref(N.AreaLight.from_array(L)),
                                           C.byref(N.SoftOpts(1, 0.0)), *(o.data_ptr() for o in out), None))
        dev = [o.cpu().numpy() for o in out]
    assert (sep[0].tri >= 0).mean() > 0.2
    for a, b in zip(sep, fus):
        for f in ("tri", "vis", "E", "Eu"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), f
    for x, f in zip(dev, ("tri", "vis", "E", "Eu")):
        assert np.array_equal(x, getattr(sep[0], f)), f
    if budget < 16:
        assert fus[0].info["retried_roots"] > 0


def test_last_polys_instead_of_a_second_run(gpu):
    """A polygon buffer too small for bt_gpu_primary / bt_gpu_point: the
    polygons are fetched from the device afterwards (bt_gpu_last_polys),
    bitwise the same as with a buffer large enough, without running the
    engine again; any other engine call drops them (BT_ERR_INVALID)."""
    import ctypes as C
    from beamtrace2007_b200 import _native as N
    from beamtrace2007_b200.renderer import GpuRenderer, PolyList, make_camera
    from conftest import piece_keys
    s, ps = scene("plant")
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, 96, 72)
    light = np.array(s.point_light, np.float32)
    with GpuRenderer(ps) as g:
        big = g.primary(cam, tile=16, cap=1 << 20)
        small = g.primary(cam, tile=16, cap=16)
        launches = g.last_info["launches"]
        assert len(big) > 16 and np.array_equal(piece_keys(small, True), piece_keys(big, True))
        sh_big = g.point_shadows(cam, big, light, cap=1 << 20)
        sh_small = g.point_shadows(cam, big, light, cap=4)
        assert len(sh_big) > 4 and np.array_equal(piece_keys(sh_small), piece_keys(sh_big))
        g.soft_shadows(cam, s.light_array(), exact=False)
        out = PolyList.alloc(8)
        st = out.struct()
        cnt = C.c_int64()
        assert N.lib().bt_gpu_last_polys(g._h, C.byref(st), C.byref(cnt)) == -1
    assert launches > 0


def test_graph_rounds_same_results(gpu):
    """Batches of rounds replayed as CUDA graphs (graph_rounds, the default)
    give bitwise the results of launching the rounds one by one: soft
    shadows (a second frame replays the captured graphs), a tiny budget
    whose retry passes change the launch parameters, a batch of jobs, and
    primary ids and point masks."""
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene("plant")
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, 128, 96)
    L = s.light_array()
    light = np.asarray(s.point_light, np.float32)
    cams = [make_camera(v.eye, v.target, v.fov + 4 * i, s.up, 64 + 16 * i, 48) for i in range(3)]
    lights = [s.light_array(k) for k in (0.5, 1.0, 3.0)]
    out = {}
    for gr in (False, True):
        r = []
        with _renderer(ps, graph_rounds=gr) as g:
            for _ in range(2):
                a = g.soft_shadows(cam, L, exact=True)
                r += [a.vis, a.E]
            r += [b.vis for b in g.batch_soft(cams, lights, exact=True)]
            r += [g.primary_ids(cam, tile=8)] + list(g.point_mask(cam, light, tile=8))
        with _renderer(ps, graph_rounds=gr, budget=4, capacity=4096) as g:
            c = g.soft_shadows(cam, L, exact=True)
            assert c.info["retried_roots"] > 100
            r += [c.vis, c.E]
        out[gr] = r
    assert len(out[False]) == len(out[True])
    for a, b in zip(out[False], out[True]):
        assert np.array_equal(a, b)

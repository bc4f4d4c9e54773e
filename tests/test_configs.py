"""The workloads at their configured sizes.

* Room, primary visibility, 256x256 (864 triangles, camera at (1, 1, 1.6)
  toward the room centre, 60 degrees): hit polygons bitwise the reference
  float build's per tile, per-pixel ids bitwise; pixels whose id depends on
  polygon order in the reference itself (the band) are counted and held at
  <= 0.01%.
* Building, point shadows: a two-floor cut of the office building
  (190K triangles) at 256x256 against the reference, and the full seven
  floors (2.1M triangles) at 1024x1024 through properties that hold at any
  size: the primary pieces tile the image plane, each root's shadowed area is
  at most its hit area, two runs are bitwise equal.
* Plant, exact soft shadows, 512x512: visibility within 1e-4 of the FP64
  build on identical shading points, every pixel.
"""
import numpy as np
import pytest

from conftest import piece_keys, scene, to_f32

pytestmark = pytest.mark.gpu

BAND_MAX = 1e-4   # fraction of pixels whose reference result depends on polygon order
VIS_TOL = 1e-4


def _renderer(ps, **kw):
    from beamtrace2007_b200.renderer import GpuRenderer
    return GpuRenderer(ps, **kw)


def _band(rf, camv, W, H, prim, shadow):
    rev = lambda p: p.select(np.arange(len(p))[::-1])  # noqa: E731
    t1, f1 = rf.rasterize(camv, W, H, prim, shadow)
    t2, f2 = rf.rasterize(camv, W, H, rev(prim), rev(shadow))
    return t1, f1, (t1 != t2) | (f1 != f2)


@pytest.mark.parametrize("name,kw,W", [("room", {}, 256), ("building", dict(floors=2, furniture=4), 256)])
def test_primary_and_point_shadows_at_config_size(name, kw, W, gpu, oracle_ready):
    from ref import RefTracer
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene(name, **kw)
    rf = RefTracer(s.pos, s.tris, "f")
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, W)
    camv = cam.as_array()
    light = np.array(s.point_light, np.float32)
    with _renderer(ps) as g:
        prim = g.primary(cam, tile=16)
        sh = g.point_shadows(cam, prim, light)
        tri_g, flag_g = g.raster(cam, prim, sh)
    pr, _ = rf.primary_tiles(camv, W, W, tile=16)
    hits = to_f32(pr).select(to_f32(pr).tri >= 0)
    assert np.array_equal(piece_keys(prim, True), piece_keys(hits, True))
    sr, _ = rf.point_shadows(camv, W, W, light.astype(np.float64), prim)
    assert np.array_equal(piece_keys(sh), piece_keys(to_f32(sr)))
    tri_r, flag_r, band = _band(rf, camv, W, W, prim, to_f32(sr))
    assert band.mean() <= BAND_MAX, f"band {band.sum()} px"
    assert np.array_equal(tri_g[~band], tri_r[~band])
    assert np.array_equal(flag_g[~band], flag_r[~band])


def test_building_full_size_point_shadows(gpu):
    """2.1M triangles, 1024x1024: size-independent properties."""
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene("building")
    assert ps.num_tris > 2_000_000
    W = 1024
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, W)
    light = np.array(s.point_light, np.float32)
    with _renderer(ps) as g:
        prim = g.primary(cam, tile=16)
        sh = g.point_shadows(cam, prim, light)
        prim2 = g.primary(cam, tile=16)
        sh2 = g.point_shadows(cam, prim2, light)
        tri, flag = g.raster(cam, prim, sh)
    # deterministic (hit polygons are appended in whatever order they finish,
    # so a shadow piece is keyed by its hit polygon's rank, not its index)
    assert np.array_equal(piece_keys(prim, True), piece_keys(prim2, True))

    def stable(sh_, prim_):
        x = np.ascontiguousarray(prim_.x, np.float32).view(np.uint32).astype(np.int64)
        y = np.ascontiguousarray(prim_.y, np.float32).view(np.uint32).astype(np.int64)
        rows = np.concatenate([np.stack([np.asarray(prim_.root, np.int64), np.asarray(prim_.tri, np.int64)], 1), x, y],
                              1)
        rank = np.empty(len(prim_), np.int64)
        rank[np.lexsort(rows.T[::-1])] = np.arange(len(prim_))
        out = to_f32(sh_)
        out.root = rank[np.asarray(sh_.root)].astype(np.int32)
        return piece_keys(out)
    assert np.array_equal(stable(sh, prim), stable(sh2, prim2))
    # the visible polygons tile the image plane (the building surrounds the camera)
    img = 4.0 * float(cam.half_w) * float(cam.half_h)
    assert abs(float(np.sum(prim.area, dtype=np.float64)) - img) <= 1e-4 * img
    assert (tri >= 0).mean() > 0.999
    # per hit polygon, the shadowed area is at most the hit area
    def poly_area(x, y, n):
        a = 0.0
        for i in range(n):
            j = (i + 1) % n
            a += float(x[i]) * float(y[j]) - float(x[j]) * float(y[i])
        return abs(a) * 0.5
    hit_area = np.array([poly_area(prim.x[k], prim.y[k], prim.n[k]) for k in range(len(prim))])
    sh_area = np.zeros(len(prim))
    for k in range(len(sh)):
        sh_area[sh.root[k]] += poly_area(sh.x[k], sh.y[k], sh.n[k])
    # (float corners: allow 1e-3 relative and 0.05 of a pixel's area)
    px_area = img / (W * W)
    excess = sh_area - hit_area * (1 + 1e-3)
    assert excess.max() <= 0.05 * px_area, f"shadow area above hit area by {excess.max() / px_area:.3g} px"
    assert 0.0 < flag.mean() < 1.0


def test_plant_soft_512_vs_fp64(gpu, oracle_ready):
    from ref import RefTracer
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene("plant")
    W = 512
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, W)
    L = s.light_array()
    with _renderer(ps) as g:
        res = g.soft_shadows(cam, L, exact=True)
    rf = RefTracer(s.pos, s.tris, "f")
    rd = RefTracer(s.pos, s.tris, "d")
    tri, X, N, _ = rf.primary_rays(cam.as_array(), W, W, threads=8)
    assert np.array_equal(res.tri, tri)
    vd, _, _, _ = rd.soft_points(L, ps.offset, tri, X, N, exact=True, threads=16)
    m = tri >= 0
    err = np.abs(res.vis.astype(np.float64) - vd)[m]
    assert err.max() <= VIS_TOL, f"max |vis - fp64| {err.max():.3g}"

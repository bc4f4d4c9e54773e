"""The engine's per-lane code, compiled for the host (tests/native/emu.cpp),
against the reference's BeamCore with the restart trail and no mailboxing:
pieces bitwise identical per root, counters identical (the equivalence the
reference itself tests in tests/test_wavefront.cpp:185-199)."""
import numpy as np
import pytest

from conftest import piece_keys, scene, to_f32

EMU_NAMES = ["kdSteps", "leafVisits", "triTests", "hits", "splits", "beams", "rootBeams", "presplitBeams",
             "fiveSplits", "climbs"]


def _stats_equal(est, rst):
    return {k: (int(est[i]), rst[k]) for i, k in enumerate(EMU_NAMES) if int(est[i]) != rst[k]}


@pytest.mark.parametrize("name", ["room", "plant"])
def test_primary_and_point_pieces_bitwise(name, native_lib, oracle_ready):
    from emu import Emulator
    from ref import RefTracer
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene(name)
    rf = RefTracer(s.pos, s.tris, "f")
    em = Emulator(ps)
    v = s.views[0]
    W, H = 96, 80
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    camv = cam.as_array()
    pe, ste = em.primary_tiles(cam, tile=16)
    pr, st = rf.primary_tiles(camv, W, H, tile=16)
    pr = to_f32(pr)
    assert len(pe) == len(pr)
    assert np.array_equal(piece_keys(pe, True), piece_keys(pr, True))
    assert _stats_equal(ste, st) == {}
    hits = pr.select(pr.tri >= 0)
    light = np.array(s.point_light, np.float32)
    pe2, ste2 = em.point(cam, light, hits)
    pr2, st2 = rf.point_shadows(camv, W, H, light.astype(np.float64), hits)
    assert np.array_equal(piece_keys(pe2), piece_keys(to_f32(pr2)))
    assert _stats_equal(ste2, st2) == {}


def test_primary_whole_image_root(native_lib, oracle_ready):
    """One root covering the whole image (beamPrimary's root, render.cpp:150-183)."""
    from emu import Emulator
    from ref import RefTracer
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene("room")
    rf = RefTracer(s.pos, s.tris, "f")
    em = Emulator(ps)
    v = s.views[0]
    cam = make_camera(v.eye, v.target, v.fov, s.up, 64, 64)
    pe, _ = em.primary_tiles(cam, tile=64)
    pr, _ = rf.primary_tiles(cam.as_array(), 64, 64, tile=64)
    assert np.array_equal(piece_keys(pe, True), piece_keys(to_f32(pr), True))


@pytest.mark.parametrize("name", ["plant", "room"])
def test_soft_points_match_float_and_fp64(name, native_lib, oracle_ready):
    from emu import Emulator
    from ref import RefTracer
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene(name)
    rf = RefTracer(s.pos, s.tris, "f")
    rd = RefTracer(s.pos, s.tris, "d")
    em = Emulator(ps)
    v = s.views[0]
    W, H = 64, 48
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    tri, X, N, _ = rf.primary_rays(cam.as_array(), W, H)
    L = s.light_array()
    ve, Ge, ste = em.soft_points(L.astype(np.float32), ps.offset, tri, X.astype(np.float32), N.astype(np.float32),
                                 exact=True)
    vf, Ef, _, st = rf.soft_points(L, ps.offset, tri, X, N, exact=True)
    vd, Ed, _, _ = rd.soft_points(L, ps.offset, tri, X, N, exact=True)
    m = tri >= 0
    assert m.sum() > 100
    assert np.abs(ve - vf)[m].max() < 1e-6           # same pieces; sums in another order
    assert np.abs(ve - vd)[m].max() < 1e-4           # the FP64 oracle bar
    assert np.abs(Ge - Ed)[m].max() < 1e-6           # FP64 Lambert accumulation
    assert _stats_equal(ste, st) == {}


REF_SCENES = {
    # the reference's own scenes, ingested from configs (its tests/test_wavefront.cpp runs
    # plant, room and random_tris)
    "random_tris": "mesh procedural random_tris n=300 seed=1 size=0.3\nup 0 1 0\n"
                   "view 0.5 0.6 3.0  0.5 0.5 0.5  50\npoint_light 1.5 2.5 1.8\n"
                   "area_light 0.6 2.2 0.7  0.5 0 0  0 0 0.5\n",
    "ref_room": "mesh procedural room\nup 0 1 0\nview 2 1.4 2  5 0.8 5  70\npoint_light 5.5 2.6 2.5\n"
                "area_light 4 2.95 4  1 0 0  0 0 1\n",
    "ref_plant": "mesh procedural plant\nup 0 1 0\nview 2.6 1.7 3.4  0 0.55 0  45\npoint_light 1.0 3.0 0.8\n"
                 "area_light 0.9 2.8 0.7  0.4 0 0  0 0 0.4\n",
    # a closed sphere over a floor (the reference's crack-test scene) and its tessellation sweep
    "ref_sphere": "mesh procedural sphere stacks=16\nmesh procedural floorquad y=-1.2 size=8\nup 0 1 0\n"
                  "view 0.3 0.8 3.2  0 0 0  45\npoint_light 1.5 3.0 1.0\narea_light 1.2 3.0 0.8  0.6 0 0  0 0 0.6\n",
    "ref_tess_sweep": "mesh procedural tess_sweep stacks=8\nup 0 1 0\nview 0 5 9  0 0 0  55\n"
                      "point_light 2 6 2\narea_light 1 6 1  1 0 0  0 0 1\n",
    # its closed-form soft-shadow scene and a one-floor cut of its office building
    "ref_analytic": "mesh procedural analytic h=1 occ=1\nup 0 1 0\nview 0 5 5  0 0 0  60\n"
                    "point_light 0.3 3 0.2\narea_light 0 3 0  1 0 0  0 0 1\n",
    "ref_building": "mesh procedural building floors=1 rooms=2 detail=6\nup 0 1 0\n"
                    "view 1.0 1.6 2.4  6 1.2 2.6  70\npoint_light 2.5 2.6 2.5\n"
                    "area_light 2.5 2.75 2.5  0.8 0 0  0 0 0.8\n",
}


@pytest.mark.parametrize("name", list(REF_SCENES))
def test_reference_scenes_bitwise(name, native_lib, oracle_ready):
    """Primary and point pieces and counters bitwise, soft-point visibility
    within 1e-6 of the float build with identical counters, on the
    reference's own scenes."""
    from emu import Emulator
    from ref import RefTracer
    from beamtrace2007_b200.ingest import parse_config
    from beamtrace2007_b200.renderer import PreparedScene, make_camera
    s = parse_config(REF_SCENES[name])
    ps = PreparedScene(s.pos, s.tris)
    rf = RefTracer(s.pos, s.tris, "f")
    em = Emulator(ps)
    v = s.views[0]
    W, H = 80, 64
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    camv = cam.as_array()
    pe, ste = em.primary_tiles(cam, tile=16)
    pr, st = rf.primary_tiles(camv, W, H, tile=16)
    pr = to_f32(pr)
    assert np.array_equal(piece_keys(pe, True), piece_keys(pr, True))
    assert _stats_equal(ste, st) == {}
    hits = pr.select(pr.tri >= 0)
    assert len(hits) > 20
    light = np.array(s.point_light, np.float32)
    pe2, ste2 = em.point(cam, light, hits)
    pr2, st2 = rf.point_shadows(camv, W, H, light.astype(np.float64), hits)
    assert np.array_equal(piece_keys(pe2), piece_keys(to_f32(pr2)))
    assert _stats_equal(ste2, st2) == {}
    tri, X, N, _ = rf.primary_rays(camv, W, H)
    L = s.light_array()
    ve, _, ste3 = em.soft_points(L.astype(np.float32), ps.offset, tri, X.astype(np.float32), N.astype(np.float32),
                                 exact=True)
    vf, _, _, st3 = rf.soft_points(L, ps.offset, tri, X, N, exact=True)
    m = tri >= 0
    assert m.sum() > 100
    assert np.abs(ve - vf)[m].max() < 1e-6
    assert _stats_equal(ste3, st3) == {}

"""Host preparation vs the reference: Scene::finalize, KdTree::build and
Camera::make must be bit-identical (the tracer's output depends on all three)."""
import numpy as np
import pytest

from conftest import scene


@pytest.mark.parametrize("name", ["room", "plant", "analytic"])
def test_finalize_kdtree_camera_bitwise(name, native_lib, oracle_ready):
    from ref import RefTracer
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene(name)
    rf = RefTracer(s.pos, s.tris, "f")
    tris, triN, area, bounds = rf.scene_arrays()
    assert np.array_equal(ps.tris, tris)
    assert np.array_equal(ps.tri_normals, triN.astype(np.float32))
    assert np.array_equal(ps.tri_area, area.astype(np.float32))
    assert np.array_equal(ps.bounds, bounds.astype(np.float32))
    kd = rf.kd_arrays()
    assert np.array_equal(ps.kd_split, kd["split"].astype(np.float32))
    assert np.array_equal(ps.kd_data, kd["data"])
    assert np.array_equal(ps.kd_offset, kd["offset"])
    assert np.array_equal(ps.kd_parent, kd["parent"])
    assert np.array_equal(ps.kd_tri_indices, kd["tri_indices"])
    assert np.array_equal(ps.kd_box, kd["node_box"].astype(np.float32))
    assert np.array_equal(ps.kd_bounds, kd["bounds"].astype(np.float32))
    assert ps.kd_leaves == kd["leaves"] and ps.kd_max_depth == kd["max_depth"]
    v = s.views[0]
    for W, H in [(256, 256), (200, 120)]:
        cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
        assert np.array_equal(cam.as_array().astype(np.float32),
                              rf.camera_make(v.eye, v.target, v.fov, s.up, W, H).astype(np.float32))


def test_degenerate_triangles_dropped(native_lib, oracle_ready):
    """Zero-area and repeated-index triangles are removed as the reference does."""
    from ref import RefTracer
    from beamtrace2007_b200.renderer import PreparedScene
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [2, 0, 0], [1, 1, 1]], np.float32)
    tris = np.array([[0, 1, 2], [0, 1, 3], [1, 1, 2], [0, 2, 4], [2, 3, 4]], np.uint32)
    ps = PreparedScene(pos, tris)
    rf = RefTracer(pos, tris, "f")
    assert np.array_equal(ps.tris, rf.scene_arrays()[0])
    assert ps.num_tris == 3


def test_single_leaf_tree(native_lib, oracle_ready):
    from ref import RefTracer
    from beamtrace2007_b200.renderer import PreparedScene
    s, _ = scene("room")
    ps = PreparedScene(s.pos, s.tris, single_leaf=True)
    rf = RefTracer(s.pos, s.tris, "f", single_leaf=True)
    assert len(ps.kd_split) == 1
    assert np.array_equal(ps.kd_tri_indices, rf.kd_arrays()["tri_indices"])


def test_binned_sah_above_threshold(native_lib, oracle_ready):
    """A scene above the 2048-reference threshold exercises the binned SAH."""
    from ref import RefTracer
    from beamtrace2007_b200 import scenes
    from beamtrace2007_b200.renderer import PreparedScene
    s = scenes.icosphere(4, displace=0.1)
    ps = PreparedScene(s.pos, s.tris)
    rf = RefTracer(s.pos, s.tris, "f")
    kd = rf.kd_arrays()
    assert ps.num_tris > 2048
    assert np.array_equal(ps.kd_data, kd["data"])
    assert np.array_equal(ps.kd_split, kd["split"].astype(np.float32))
    assert np.array_equal(ps.kd_tri_indices, kd["tri_indices"])

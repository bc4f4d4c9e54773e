"""bt_kd_build_gpu: the SAH kd-tree built on the GPU is the host build's
tree (which tests/test_host_scene.py pins to the reference's
KdTree::build), array for array: split planes, node words, leaf offsets,
parents, node boxes, the leaves' triangle order, leaf count and depth --
on every scene family, with both split searches (binned SAH above the bin
threshold, the exact sweep below), with and without clipping, at a depth
limit, as a single leaf, and on interpenetrating triangles."""
import numpy as np
import pytest

from conftest import scene

ARRAYS = ("kd_split", "kd_data", "kd_offset", "kd_parent", "kd_box", "kd_tri_indices", "kd_bounds")


def _same_tree(a, b):
    for k in ARRAYS:
        x, y = getattr(a, k), getattr(b, k)
        assert x.shape == y.shape, (k, x.shape, y.shape)
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), k
    assert (a.kd_leaves, a.kd_max_depth) == (b.kd_leaves, b.kd_max_depth)


def test_gpu_build_rejects_bad_input(native_lib):
    """Argument checks come before any device work (so this runs without a
    GPU): an out-of-range triangle index is BT_ERR_INVALID."""
    import ctypes as C
    from beamtrace2007_b200 import _native as N
    pos = np.zeros((3, 3), np.float32)
    tris = np.array([[0, 1, 5]], np.uint32)
    area = np.ones(1, np.float32)
    b = np.array([0, 0, 0, 1, 1, 1], np.float32)
    h = C.c_void_p()
    assert N.lib().bt_kd_build_gpu(N.ptr(pos), 3, N.ptr(tris), N.ptr(area), 1, N.ptr(b), None, 0, C.byref(h),
                                   None) == -1  # BT_ERR_INVALID
    assert b"out of range" in N.lib().bt_gpu_last_error()


CASES = [
    ("room", {}, {}),
    ("plant", {}, {}),
    ("plant", {}, dict(bin_threshold=64, bins=16)),        # the binned search on a small scene
    ("plant", {}, dict(clip_bounds=0)),
    ("plant", {}, dict(max_depth=7)),
    ("plant", {}, dict(single_leaf=1)),
    ("displaced_sphere", {}, {}),
    ("building", dict(floors=2, furniture=6), {}),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,kd", CASES)
def test_gpu_tree_is_the_host_tree(name, kw, kd, gpu):
    from beamtrace2007_b200.renderer import PreparedScene
    s, _ = scene(name, **kw)
    host = PreparedScene(s.pos, s.tris, **kd)
    dev = PreparedScene(s.pos, s.tris, kd_device=0, **kd)
    _same_tree(dev, host)


@pytest.mark.gpu
def test_gpu_tree_interpenetrating_and_config_scenes(gpu):
    """Random interpenetrating triangles (many straddling references and
    coincident events) and the reference's own plant config."""
    from beamtrace2007_b200.ingest import parse_config
    from beamtrace2007_b200.renderer import PreparedScene
    for text in ("mesh procedural random_tris n=3000 seed=5 size=0.25\n", "mesh procedural plant\n",
                 "mesh procedural tess_sweep stacks=12\n"):
        sf = parse_config(text)
        _same_tree(PreparedScene(sf.pos, sf.tris, kd_device=0), PreparedScene(sf.pos, sf.tris))


@pytest.mark.gpu
def test_gpu_tree_full_building(gpu):
    """2.1M triangles: the same tree, and the GPU build's time beside the
    host build's."""
    from beamtrace2007_b200.renderer import PreparedScene
    s, host = scene("building")
    dev = PreparedScene(s.pos, s.tris, kd_device=0)
    _same_tree(dev, host)
    print(f"building kd build: host {host.kd_build_ms:.0f} ms, GPU {dev.kd_build_ms:.0f} ms")


def _grid_tris(n, z=0.0, jitter=0.0, seed=0):
    """n x n quads (2n^2 triangles) on the plane z (x, y in [-1, 1])."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(-1, 1, n + 1)
    pos = np.array([[x, y, z + jitter * rng.uniform(-1, 1)] for y in xs for x in xs], np.float32)
    tris = []
    for j in range(n):
        for i in range(n):
            a = j * (n + 1) + i
            tris += [[a, a + 1, a + n + 2], [a, a + n + 2, a + n + 1]]
    return pos, np.array(tris, np.uint32)


@pytest.mark.gpu
def test_gpu_tree_edge_cases(gpu):
    """Degenerate inputs: one triangle, two, a flat grid (planar events and a
    zero-extent axis), one triangle repeated (identical events), and a grid
    across zero (positions of both zero signs)."""
    from beamtrace2007_b200.renderer import PreparedScene
    one = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.uint32))
    two = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32), np.array([[0, 1, 2], [0, 1, 3]],
                                                                                          np.uint32))
    flat = _grid_tris(40)
    rep_pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    rep = (rep_pos, np.tile(np.array([[0, 1, 2]], np.uint32), (300, 1)))
    signed = _grid_tris(30, z=0.0, jitter=0.25, seed=4)
    signed[0][np.abs(signed[0]) < 1e-9] = -0.0
    for pos, tris in (one, two, flat, rep, signed):
        _same_tree(PreparedScene(pos, tris, kd_device=0), PreparedScene(pos, tris))

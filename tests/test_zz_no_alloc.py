"""bt_gpu_soft_points_noalloc: soft shadows for callers that cannot allocate
device memory.

An application whose own allocator owns the GPU's memory cannot call
cudaMalloc beside it; this entry point takes the scene and the shading
points in the caller's device buffers and works in a fixed scratch array
inside the library.  Its results must match bt_gpu_soft_points_device (the
context-based entry point) on the same points within the soft-shadow bars
of the parity tests, on two calls in a row: what the first call leaves in
the shared scratch array must not leak into the second.

This file is collected last, so a run that stops at its first failure has
run every other test before it."""
import ctypes as C

import numpy as np
import pytest

from conftest import scene

VIS_TOL = 1e-4   # |vis| bar of the soft-shadow parity tests
E_REL = 1e-5     # |E| bar, relative to the largest E


def _descs(pos, tris, nrm, bounds, split, data, offset, parent, box, tri_idx, kd_bounds, nv, nt, nn, nr):
    from beamtrace2007_b200 import _native as N
    sd = N.SceneDesc(pos, nv, tris, nrm, nt, (C.c_float * 6)(*bounds))
    kd = N.KdDesc(split, data, offset, parent, box, nn, tri_idx, nr, (C.c_float * 6)(*kd_bounds))
    return sd, kd


def _call(sd, kd, light, opts, n, tri, X, Nn, vis, E, Eu, info=None):
    from beamtrace2007_b200 import _native as N
    return N.lib().bt_gpu_soft_points_noalloc(C.byref(sd), C.byref(kd), C.byref(light), C.byref(opts), n, tri, X,
                                              Nn, vis, E, Eu, C.byref(info) if info is not None else None)


def test_sizes_over_the_limit_are_rejected(native_lib):
    """Too large a scene or too many points: BT_ERR_TOO_LARGE with a message
    naming the limit, before any GPU work (so this runs without a GPU)."""
    from beamtrace2007_b200 import _native as N
    dummy = np.zeros(16, np.float32)
    p = N.ptr(dummy)
    light = N.AreaLight.from_array(np.zeros(9, np.float32))
    opts = N.SoftOpts()
    b = [0, 0, 0, 1, 1, 1]
    # 2^21 kd nodes alone need 88 MiB
    sd, kd = _descs(p, p, p, b, p, p, p, p, p, p, b, 3, 1, 1 << 21, 1)
    assert _call(sd, kd, light, opts, 0, None, None, None, None, None, None) == -8
    assert b"BT_NOALLOC_SCRATCH_BYTES" in N.lib().bt_gpu_last_error()
    # a small scene with a million points: 168 MB of root records
    sd, kd = _descs(p, p, p, b, p, p, p, p, p, p, b, 3, 1, 1, 1)
    assert _call(sd, kd, light, opts, 1 << 20, p, p, p, p, p, p) == -8
    # bad arguments stay BT_ERR_INVALID
    assert _call(sd, kd, light, opts, -1, p, p, p, p, p, p) == -1


def _device_scene(ps):
    """The finalised scene and its kd-tree copied into device buffers that
    the test allocates (as the caller's own allocator would)."""
    import torch
    keep = {}

    def dev(a, name):
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint32:
            a = a.view(np.int32)
        t = torch.from_numpy(a).cuda()
        keep[name] = t
        return C.c_void_p(t.data_ptr())

    sd, kd = _descs(dev(ps.pos, "pos"), dev(ps.tris, "tris"), dev(ps.tri_normals, "nrm"), ps.bounds,
                    dev(ps.kd_split, "split"), dev(ps.kd_data, "data"), dev(ps.kd_offset, "offset"),
                    dev(ps.kd_parent, "parent"), dev(ps.kd_box, "box"), dev(ps.kd_tri_indices, "idx"),
                    ps.kd_bounds, len(ps.pos), len(ps.tris), len(ps.kd_split), len(ps.kd_tri_indices))
    return sd, kd, keep


@pytest.mark.gpu
def test_noalloc_matches_device_entry_point(gpu):
    import torch
    from beamtrace2007_b200 import _native as N
    from beamtrace2007_b200.renderer import GpuRenderer, make_camera
    s, ps = scene("plant")
    v = s.views[0]
    W, H = 128, 96
    n = W * H
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    lights = [s.light_array(1.0), s.light_array(4.0)]
    opts = N.SoftOpts()
    opts.exact = 1
    dev = torch.device("cuda:0")
    ref = []
    with GpuRenderer(ps) as g:
        tri = np.zeros(n, np.int32)
        X = np.zeros(3 * n, np.float32)
        Nn = np.zeros(3 * n, np.float32)
        N.check(N.lib().bt_gpu_primary_rays(g._h, C.byref(cam), N.ptr(tri), N.ptr(X), N.ptr(Nn)))
        dtri = torch.from_numpy(tri).to(dev)
        dX = torch.from_numpy(X).to(dev)
        dN = torch.from_numpy(Nn).to(dev)
        for L in lights:
            out = [torch.zeros(n, dtype=torch.float32, device=dev) for _ in range(3)]
            torch.cuda.synchronize()
            N.check(N.lib().bt_gpu_soft_points_device(
                g._h, C.byref(N.AreaLight.from_array(L)), C.byref(opts), n, dtri.data_ptr(), dX.data_ptr(),
                dN.data_ptr(), out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), None))
            ref.append([o.cpu().numpy() for o in out])
    m = tri >= 0
    assert m.sum() > n // 8
    sd, kd, keep = _device_scene(ps)
    # two calls in a row, each against the context-based entry point
    for L, (rv, rE, rEu) in zip(lights, ref):
        out = [torch.full((n,), 7.0, dtype=torch.float32, device=dev) for _ in range(3)]
        info = N.RunInfo()
        torch.cuda.synchronize()
        N.check(_call(sd, kd, N.AreaLight.from_array(L), opts, n, dtri.data_ptr(), dX.data_ptr(), dN.data_ptr(),
                      out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), info))
        vis, E, Eu = (o.cpu().numpy() for o in out)
        assert info.tri_tests > 0
        assert np.abs(vis - rv).max() <= VIS_TOL
        assert np.abs(E - rE).max() <= E_REL * np.abs(rE).max()
        assert np.abs(Eu - rEu).max() <= E_REL * np.abs(rEu).max()
        assert np.all(vis[~m] == -1)


def _defect(ps, what):
    """Host copies of the kd-tree and triangle arrays with one index made
    invalid; returns (array name, the bad copy, the phrase the error names)."""
    if what == "child":
        # an interior node whose child index points back at itself
        data = ps.kd_data.copy()
        i = int(np.nonzero((data & 3) != 3)[0][-1])
        data[i] = (np.uint32(i) << np.uint32(2)) | (data[i] & np.uint32(3))
        return "data", data, (b"kd node",)
    if what == "leaf":
        # a leaf whose reference range runs one past the end of the list
        data, offset = ps.kd_data, ps.kd_offset.copy()
        leaves = np.nonzero(((data & 3) == 3) & ((data >> 2) > 0))[0]
        i = int(leaves[0])
        offset[i] = np.uint32(len(ps.kd_tri_indices) - int(data[i] >> 2) + 1)
        return "offset", offset, (b"kd node",)
    if what == "reference":
        # a leaf reference to a triangle past the last one
        idx = ps.kd_tri_indices.copy()
        idx[0] = np.uint32(len(ps.tris))
        return "idx", idx, (b"kd reference",)
    # a referenced triangle whose last vertex index is past the last vertex
    # (found through its reference, or through the triangle itself when the
    # index is its first)
    tris = ps.tris.copy()
    tris[int(ps.kd_tri_indices[0]), 2] = np.uint32(len(ps.pos) + 5)
    return "tris", tris, (b"kd reference", b"triangle")


@pytest.mark.gpu
def test_noalloc_rejects_malformed_inputs(gpu):
    """A child index pointing backwards, a leaf range past the reference
    list, a reference past the last triangle and a vertex index past the
    last vertex: each returns BT_ERR_INVALID naming what is malformed (the
    packing kernel checks every index before it uses it, so no access goes
    out of range), and a valid call after them still gives the context
    entry point's results."""
    import torch
    from beamtrace2007_b200 import _native as N
    from beamtrace2007_b200.renderer import GpuRenderer, make_camera
    s, ps = scene("room")
    light = N.AreaLight.from_array(s.light_array())
    opts = N.SoftOpts()
    opts.exact = 1
    fields = {"data": "data", "offset": "offset", "idx": "tri_indices", "tris": "tris"}
    for what in ("child", "leaf", "reference", "vertex"):
        sd, kd, keep = _device_scene(ps)
        name, arr, phrases = _defect(ps, what)
        bad = torch.from_numpy(np.ascontiguousarray(arr).view(np.int32)).cuda()
        setattr(sd if name == "tris" else kd, fields[name], bad.data_ptr())
        torch.cuda.synchronize()
        assert _call(sd, kd, light, opts, 0, None, None, None, None, None, None) == -1, what
        msg = N.lib().bt_gpu_last_error()
        assert any(p in msg for p in phrases), (what, msg)
    # the next valid call, on points, against the context entry point
    v = s.views[0]
    W, H = 48, 40
    n = W * H
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    dev = torch.device("cuda:0")
    with GpuRenderer(ps) as g:
        tri = np.zeros(n, np.int32)
        X = np.zeros(3 * n, np.float32)
        Nn = np.zeros(3 * n, np.float32)
        N.check(N.lib().bt_gpu_primary_rays(g._h, C.byref(cam), N.ptr(tri), N.ptr(X), N.ptr(Nn)))
        dtri, dX, dN = (torch.from_numpy(a).to(dev) for a in (tri, X, Nn))
        ref = [torch.zeros(n, dtype=torch.float32, device=dev) for _ in range(3)]
        torch.cuda.synchronize()
        N.check(N.lib().bt_gpu_soft_points_device(g._h, C.byref(light), C.byref(opts), n, dtri.data_ptr(),
                                                  dX.data_ptr(), dN.data_ptr(), *(r.data_ptr() for r in ref), None))
    sd, kd, keep = _device_scene(ps)
    out = [torch.full((n,), 7.0, dtype=torch.float32, device=dev) for _ in range(3)]
    torch.cuda.synchronize()
    N.check(_call(sd, kd, light, opts, n, dtri.data_ptr(), dX.data_ptr(), dN.data_ptr(),
                  *(o.data_ptr() for o in out)))
    rv, rE, _ = (r.cpu().numpy() for r in ref)
    vis, E, _ = (o.cpu().numpy() for o in out)
    assert (tri >= 0).sum() > n // 4
    assert np.abs(vis - rv).max() <= VIS_TOL
    assert np.abs(E - rE).max() <= E_REL * np.abs(rE).max()


def test_fixed_queue_pool(native_lib):
    """The queues of the allocation-free call get what the scratch array
    leaves after the scene and the points (the layout of the header's limit:
    44 B per kd node, 64 per reference, 32 per triangle, 168 per point, each
    section rounded up to 256 B, plus a few small sections of counters):
    for the room scene at 128 x 96 points, 300,000 to 349,525 records per
    queue, as the header states -- about a hundredth of a context's 2^25 --
    and room for the admission of a warp's 32 roots at their initial
    reservation of 128 slots each, many times over."""
    _, ps = scene("room")

    def r256(b):
        return (b + 255) // 256 * 256
    nn, nr, nt, n = len(ps.kd_split), len(ps.kd_tri_indices), len(ps.tris), 128 * 96
    scene_and_points = (r256(8 * nn) + r256(32 * nn) + r256(4 * nn) + r256(64 * nr) + r256(32 * nt) + r256(96 * n)
                        + 6 * r256(4 * n) + 2 * r256(8 * n) + r256(32 * n))
    limit = 64 << 20
    caps = [(limit - scene_and_points - small) // (3 * 64) for small in (0, 16 << 10)]
    assert all(300_000 < c < 349_526 for c in caps)
    assert all(c >= 64 * 32 * 128 for c in caps)
    assert (1 << 25) // caps[0] >= 90

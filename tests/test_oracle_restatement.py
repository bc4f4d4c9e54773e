"""Pins of the FP64 restatement of soft-shadow visibility
(oracle/restate_soft.py) before it is trusted as a checker: the reference's
closed-form known answer (tests/test_tracing.cpp:255-312 of the reference)
and the reference's own double build on identical shading points."""
import numpy as np
import pytest

from conftest import scene


def _closed(px, pz, H, h, occ=1.0):
    k = H / h
    cx, cz, half = px * (1 - k), pz * (1 - k), occ * k / 2
    ox = max(0.0, min(0.5, cx + half) - max(-0.5, cx - half))
    oz = max(0.0, min(0.5, cz + half) - max(-0.5, cz - half))
    return 1 - ox * oz


def test_restatement_closed_form():
    """Square occluder (side 1 at height 1) under a unit square light at 3:
    the visible fraction on the floor has a closed form."""
    from restate_soft import soft_points
    from beamtrace2007_b200.scenes import Pcg32
    s, ps = scene("analytic")
    rng = Pcg32(23)
    pts = np.array([[rng.uniform(-1.5, 1.5), 0.0, rng.uniform(-1.5, 1.5)] for _ in range(60)])
    floor = next(t for t in range(ps.num_tris) if np.all(ps.pos[ps.tris[t]][:, 1] == 0))
    tri = np.full(len(pts), floor, np.int32)
    N = np.tile([0.0, 1.0, 0.0], (len(pts), 1))
    off = 1e-4
    vis, _ = soft_points(ps.pos, ps.tris, s.light_array(), off, tri, pts, N)
    ref = np.array([_closed(p[0], p[2], 3 - off, 1 - off) for p in pts])
    assert np.abs(vis - ref).max() < 1e-9


def test_restatement_vs_reference_double(oracle_ready):
    """On the plant, at shading points from the reference's primary rays:
    within 1e-7 of the reference's FP64 build (bt_render_d), vis and exact E."""
    from ref import RefTracer
    from restate_soft import soft_points
    from beamtrace2007_b200.renderer import make_camera
    s, ps = scene("plant")
    rf = RefTracer(s.pos, s.tris, "f")
    rd = RefTracer(s.pos, s.tris, "d")
    v = s.views[0]
    W, H = 40, 32
    cam = make_camera(v.eye, v.target, v.fov, s.up, W, H)
    tri, X, N, _ = rf.primary_rays(cam.as_array(), W, H)
    idx = np.nonzero(tri >= 0)[0][::7][:120]
    L = s.light_array(2.0)
    vd, Ed, _, _ = rd.soft_points(L, ps.offset, tri[idx], X[idx], N[idx], exact=True, threads=4)
    vr, Er = soft_points(ps.pos, ps.tris, L, ps.offset, tri[idx], X[idx], N[idx])
    assert (vr < 1).sum() > 20  # the sample has shadowed points
    assert np.abs(vr - vd).max() < 1e-7
    assert np.abs(Er - Ed).max() < 1e-7 * max(1.0, np.abs(Ed).max())


def test_restatement_vs_golden():
    """The committed fixture (tests/golden/make_golden.py: the reference's
    double build at its own shading points, light scales 1 and 4)."""
    import os
    from conftest import ROOT
    from restate_soft import soft_points
    g = np.load(os.path.join(ROOT, "tests", "golden", "plant_soft_points.npz"))
    s, ps = scene("plant")
    for k in range(len(g["scales"])):
        vr, Er = soft_points(ps.pos, ps.tris, g[f"light{k}"], float(g["offset"]), g["tri"],
                             g["X"].astype(np.float64), g["N"].astype(np.float64))
        assert np.abs(vr - g[f"vis{k}"]).max() < 1e-7
        assert np.abs(Er - g[f"E{k}"]).max() < 1e-7 * max(1.0, np.abs(g[f"E{k}"]).max())

"""Writes tests/golden/plant_soft_points.npz from the reference itself.

Run here, where the reference is compiled from its sources (oracle/_ref):
    python tests/golden/make_golden.py

Shading points: the reference float build's primary rays of the seeded
plant (a 40x32 camera on its first view; every 7th covered pixel, at most
120), so tri/X/N are the reference's own.  Outputs: visibility and exact E
of the reference's double build (bt_render_d, the FP64 oracle) at light
scales 1 and 4.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main():
    from ref import RefTracer
    from beamtrace2007_b200 import scenes
    from beamtrace2007_b200.renderer import PreparedScene
    s = scenes.plant()
    ps = PreparedScene(s.pos, s.tris)
    rf = RefTracer(s.pos, s.tris, "f")
    rd = RefTracer(s.pos, s.tris, "d")
    v = s.views[0]
    W, H = 40, 32
    cam = rf.camera_make(v.eye, v.target, v.fov, s.up, W, H)
    tri, X, N, _ = rf.primary_rays(cam, W, H)
    idx = np.nonzero(tri >= 0)[0][::7][:120]
    out = {"tri": tri[idx].astype(np.int32), "X": X[idx].astype(np.float32), "N": N[idx].astype(np.float32),
           "offset": np.float32(ps.offset), "scales": np.array([1.0, 4.0])}
    for k, sc in enumerate(out["scales"]):
        L = s.light_array(float(sc))
        vd, Ed, _, _ = rd.soft_points(L, ps.offset, out["tri"], out["X"].astype(np.float64),
                                      out["N"].astype(np.float64), exact=True, threads=4)
        out[f"light{k}"] = np.asarray(L, np.float32)
        out[f"vis{k}"] = vd
        out[f"E{k}"] = Ed
    np.savez_compressed(os.path.join(HERE, "plant_soft_points.npz"), **out)
    print("wrote", len(idx), "points")


if __name__ == "__main__":
    main()

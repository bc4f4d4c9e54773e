"""The kd slab decision is conservative (the reference's own fuzz test,
tests/test_geometry.cpp:115-227): for 4,000 random beams, boxes and split
planes, when this package's decide (beam_math.cuh, built for the host by
tests/native/emu.cpp) sends a beam to one child only, none of 64 rays inside
the beam -- its corners and random interior points, traced in double --
meets the other child within the box: with "far", every ray is past the
split plane where it enters the box; with "near", none reaches it before
leaving the box."""
import ctypes as C

import numpy as np

BEAMS, RAYS = 4000, 64
NEAR, FAR = 0, 1


def _emu():
    import build_emu
    lib = C.CDLL(build_emu.build())
    f = C.POINTER(C.c_float)
    lib.emu_decide.restype = C.c_int
    lib.emu_decide.argtypes = [f, f, f, f, f, f, C.c_int, C.c_int, C.c_float, f, f]
    return lib


def _f(a):
    return np.ascontiguousarray(a, np.float32).ctypes.data_as(C.POINTER(C.c_float))


def _segment(O, D, lo, hi):
    """[t0, t1] of the ray O + t D (t >= 0) inside the box, or None."""
    t0, t1 = 0.0, np.inf
    for c in range(3):
        if D[c] == 0:
            if O[c] < lo[c] or O[c] > hi[c]:
                return None
            continue
        ta, tb = (lo[c] - O[c]) / D[c], (hi[c] - O[c]) / D[c]
        t0, t1 = max(t0, min(ta, tb)), min(t1, max(ta, tb))
    return (t0, t1) if t0 <= t1 else None


def test_kd_decision_is_conservative():
    lib = _emu()
    rng = np.random.default_rng(11)
    decided = {NEAR: 0, FAR: 0}
    done = 0
    while done < BEAMS:
        O = rng.uniform(-1, 1, 3).astype(np.float32)
        d = rng.normal(size=3)
        p0 = (O + d / np.linalg.norm(d)).astype(np.float32)
        u = rng.normal(size=3).astype(np.float32)
        v = rng.normal(size=3).astype(np.float32)
        n = int(rng.integers(3, 5))
        ang = np.sort(rng.uniform(0, 2 * np.pi, n))
        r = rng.uniform(0.02, 0.4)
        qx = (r * np.cos(ang)).astype(np.float32)
        qy = (r * np.sin(ang)).astype(np.float32)
        lo = rng.uniform(-3, 1, 3)
        hi = lo + rng.uniform(0.2, 3, 3)
        box = np.concatenate([lo, hi]).astype(np.float32)
        axis = int(rng.integers(3))
        split = np.float32(box[axis] + rng.uniform(0.05, 0.95) * (box[3 + axis] - box[axis]))
        uvd = np.zeros(9, np.float32)
        dec = lib.emu_decide(_f(O), _f(p0), _f(u), _f(v), _f(qx), _f(qy), n, axis, C.c_float(split), _f(box),
                             _f(uvd))
        if dec < 0:
            continue  # not a pre-split piece, or the split behind the apex
        done += 1
        if dec not in (NEAR, FAR):
            continue
        decided[dec] += 1
        U, V, Dd = (uvd[3 * k:3 * k + 3].astype(np.float64) for k in range(3))
        w = rng.dirichlet(np.ones(n), RAYS - n)
        pts = np.concatenate([np.stack([qx, qy], 1), w @ np.stack([qx, qy], 1)]).astype(np.float64)
        Od, lo_d, hi_d = O.astype(np.float64), box[:3].astype(np.float64), box[3:].astype(np.float64)
        for x, y in pts:
            D = Dd + x * U + y * V
            seg = _segment(Od, D, lo_d, hi_d)
            if seg is None:
                continue
            t0, t1 = seg
            if D[axis] == 0:
                tsp = np.inf  # never reaches the split, which lies ahead
            else:
                tsp = (float(split) - Od[axis]) / D[axis]
            tol = 1e-5 * max(1.0, abs(tsp))
            if dec == FAR:
                assert tsp <= t0 + tol, ("far", O, p0, u, v, qx, qy, box, axis, split, x, y, tsp, t0)
            else:
                assert tsp >= t1 - tol, ("near", O, p0, u, v, qx, qy, box, axis, split, x, y, tsp, t1)
    assert decided[NEAR] > 100 and decided[FAR] > 100, decided

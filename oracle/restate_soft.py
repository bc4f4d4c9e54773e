"""Test infrastructure only: an independent FP64 restatement of exact
area-light soft shadows for supplied shading points.

The reference (joelsalzman/beamtrace2007) traces a beam from the shading
point through the light polygon, splitting it at every triangle that
partly covers it (src/beam/beam_core.h:386-546, src/render/render.cpp:
305-337).  The quantity it computes is geometric: the part of the light
polygon that the shading point sees.  This module computes the same
quantity another way, brute force and without the kd-tree, so that it
checks the tracer rather than repeating it:

  root     = the light quad in light-plane coordinates, clipped by the
             shading point's horizon (lightBeamSetup, src/render/
             soft_core.h:38-73); apex = x + offset * n;
  occluder = every triangle but the shading point's own, clipped to the
             slab between the apex and the light plane (the beam's far
             plane, q.farIsPlane), projected centrally from the apex onto
             the light plane (BeamPlane::project, src/beam/beam_types.h:
             28-37): a convex polygon;
  visible  = root minus the union of the occluders, kept as a list of
             convex pieces (each occluder splits every piece it overlaps
             edge by edge; its inside is dropped);
  vis      = area(visible) / area(light quad);
  E        = sum over the visible pieces of Lambert's polygon integral
             seen from x with normal n (polygonFormFactorG,
             src/render/soft_core.h:18-33), exact mode.

Everything is float64 numpy; the per-piece polygon work runs in Python
loops on the few triangles that survive a vectorised cull, so this is for
hundreds of points, not images.
"""
from __future__ import annotations

import numpy as np


def _light_frame(c, U, V):
    """Orthonormal basis (e1, e2) of the light plane and its unit normal."""
    nL = np.cross(U, V)
    nL /= np.linalg.norm(nL)
    e1 = U / np.linalg.norm(U)
    e2 = np.cross(nL, e1)
    return e1, e2, nL


def _area(P):
    x, y = P[:, 0], P[:, 1]
    return 0.5 * float(np.dot(x, np.roll(y, -1)) - np.dot(np.roll(x, -1), y))


def _clip_halfplane(P, a, b, c):
    """Part of convex polygon P (k x 2) with a x + b y + c >= 0."""
    if len(P) == 0:
        return P
    d = P[:, 0] * a + P[:, 1] * b + c
    out = []
    k = len(P)
    for i in range(k):
        j = (i + 1) % k
        if d[i] >= 0:
            out.append(P[i])
        if (d[i] >= 0) != (d[j] >= 0):
            t = d[i] / (d[i] - d[j])
            out.append(P[i] + t * (P[j] - P[i]))
    return np.array(out) if len(out) >= 3 else np.zeros((0, 2))


def _clip3(P, nrm, off):
    """Part of a 3D convex polygon with nrm . p + off >= 0."""
    d = P @ nrm + off
    out = []
    k = len(P)
    for i in range(k):
        j = (i + 1) % k
        if d[i] >= 0:
            out.append(P[i])
        if (d[i] >= 0) != (d[j] >= 0):
            t = d[i] / (d[i] - d[j])
            out.append(P[i] + t * (P[j] - P[i]))
    return np.array(out) if len(out) >= 3 else np.zeros((0, 3))


def _subtract(pieces, Q, tiny):
    """Convex pieces minus convex polygon Q (counter-clockwise)."""
    qlo, qhi = Q.min(0), Q.max(0)
    out = []
    for P in pieces:
        if (P.max(0) < qlo).any() or (P.min(0) > qhi).any():
            out.append(P)
            continue
        cur = P
        k = len(Q)
        for i in range(k):
            p, q = Q[i], Q[(i + 1) % k]
            # inside Q is the left of p->q: a x + b y + c >= 0
            a, b = -(q[1] - p[1]), q[0] - p[0]
            c = -(a * p[0] + b * p[1])
            outside = _clip_halfplane(cur, -a, -b, -c)
            if len(outside) and _area(outside) > tiny:
                out.append(outside)
            cur = _clip_halfplane(cur, a, b, c)
            if len(cur) == 0:
                break
    return out


def _form_factor(x, n, P3):
    """Lambert's formula: integral of cos cos / r^2 over a planar polygon."""
    s = 0.0
    k = len(P3)
    for i in range(k):
        a, b = P3[i] - x, P3[(i + 1) % k] - x
        la, lb = np.linalg.norm(a), np.linalg.norm(b)
        if la == 0 or lb == 0:
            continue
        cth = np.clip(np.dot(a, b) / (la * lb), -1.0, 1.0)
        g = np.cross(a, b)
        lg = np.linalg.norm(g)
        if lg == 0:
            continue
        s += np.arccos(cth) * np.dot(g, n) / lg
    return abs(s) * 0.5


def soft_points(pos, tris, light, offset, tri, X, N):
    """vis and exact E for each shading point (tri < 0: vis -1, E 0)."""
    pos = np.asarray(pos, np.float64)
    tris = np.asarray(tris, np.int64)
    L = np.asarray(light, np.float64).ravel()
    c, U, V = L[0:3], L[3:6], L[6:9]
    e1, e2, nL = _light_frame(c, U, V)
    hu, hv = np.linalg.norm(U) / 2, np.linalg.norm(V) / 2
    # the light quad in (e1, e2) coordinates
    uq = np.array([np.dot(U, e1), np.dot(U, e2)]) / 2
    vq = np.array([np.dot(V, e1), np.dot(V, e2)]) / 2
    quad = np.array([-uq - vq, uq - vq, uq + vq, -uq + vq])
    if _area(quad) < 0:
        quad = quad[::-1]
    light_area = _area(quad)
    tiny = light_area * 1e-15
    V0, V1, V2 = pos[tris[:, 0]], pos[tris[:, 1]], pos[tris[:, 2]]
    n = len(tri)
    vis = np.full(n, -1.0)
    E = np.zeros(n)
    for k in range(n):
        if tri[k] < 0:
            continue
        x = np.asarray(X[k], np.float64)
        ns = np.asarray(N[k], np.float64)
        h = np.dot(x - c, nL)
        if not h > 0:  # behind the emitter
            vis[k] = 0.0
            continue
        apex = x + ns * offset
        ha = np.dot(apex - c, nL)
        # horizon: ns . (p - x) >= 0 for p = c + s e1 + t e2
        root = _clip_halfplane(quad, np.dot(ns, e1), np.dot(ns, e2), np.dot(ns, c - x))
        if len(root) == 0 or _area(root) <= 0:
            vis[k] = 0.0
            continue
        # cull: triangles with a vertex strictly between the apex and the light plane
        dv = [np.dot(Vi - c, nL) for Vi in (V0, V1, V2)]  # height above the light plane
        dmin = np.minimum(np.minimum(dv[0], dv[1]), dv[2])
        dmax = np.maximum(np.maximum(dv[0], dv[1]), dv[2])
        cand = (dmax > 0) & (dmin < ha)
        cand[tri[k]] = False
        # projected bounding box of fully-in-front triangles
        idx = np.nonzero(cand)[0]
        rlo, rhi = root.min(0), root.max(0)
        keep = []
        for t in idx:
            P = np.stack([V0[t], V1[t], V2[t]])
            hp = P @ nL - np.dot(c, nL)
            if (hp < ha).all():
                lam = ha / (ha - hp)
                Q = apex + (P - apex) * lam[:, None]
                s = (Q - c) @ e1
                tt = (Q - c) @ e2
                if s.max() < rlo[0] or s.min() > rhi[0] or tt.max() < rlo[1] or tt.min() > rhi[1]:
                    continue
            keep.append(t)
        pieces = [root]
        for t in keep:
            P = np.stack([V0[t], V1[t], V2[t]])
            # between the light plane (height > 0) and the apex's parallel plane (height < ha)
            P = _clip3(P, nL, -np.dot(c, nL))
            if len(P) == 0:
                continue
            # (just below the apex plane: points on it project to infinity,
            # and everything that close to it projects far outside the light)
            P = _clip3(P, -nL, np.dot(c, nL) + ha * (1 - 1e-9))
            if len(P) == 0:
                continue
            hp = P @ nL - np.dot(c, nL)
            lam = ha / (ha - hp)
            Q = apex + (P - apex) * lam[:, None]
            q2 = np.stack([(Q - c) @ e1, (Q - c) @ e2], 1)
            a = _area(q2)
            if abs(a) <= tiny:
                continue
            if a < 0:
                q2 = q2[::-1]
            pieces = _subtract(pieces, q2, tiny)
            if not pieces:
                break
        vis[k] = sum(_area(p) for p in pieces) / light_area
        E[k] = sum(_form_factor(x, ns, c + p[:, 0:1] * e1 + p[:, 1:2] * e2) for p in pieces)
    return vis, E

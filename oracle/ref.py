"""ctypes wrapper over the oracle libraries.  Test infrastructure only.

``RefTracer`` drives the reference's own CPU beam tracer, compiled from its
sources by ``oracle/Makefile`` into ``oracle/_ref/libbtref_{f,d}.so``
(Real = float for the float build, Real = double for the FP64 oracle,
``bt_render`` / ``bt_render_d`` of joelsalzman/beamtrace2007).  Nothing in the
package imports this module; tests, ``__graft_entry__.smoke()`` and the CPU
legs of ``bench.py`` do.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

# TraceStats field order (src/util/stats.h:8-42), as packed by ref_capi.cpp.
STAT_NAMES = ("kdSteps", "leafVisits", "triTests", "hits", "splits", "beams", "rootBeams", "presplitBeams",
              "mailboxSkips", "fiveSplits", "visibleTris", "rays", "climbs")

_P = C.c_void_p


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def ref_available(prec: str = "f") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libbtref_{prec}.so"))


_LIBS: dict = {}


def _lib(prec: str):
    if prec in _LIBS:
        return _LIBS[prec]
    path = os.path.join(REF_DIR, f"libbtref_{prec}.so")
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference sources exist")
    lib = C.CDLL(path)
    lib.btr_create.restype = _P
    lib.btr_create.argtypes = [_P, C.c_int64, _P, C.c_int64, C.c_double, C.c_int]
    lib.btr_destroy.argtypes = [_P]
    lib.btr_num_tris.restype = C.c_int64
    lib.btr_num_tris.argtypes = [_P]
    lib.btr_primary_tiles.restype = C.c_int64
    lib.btr_point_shadows.restype = C.c_int64
    lib.btr_form_factor.restype = C.c_double
    lib.btr_real_size.restype = C.c_int
    _LIBS[prec] = lib
    return lib


def unpack_stats(s: np.ndarray) -> dict:
    d = {k: int(s[i]) for i, k in enumerate(STAT_NAMES)}
    d["droppedArea"] = float(s[13:14].view(np.float64)[0])
    return d


@dataclass
class Polys:
    """Output pieces: corners (n, 4) x/y, corner count, triangle, area, root."""
    x: np.ndarray
    y: np.ndarray
    n: np.ndarray
    tri: np.ndarray
    area: np.ndarray
    root: np.ndarray

    def __len__(self):
        return len(self.n)


def _alloc_polys(cap):
    return Polys(np.zeros((cap, 4)), np.zeros((cap, 4)), np.zeros(cap, np.int32), np.zeros(cap, np.int32),
                 np.zeros(cap), np.zeros(cap, np.int32))


def _trim(p: Polys, n) -> Polys:
    return Polys(p.x[:n], p.y[:n], p.n[:n], p.tri[:n], p.area[:n], p.root[:n])


class RefTracer:
    """The reference CPU tracer on one scene (Scene::finalize + KdTree::build)."""

    def __init__(self, pos: np.ndarray, tris: np.ndarray, prec: str = "f", cost_intersect: float = 0.4,
                 single_leaf: bool = False):
        self.prec = prec
        self.lib = _lib(prec)
        pos = np.ascontiguousarray(pos, np.float32)
        tris = np.ascontiguousarray(tris, np.uint32)
        # a c_void_p, so that calls without declared argument types still pass
        # the whole 64-bit pointer (a bare int would go as a 32-bit C int)
        self.h = C.c_void_p(self.lib.btr_create(_ptr(pos), len(pos), _ptr(tris), len(tris), float(cost_intersect),
                                                int(single_leaf)))
        self.num_tris = int(self.lib.btr_num_tris(self.h))

    def close(self):
        if self.h is not None and self.h.value:
            self.lib.btr_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- scene and tree ----
    def scene_arrays(self):
        nt = self.num_tris
        tris = np.zeros((nt, 3), np.uint32)
        triN = np.zeros((nt, 3))
        area = np.zeros(nt)
        bounds = np.zeros(6)
        self.lib.btr_scene_export(self.h, _ptr(tris), _ptr(triN), _ptr(area), _ptr(bounds))
        return tris, triN, area, bounds

    def kd_arrays(self):
        sz = np.zeros(5, np.int64)
        self.lib.btr_kd_sizes(self.h, _ptr(sz))
        nn, nr = int(sz[0]), int(sz[1])
        split = np.zeros(nn)
        data = np.zeros(nn, np.uint32)
        offset = np.zeros(nn, np.uint32)
        idx = np.zeros(max(nr, 1), np.uint32)
        parent = np.zeros(nn, np.uint32)
        box = np.zeros((nn, 6))
        bounds = np.zeros(6)
        self.lib.btr_kd_export(self.h, _ptr(split), _ptr(data), _ptr(offset), _ptr(idx), _ptr(parent), _ptr(box),
                               _ptr(bounds))
        return dict(split=split, data=data, offset=offset, tri_indices=idx[:nr], parent=parent, node_box=box,
                    bounds=bounds, leaves=int(sz[2]), max_depth=int(sz[3]), build_ms=int(sz[4]))

    @staticmethod
    def tolerances(prec: str = "f"):
        out = np.zeros(3)
        _lib(prec).btr_tolerances(_ptr(out))
        return dict(eps_rel=out[0], kd_rel=out[1], deg_rel=out[2])

    # ---- camera ----
    def camera_make(self, eye, target, fov, up, W, H) -> np.ndarray:
        out = np.zeros(14)
        e, t, u = (np.asarray(v, np.float64) for v in (eye, target, up))
        self.lib.btr_camera_make(_ptr(e), _ptr(t), C.c_double(fov), _ptr(u), int(W), int(H), _ptr(out))
        return out

    # ---- soft shadows ----
    def primary_rays(self, cam: np.ndarray, W: int, H: int, threads: int = 1):
        n = W * H
        tri = np.zeros(n, np.int32)
        X = np.zeros((n, 3))
        N = np.zeros((n, 3))
        st = np.zeros(14, np.uint64)
        cam = np.ascontiguousarray(cam, np.float64)
        self.lib.btr_primary_rays(self.h, _ptr(cam), int(W), int(H), int(threads), _ptr(tri), _ptr(X), _ptr(N),
                                  _ptr(st))
        return tri, X, N, unpack_stats(st)

    def soft_points(self, light: np.ndarray, offset: float, tri, X, N, exact=False, mailbox=False, trail=True,
                    threads: int = 1):
        tri = np.ascontiguousarray(tri, np.int32)
        X = np.ascontiguousarray(X, np.float64)
        N = np.ascontiguousarray(N, np.float64)
        n = len(tri)
        vis, E, Eu = np.zeros(n), np.zeros(n), np.zeros(n)
        st = np.zeros(14, np.uint64)
        light = np.ascontiguousarray(light, np.float64)
        self.lib.btr_soft_points(self.h, _ptr(light), C.c_double(offset), C.c_int64(n), _ptr(tri), _ptr(X),
                                 _ptr(N), int(exact), int(mailbox), int(trail), int(threads), _ptr(vis), _ptr(E),
                                 _ptr(Eu), _ptr(st))
        return vis, E, Eu, unpack_stats(st)

    def soft_points_ray(self, light, offset, tri, X, N, px, py, samples=256, jitter=True, threads=1):
        tri = np.ascontiguousarray(tri, np.int32)
        X = np.ascontiguousarray(X, np.float64)
        N = np.ascontiguousarray(N, np.float64)
        px = np.ascontiguousarray(px, np.int32)
        py = np.ascontiguousarray(py, np.int32)
        vis = np.zeros(len(tri))
        light = np.ascontiguousarray(light, np.float64)
        self.lib.btr_soft_points_ray(self.h, _ptr(light), C.c_double(offset), C.c_int64(len(tri)), _ptr(tri),
                                     _ptr(X), _ptr(N), _ptr(px), _ptr(py), int(samples), int(jitter), int(threads),
                                     _ptr(vis))
        return vis

    def soft_image(self, cam, W, H, light, exact=False, threads=1, mailbox=True, trail=False):
        n = W * H
        tri = np.zeros(n, np.int32)
        vis, E, Eu = (np.zeros(n, np.float32) for _ in range(3))
        timing = np.zeros(2)
        st = np.zeros(14, np.uint64)
        cam = np.ascontiguousarray(cam, np.float64)
        light = np.ascontiguousarray(light, np.float64)
        self.lib.btr_soft_image(self.h, _ptr(cam), int(W), int(H), _ptr(light), int(exact), int(threads),
                                int(mailbox), int(trail), _ptr(tri), _ptr(vis), _ptr(E), _ptr(Eu), _ptr(timing),
                                _ptr(st))
        return dict(tri=tri, vis=vis, E=E, Eu=Eu, primary_s=timing[0], trace_s=timing[1], stats=unpack_stats(st))

    # ---- primary visibility and point shadows ----
    def primary_tiles(self, cam, W, H, cull=False, tile=16, mailbox=False, trail=True, cap=None) -> tuple:
        cap = cap or max(1 << 16, 4 * W * H)
        p = _alloc_polys(cap)
        st = np.zeros(14, np.uint64)
        cam = np.ascontiguousarray(cam, np.float64)
        n = self.lib.btr_primary_tiles(self.h, _ptr(cam), int(W), int(H), int(cull), int(tile), int(mailbox),
                                       int(trail), C.c_int64(cap), _ptr(p.x), _ptr(p.y), _ptr(p.n), _ptr(p.tri),
                                       _ptr(p.area), _ptr(p.root), _ptr(st))
        if n > cap:
            return self.primary_tiles(cam, W, H, cull, tile, mailbox, trail, cap=int(n))
        return _trim(p, int(n)), unpack_stats(st)

    def point_shadows(self, cam, W, H, light, hits: Polys, mailbox=False, trail=True, cap=None) -> tuple:
        cap = cap or max(1 << 16, 4 * len(hits))
        p = _alloc_polys(cap)
        st = np.zeros(14, np.uint64)
        cam = np.ascontiguousarray(cam, np.float64)
        light = np.ascontiguousarray(light, np.float64)
        hx = np.ascontiguousarray(hits.x, np.float64)
        hy = np.ascontiguousarray(hits.y, np.float64)
        hn = np.ascontiguousarray(hits.n, np.int32)
        ht = np.ascontiguousarray(hits.tri, np.int32)
        n = self.lib.btr_point_shadows(self.h, _ptr(cam), int(W), int(H), _ptr(light), C.c_int64(len(hits)),
                                       _ptr(hx), _ptr(hy), _ptr(hn), _ptr(ht), int(mailbox), int(trail),
                                       C.c_int64(cap), _ptr(p.x), _ptr(p.y), _ptr(p.n), _ptr(p.tri), _ptr(p.area),
                                       _ptr(p.root), _ptr(st))
        if n > cap:
            return self.point_shadows(cam, W, H, light, hits, mailbox, trail, cap=int(n))
        return _trim(p, int(n)), unpack_stats(st)

    def rasterize(self, cam, W, H, prim: Polys, shadow: Polys | None = None):
        tri = np.zeros(W * H, np.int32)
        flag = np.zeros(W * H, np.uint8)
        cam = np.ascontiguousarray(cam, np.float64)
        args = []
        for p in (prim, shadow):
            if p is None or len(p) == 0:
                args += [C.c_int64(0), None, None, None, None]
            else:
                args += [C.c_int64(len(p)), _ptr(np.ascontiguousarray(p.x, np.float64)),
                         _ptr(np.ascontiguousarray(p.y, np.float64)), _ptr(np.ascontiguousarray(p.n, np.int32)),
                         _ptr(np.ascontiguousarray(p.tri, np.int32))]
        # keep the converted arrays alive for the call
        keep = [prim, shadow]
        self.lib.btr_rasterize(_ptr(cam), int(W), int(H), *args, _ptr(tri), _ptr(flag))
        del keep
        return tri.reshape(H, W), flag.reshape(H, W)

    def form_factor(self, x, n, poly) -> float:
        x = np.ascontiguousarray(x, np.float64)
        n = np.ascontiguousarray(n, np.float64)
        poly = np.ascontiguousarray(poly, np.float64)
        return float(self.lib.btr_form_factor(_ptr(x), _ptr(n), _ptr(poly), int(len(poly))))


def ref_gpu_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libbtref_gpu.so"))


class RefGpu:
    """The reference's own GPU renderer (cuda/gpu_render.cu + cuda/wavefront.cu
    compiled for sm_100a from its sources by `make -C oracle ref_gpu`), driven
    through oracle/ref_gpu_capi.cpp.  Baseline timing only."""

    def __init__(self, pos: np.ndarray, tris: np.ndarray, cost_intersect: float = 0.4):
        lib = C.CDLL(os.path.join(REF_DIR, "libbtref_gpu.so"))
        lib.btrg_available.restype = C.c_int
        lib.btrg_create.restype = C.c_void_p
        lib.btrg_create.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_double]
        lib.btrg_soft.restype = None
        lib.btrg_soft.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p]
        lib.btrg_destroy.restype = None
        lib.btrg_destroy.argtypes = [C.c_void_p]
        lib.btrg_primary_point.restype = None
        lib.btrg_primary_point.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        self.lib = lib
        pos = np.ascontiguousarray(pos, np.float32)
        tris = np.ascontiguousarray(tris, np.uint32)
        self.h = lib.btrg_create(pos.ctypes.data, len(pos), tris.ctypes.data, len(tris), float(cost_intersect))

    def soft(self, cam, W, H, light, exact=True) -> dict:
        """GpuRenderer::softShadows; timing = primary s, trace s, kernel s,
        CPU-fallback s, overflow pixels (gpu_render.h:59-64)."""
        n = W * H
        tri = np.zeros(n, np.int32)
        vis, E = np.zeros(n, np.float32), np.zeros(n, np.float32)
        tm = np.zeros(5)
        cam = np.ascontiguousarray(cam, np.float64)
        light = np.ascontiguousarray(light, np.float64)
        self.lib.btrg_soft(self.h, cam.ctypes.data, int(W), int(H), light.ctypes.data, int(exact), tri.ctypes.data,
                           vis.ctypes.data, E.ctypes.data, tm.ctypes.data)
        return dict(tri=tri, vis=vis, E=E, primary_s=tm[0], trace_s=tm[1], kernel_s=tm[2], fallback_s=tm[3],
                    overflow_px=int(tm[4]))

    def primary_point(self, cam, W, H, light, tile=16) -> dict:
        """GpuRenderer::primary (tile roots) then pointShadows on its hit
        polygons, each wall-clocked around the synchronous call."""
        out = np.zeros(10)
        cam = np.ascontiguousarray(cam, np.float64)
        light = np.ascontiguousarray(light, np.float64)
        self.lib.btrg_primary_point(self.h, cam.ctypes.data, int(W), int(H), int(tile), light.ctypes.data,
                                    out.ctypes.data)
        return dict(primary_s=out[0], point_s=out[1], hits=int(out[2]), shadow_polys=int(out[3]),
                    primary_kernel_s=out[4], point_kernel_s=out[5], primary_overflow=int(out[6]),
                    point_overflow=int(out[7]), primary_fallback_s=out[8], point_fallback_s=out[9])

    def close(self):
        if self.h:
            self.lib.btrg_destroy(self.h)
            self.h = None


def ref_config(text: str, prec: str = "f") -> dict:
    """The reference's parseConfig + buildScene on config text: its scene
    (pos, tris, tri_mat, mat_color), views (eye, target, fov per row) and
    lights, as float64 copies of its Real values.  Raises ValueError with
    the reference's message when it rejects the config."""
    lib = _lib(prec)
    lib.btr_config_build.restype = _P
    lib.btr_config_build.argtypes = [C.c_char_p]
    lib.btr_config_error.restype = C.c_char_p
    lib.btr_config_free.argtypes = [_P]
    lib.btr_config_counts.argtypes = [_P, _P]
    lib.btr_config_arrays.argtypes = [_P] * 7
    h = lib.btr_config_build(text.encode())
    if not h:
        raise ValueError(lib.btr_config_error().decode(errors="replace"))
    h = C.c_void_p(h)
    try:
        n = np.zeros(7, np.int64)
        lib.btr_config_counts(h, _ptr(n))
        nv, nt, nm, nview = (int(x) for x in n[:4])
        out = dict(pos=np.zeros((nv, 3)), tris=np.zeros((nt, 3), np.uint32), tri_mat=np.zeros(nt, np.uint16),
                   mat_color=np.zeros((nm, 3)), views=np.zeros((nview, 7)), lights=np.zeros(22))
        lib.btr_config_arrays(h, *(_ptr(out[k]) for k in ("pos", "tris", "tri_mat", "mat_color", "views", "lights")))
        out.update(cull_backfaces=bool(n[4]), has_point_light=bool(n[5]), has_area_light=bool(n[6]))
        return out
    finally:
        lib.btr_config_free(h)

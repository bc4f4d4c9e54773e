"""Host-side mirror of the reference's GPU renderer interface.

``GpuRenderer`` keeps the names and meaning of ``bt::GpuRenderer``
(cuda/gpu_render.h:26-73 of joelsalzman/beamtrace2007): ``soft_shadows``,
``primary``, ``point_shadows``, the tunables ``wf_budget``,
``wf_primary_budget``, ``wf_capacity`` and the last-run fields
``last_rounds``, ``last_max_queue``, ``last_overflow_pixels``,
``last_kernel_seconds``.  Differences: errors raise ``BtError`` instead of
aborting, and roots over budget are retried on the GPU (``last_overflow_pixels``
counts them), never recomputed on the CPU.

``PreparedScene`` is the host preparation the reference does before
constructing its renderer: Scene::finalize and KdTree::build (beam SAH cost
0.4, apps/bt_render.cpp:172), both through the C-ABI.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from ._native import check, ptr


@dataclass
class PolyList:
    """Polygons on a query plane (OutBeam): x, y (m, 4) with the last corner
    repeated for triangles, n, tri, area and the root each came from."""
    x: np.ndarray
    y: np.ndarray
    n: np.ndarray
    tri: np.ndarray
    area: np.ndarray
    root: np.ndarray

    def __len__(self):
        return int(len(self.n))

    @staticmethod
    def alloc(cap: int) -> "PolyList":
        # uninitialised: the library fills the first `count` entries and
        # head() keeps only those (zeroing a frame-sized buffer costs more
        # than a small frame's whole engine run)
        cap = max(int(cap), 1)
        return PolyList(np.empty((cap, 4), np.float32), np.empty((cap, 4), np.float32), np.empty(cap, np.int32),
                        np.empty(cap, np.int32), np.empty(cap, np.float32), np.empty(cap, np.int32))

    def struct(self) -> N.Polys:
        for a in (self.x, self.y, self.n, self.tri, self.area, self.root):
            assert a.flags["C_CONTIGUOUS"]
        return N.Polys(ptr(self.x), ptr(self.y), ptr(self.n), ptr(self.tri), ptr(self.area), ptr(self.root),
                       len(self.n))

    def head(self, k: int) -> "PolyList":
        return PolyList(self.x[:k], self.y[:k], self.n[:k], self.tri[:k], self.area[:k], self.root[:k])

    def select(self, m) -> "PolyList":
        return PolyList(*(np.ascontiguousarray(a[m]) for a in (self.x, self.y, self.n, self.tri, self.area,
                                                               self.root)))


def make_camera(eye, target, fov: float, up, W: int, H: int) -> N.Camera:
    """Camera::make (src/render/render.cpp:14-25) through the C-ABI."""
    cam = N.Camera()
    e = np.asarray(eye, np.float32)
    t = np.asarray(target, np.float32)
    u = np.asarray(up, np.float32)
    N.lib().bt_camera_make(ptr(e), ptr(t), C.c_float(fov), ptr(u), int(W), int(H), C.byref(cam))
    return cam


def kd_params_default(cost_intersect: float = 0.4) -> dict:
    """The kd-tree build parameters PreparedScene uses by default."""
    kp = N.KdParams()
    N.lib().bt_kd_params_default(C.byref(kp))
    kp.cost_intersect = cost_intersect
    return {k: getattr(kp, k) for k, _ in kp._fields_}


class PreparedScene:
    """A finalised scene and its kd-tree, as host arrays.  The tree is built
    on the host (bt_kd_build) or, with `kd_device`, on that CUDA device
    (bt_kd_build_gpu: the same tree); `kd` overrides other bt_kd_params
    fields.  `kd_build_ms`: the build's wall-clock time."""

    def __init__(self, pos: np.ndarray, tris: np.ndarray, cost_intersect: float = 0.4, single_leaf: bool = False,
                 kd_device: int | None = None, **kd):
        L = N.lib()
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        tris_in = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
        nt_in = len(tris_in)
        tris_out = np.zeros((max(nt_in, 1), 3), np.uint32)
        tri_n = np.zeros((max(nt_in, 1), 3), np.float32)
        area = np.zeros(max(nt_in, 1), np.float32)
        bounds = np.zeros(6, np.float32)
        nt = L.bt_scene_finalize(ptr(pos), len(pos), ptr(tris_in), nt_in, ptr(tris_out), ptr(tri_n), ptr(area),
                                 ptr(bounds))
        if nt < 0:
            raise N.BtError(-1, "triangle index out of range")
        if nt == 0:
            raise N.BtError(-1, "scene has no triangles")
        self.pos = pos
        self.tris = np.ascontiguousarray(tris_out[:nt])
        self.tri_normals = np.ascontiguousarray(tri_n[:nt])
        self.tri_area = np.ascontiguousarray(area[:nt])
        self.bounds = bounds
        kp = N.KdParams()
        L.bt_kd_params_default(C.byref(kp))
        kp.cost_intersect = cost_intersect
        kp.single_leaf = int(single_leaf)
        for k, v in kd.items():
            setattr(kp, k, v)
        h = C.c_void_p()
        t0 = time.perf_counter()
        if kd_device is None:
            check(L.bt_kd_build(ptr(self.pos), ptr(self.tris), ptr(self.tri_area), nt, ptr(self.bounds), C.byref(kp),
                                C.byref(h)))
        else:
            check(L.bt_kd_build_gpu(ptr(self.pos), len(self.pos), ptr(self.tris), ptr(self.tri_area), nt,
                                    ptr(self.bounds), C.byref(kp), int(kd_device), C.byref(h), None))
        self.kd_build_ms = (time.perf_counter() - t0) * 1e3
        try:
            d = N.KdDesc()
            L.bt_kd_view(h, C.byref(d))
            nn, nr = d.num_nodes, d.num_refs

            def take(p, dtype, n):
                return np.ctypeslib.as_array(C.cast(p, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))),
                                             shape=(n,)).copy() if n else np.zeros(0, dtype)

            self.kd_split = take(d.split, np.float32, nn)
            self.kd_data = take(d.data, np.uint32, nn)
            self.kd_offset = take(d.offset, np.uint32, nn)
            self.kd_parent = take(d.parent, np.uint32, nn)
            self.kd_box = take(d.node_box, np.float32, 6 * nn).reshape(nn, 6)
            self.kd_tri_indices = take(d.tri_indices, np.uint32, nr)
            self.kd_bounds = np.array(list(d.bounds), np.float32)
            nl, md = C.c_int32(), C.c_int32()
            L.bt_kd_sizes(h, None, None, C.byref(nl), C.byref(md))
            self.kd_leaves, self.kd_max_depth = nl.value, md.value
        finally:
            L.bt_kd_free(h)

    # the arrays that make up a prepared scene (saved and restored by the
    # resident-scene cache, beamtrace2007_b200.ingest.SceneCache)
    ARRAYS = ("pos", "tris", "tri_normals", "tri_area", "bounds", "kd_split", "kd_data", "kd_offset", "kd_parent",
              "kd_box", "kd_tri_indices", "kd_bounds")

    def to_arrays(self) -> dict:
        d = {k: getattr(self, k) for k in self.ARRAYS}
        d["kd_sizes"] = np.array([self.kd_leaves, self.kd_max_depth], np.int64)
        return d

    @classmethod
    def from_arrays(cls, d) -> "PreparedScene":
        """A scene prepared earlier (to_arrays), without finalising or
        building again."""
        ps = cls.__new__(cls)
        dtypes = dict(pos=np.float32, tris=np.uint32, tri_normals=np.float32, tri_area=np.float32,
                      bounds=np.float32, kd_split=np.float32, kd_data=np.uint32, kd_offset=np.uint32,
                      kd_parent=np.uint32, kd_box=np.float32, kd_tri_indices=np.uint32, kd_bounds=np.float32)
        for k in cls.ARRAYS:
            setattr(ps, k, np.ascontiguousarray(d[k], dtypes[k]))
        n = len(ps.kd_split)
        if not (len(ps.kd_data) == len(ps.kd_offset) == len(ps.kd_parent) == len(ps.kd_box) == n
                and ps.tris.ndim == 2 and len(ps.tri_normals) == len(ps.tris) == len(ps.tri_area)):
            raise ValueError("inconsistent prepared-scene arrays")
        ps.kd_leaves, ps.kd_max_depth = (int(x) for x in d["kd_sizes"])
        ps.kd_build_ms = 0.0
        return ps

    @property
    def num_tris(self) -> int:
        return len(self.tris)

    def descs(self):
        sd = N.SceneDesc(ptr(self.pos), len(self.pos), ptr(self.tris), ptr(self.tri_normals), len(self.tris),
                         (C.c_float * 6)(*self.bounds))
        kd = N.KdDesc(ptr(self.kd_split), ptr(self.kd_data), ptr(self.kd_offset), ptr(self.kd_parent),
                      ptr(self.kd_box), len(self.kd_split), ptr(self.kd_tri_indices), len(self.kd_tri_indices),
                      (C.c_float * 6)(*self.kd_bounds))
        return sd, kd

    @property
    def offset(self) -> float:
        """Apex offset length(bounds.diag()) * kEpsRel in float32 (render.cpp:348)."""
        d = (self.bounds[3:] - self.bounds[:3]).astype(np.float32)
        l = np.sqrt(np.float32(np.float32(d[0] * d[0] + d[1] * d[1]) + np.float32(d[2] * d[2])), dtype=np.float32)
        return float(np.float32(l * np.float32(2e-5)))


@dataclass
class SoftResult:
    tri: np.ndarray
    vis: np.ndarray
    E: np.ndarray
    Eu: np.ndarray
    info: dict = field(default_factory=dict)


def gpu_available() -> dict | None:
    info = N.GpuInfo()
    if N.lib().bt_gpu_available(C.byref(info)) != N.BT_OK:
        return None
    return dict(name=info.name.decode(), sm_count=info.sm_count, mem_gb=info.mem_gb,
                cc=(info.cc_major, info.cc_minor))


class GpuRenderer:
    """bt::GpuRenderer over the C-ABI: the scene and its kd-tree are resident
    on one GPU for the renderer's lifetime."""

    def __init__(self, scene: PreparedScene, device: int = 0, budget: int = 2048, primary_budget: int = 4096,
                 capacity: int = 0, blocks_per_sm: int = 0, kernel_timing: bool = False,
                 tail_records: int = 0, eps_stats: bool = False, yield_pct: int = 0, fuse_primary: bool = False,
                 eps_fp64: bool = False, graph_rounds: bool = True, trace_ctas: int = 0):
        self.scene = scene
        cfg = N.GpuConfig()
        N.lib().bt_gpu_config_default(C.byref(cfg))
        cfg.device = device
        cfg.budget = budget
        cfg.primary_budget = primary_budget
        cfg.capacity = capacity
        cfg.blocks_per_sm = blocks_per_sm
        cfg.kernel_timing = int(kernel_timing)
        cfg.tail_records = int(tail_records)
        cfg.eps_stats = int(eps_stats)
        cfg.yield_pct = int(yield_pct)
        cfg.fuse_primary = int(fuse_primary)
        cfg.eps_fp64 = int(eps_fp64)
        cfg.graph_rounds = int(graph_rounds)
        cfg.trace_ctas = int(trace_ctas)
        self.config = cfg
        sd, kd = scene.descs()
        h = C.c_void_p()
        check(N.lib().bt_gpu_create(C.byref(sd), C.byref(kd), C.byref(cfg), C.byref(h)))
        self._h = h
        self.last_info: dict = {}
        self.last_rounds = 0
        self.last_max_queue = 0
        self.last_overflow_pixels = 0
        self.last_kernel_seconds = 0.0

    def close(self):
        if getattr(self, "_h", None):
            N.lib().bt_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _record(self, info: N.RunInfo):
        d = info.as_dict()
        self.last_info = d
        self.last_rounds = d["launches"]
        self.last_max_queue = d["max_spill"]
        self.last_overflow_pixels = d["retried_roots"]
        self.last_kernel_seconds = d["ms_trace"] * 1e-3
        return d

    # ---- soft shadows
    def soft_shadows(self, cam: N.Camera, light, exact: bool = False, offset: float = 0.0) -> SoftResult:
        n = cam.W * cam.H
        tri = np.zeros(n, np.int32)
        vis, E, Eu = (np.zeros(n, np.float32) for _ in range(3))
        L = light if isinstance(light, N.AreaLight) else N.AreaLight.from_array(light)
        o = N.SoftOpts(int(exact), float(offset))
        info = N.RunInfo()
        check(N.lib().bt_gpu_soft(self._h, C.byref(cam), C.byref(L), C.byref(o), ptr(tri), ptr(vis), ptr(E),
                                  ptr(Eu), C.byref(info)))
        return SoftResult(tri, vis, E, Eu, self._record(info))

    def add_scene(self, scene: "PreparedScene") -> int:
        """Adds a scene to this context's pool (bt_gpu_add_scene); returns its id."""
        sd, kd = scene.descs()
        sid = C.c_int32()
        check(N.lib().bt_gpu_add_scene(self._h, C.byref(sd), C.byref(kd), C.byref(sid)))
        self._pool = getattr(self, "_pool", [self.scene]) + [scene]
        return sid.value

    def batch_soft(self, cams, lights, exact: bool = True, offset: float = 0.0, device_outputs: bool = False,
                   scenes=None):
        """Soft shadows of several images in one engine run
        (bt_gpu_batch_soft); `scenes` gives each job's scene id in this
        context's pool (default: all the context's own scene, id 0).
        Returns one SoftResult per job (host arrays), or, with
        device_outputs, (tri, vis, E, Eu) CUDA tensors per job and the run
        info."""
        import torch
        dev = torch.device("cuda", self.config.device)
        jobs = (N.SoftJob * max(len(cams), 1))()
        outs = []
        for j, (cam, light) in enumerate(zip(cams, lights)):
            n = cam.W * cam.H
            t = (torch.empty(n, dtype=torch.int32, device=dev),) + tuple(
                torch.empty(n, dtype=torch.float32, device=dev) for _ in range(3))
            outs.append(t)
            L = light if isinstance(light, N.AreaLight) else N.AreaLight.from_array(light)
            jobs[j] = N.SoftJob(cam, L, N.SoftOpts(int(exact), float(offset)), t[0].data_ptr(), t[1].data_ptr(),
                                t[2].data_ptr(), t[3].data_ptr(), int(scenes[j]) if scenes is not None else 0)
        info = N.RunInfo()
        # (the engine runs on its own stream and returns when its outputs
        # are written; nothing of torch's writes to these buffers)
        check(N.lib().bt_gpu_batch_soft(self._h, len(cams), jobs, C.byref(info)))
        rec = self._record(info)
        if device_outputs:
            return outs, rec
        return [SoftResult(*(x.cpu().numpy() for x in t), info=rec) for t in outs]

    def soft_points(self, light, tri, X, N_, exact: bool = False, offset: float = 0.0) -> SoftResult:
        tri = np.ascontiguousarray(tri, np.int32)
        X = np.ascontiguousarray(X, np.float32).reshape(-1, 3)
        N_ = np.ascontiguousarray(N_, np.float32).reshape(-1, 3)
        n = len(tri)
        vis, E, Eu = (np.zeros(max(n, 1), np.float32) for _ in range(3))
        L = light if isinstance(light, N.AreaLight) else N.AreaLight.from_array(light)
        o = N.SoftOpts(int(exact), float(offset))
        info = N.RunInfo()
        check(N.lib().bt_gpu_soft_points(self._h, C.byref(L), C.byref(o), n, ptr(tri), ptr(X), ptr(N_), ptr(vis),
                                         ptr(E), ptr(Eu), C.byref(info)))
        return SoftResult(tri, vis[:n], E[:n], Eu[:n], self._record(info))

    # ---- primary visibility and point shadows
    def _fetch_rest(self, out: PolyList, n: int) -> PolyList:
        """The last call produced n > len(out) polygons: fetch them all again
        from the device (bt_gpu_last_polys) instead of repeating the call."""
        if n <= len(out):
            return out.head(n)
        out = PolyList.alloc(n)
        s = out.struct()
        cnt = C.c_int64()
        check(N.lib().bt_gpu_last_polys(self._h, C.byref(s), C.byref(cnt)))
        return out.head(cnt.value)

    def primary(self, cam: N.Camera, cull: bool = False, tile: int = 16, cap: int = 0) -> PolyList:
        cap = cap or max(1 << 16, 2 * cam.W * cam.H)
        out = PolyList.alloc(cap)
        s = out.struct()
        cnt = C.c_int64()
        info = N.RunInfo()
        check(N.lib().bt_gpu_primary(self._h, C.byref(cam), int(cull), int(tile), C.byref(s), C.byref(cnt),
                                     C.byref(info)))
        self._record(info)
        return self._fetch_rest(out, cnt.value)

    def point_shadows(self, cam: N.Camera, hits: PolyList, light, cap: int = 0) -> PolyList:
        light = np.asarray(light, np.float32)
        cap = cap or max(1 << 16, 4 * len(hits))
        hs = hits.struct()
        out = PolyList.alloc(cap)
        s = out.struct()
        cnt = C.c_int64()
        info = N.RunInfo()
        check(N.lib().bt_gpu_point(self._h, C.byref(cam), C.byref(hs), len(hits), ptr(light), C.byref(s),
                                   C.byref(cnt), C.byref(info)))
        self._record(info)
        return self._fetch_rest(out, cnt.value)

    def primary_ids(self, cam: N.Camera, cull: bool = False, tile: int = 16) -> np.ndarray:
        """Per-pixel hit-triangle ids, polygons kept on the GPU (bt_gpu_primary_ids)."""
        tri = np.zeros(cam.W * cam.H, np.int32)
        info = N.RunInfo()
        check(N.lib().bt_gpu_primary_ids(self._h, C.byref(cam), int(cull), int(tile), ptr(tri), C.byref(info)))
        self._record(info)
        return tri.reshape(cam.H, cam.W)

    def point_mask(self, cam: N.Camera, light, cull: bool = False, tile: int = 16):
        """(ids, shadow mask) of a point light, all on the GPU (bt_gpu_point_mask)."""
        light = np.ascontiguousarray(light, np.float32)
        tri = np.zeros(cam.W * cam.H, np.int32)
        mask = np.zeros(cam.W * cam.H, np.uint8)
        info = N.RunInfo()
        check(N.lib().bt_gpu_point_mask(self._h, C.byref(cam), int(cull), int(tile), ptr(light), ptr(tri), ptr(mask),
                                        C.byref(info)))
        self._record(info)
        return tri.reshape(cam.H, cam.W), mask.reshape(cam.H, cam.W)

    def raster(self, cam: N.Camera, prim: PolyList, shadow: PolyList | None = None):
        tri = np.zeros(cam.W * cam.H, np.int32)
        flag = np.zeros(cam.W * cam.H, np.uint8)
        ps = prim.struct()
        ss = shadow.struct() if shadow is not None and len(shadow) else None
        check(N.lib().bt_gpu_raster(self._h, C.byref(cam), C.byref(ps), len(prim),
                                    C.byref(ss) if ss is not None else None, len(shadow) if ss is not None else 0,
                                    ptr(tri), ptr(flag)))
        return tri.reshape(cam.H, cam.W), flag.reshape(cam.H, cam.W)

"""Scene ingest: the reference's scene configs, OBJ/PLY meshes and
procedural scenes, and a resident-scene cache for the server.

``load_config(path)`` / ``parse_config(text)`` run the native ingest
(``bt_scene_load_config`` / ``bt_scene_parse_config``), which builds the
scene the reference builds from the same config (loadConfig / parseConfig +
buildScene, src/scene/scene.cpp:127-262, with the loaders of
src/scene/loaders.cpp and the scenes of src/scene/procedural.cpp), float
for float.  The result is a ``SceneFile``: a ``SceneData`` (positions,
triangles, up, views, lights) plus the config's materials, culling,
intensity and background.

``SceneCache`` keeps prepared scenes (finalised triangles and the SAH
kd-tree, the work that gates admitting a scene: about 9 s for 2.1M
triangles on the host, 0.7 s with the GPU build) on disk, keyed by the config text, the bytes of every
mesh file it names and the library's kd-tree parameters, and in memory, so
that a scene ingested once is admitted again by reading its arrays back.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .scenes import SceneData, View

# bumped when the cached arrays' layout or the ingest's output changes
CACHE_FORMAT = 1


@dataclass
class SceneFile(SceneData):
    tri_mat: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint16))    # material per triangle
    mat_color: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))  # albedo per material
    cull_backfaces: bool = False
    light_intensity: float = 1.0
    background: tuple = (0.0, 0.0, 0.0)
    path: str = ""


def _tuple(a) -> tuple:
    return tuple(float(x) for x in a)


def _read(handle, path: str) -> SceneFile:
    L = N.lib()
    info = N.SceneFileInfo()
    L.bt_scene_file_info_get(handle, C.byref(info))
    pos = np.zeros((info.num_verts, 3), np.float32)
    tris = np.zeros((info.num_tris, 3), np.uint32)
    mat = np.zeros(info.num_tris, np.uint16)
    color = np.zeros((info.num_materials, 3), np.float32)
    views = np.zeros((info.num_views, 7), np.float32)
    L.bt_scene_file_arrays(handle, N.ptr(pos), N.ptr(tris), N.ptr(mat), N.ptr(color), N.ptr(views))
    return SceneFile(
        name=info.name.decode(errors="replace"), pos=pos, tris=tris, up=_tuple(info.up),
        views=[View(_tuple(v[:3]), _tuple(v[3:6]), float(v[6])) for v in views],
        point_light=_tuple(info.point_light) if info.has_point_light else None,
        area_light=(_tuple(info.light_c), _tuple(info.light_u), _tuple(info.light_v)) if info.has_area_light else None,
        tri_mat=mat, mat_color=color, cull_backfaces=bool(info.cull_backfaces),
        light_intensity=float(info.light_intensity), background=_tuple(info.background), path=path)


def _ingest(fn, arg: bytes, path: str) -> SceneFile:
    L = N.lib()
    h = C.c_void_p()
    N.check(fn(arg, C.byref(h)))
    try:
        return _read(h, path)
    finally:
        L.bt_scene_file_free(h)


def load_config(path: str) -> SceneFile:
    """loadConfig + buildScene: the scene of a config file."""
    return _ingest(N.lib().bt_scene_load_config, os.fsencode(path), path)


def parse_config(text: str) -> SceneFile:
    """parseConfig + buildScene on config text (mesh paths as written)."""
    return _ingest(N.lib().bt_scene_parse_config, text.encode(), "")


def mesh_files(text: str) -> list[str]:
    """The obj/ply files a config names, in order (the `mesh` lines)."""
    out = []
    for line in text.splitlines():
        line = line.split("#", 1)[0]
        t = line.split()
        if len(t) >= 3 and t[0] == "mesh" and t[1] in ("obj", "ply"):
            out.append(t[2])
    return out


class SceneCache:
    """Prepared scenes by config: ``get(path)`` returns (SceneFile,
    PreparedScene), from memory, else from `directory` (when given), else by
    ingesting and preparing the scene (and storing it).  With `kd_device`
    the kd-tree of a scene prepared here is built on that CUDA device
    (bt_kd_build_gpu; the same tree, so the same cache entry)."""

    def __init__(self, directory: str | None = None, kd_device: int | None = None):
        self.directory = directory
        self.kd_device = kd_device
        self._mem: dict = {}
        self._lock = threading.Lock()
        self.hits = self.disk_hits = self.misses = 0

    @staticmethod
    def key(path: str) -> str:
        from .renderer import kd_params_default
        h = hashlib.sha256()
        h.update(f"bt-scene-cache {CACHE_FORMAT}\n".encode())
        h.update(json.dumps(kd_params_default(), sort_keys=True).encode())
        with open(path, "rb") as f:
            text = f.read()
        h.update(text)
        for m in mesh_files(text.decode(errors="replace")):
            h.update(b"\0mesh\0" + m.encode() + b"\0")
            try:
                with open(m, "rb") as f:
                    for chunk in iter(lambda: f.read(1 << 24), b""):
                        h.update(chunk)
            except OSError:
                h.update(b"<missing>")  # the ingest reports it
        return h.hexdigest()

    def _file(self, key: str) -> str:
        return os.path.join(self.directory, key + ".npz")

    def get(self, path: str):
        from .renderer import PreparedScene
        key = self.key(path)
        with self._lock:
            if key in self._mem:
                self.hits += 1
                return self._mem[key]
        got = self._load(key, path) if self.directory else None
        if got is not None:
            self.disk_hits += 1
        else:
            self.misses += 1
            sf = load_config(path)
            got = (sf, PreparedScene(sf.pos, sf.tris, kd_device=self.kd_device))
            if self.directory:
                self._store(key, *got)
        with self._lock:
            self._mem[key] = got
        return got

    def _store(self, key: str, sf: SceneFile, ps) -> None:
        os.makedirs(self.directory, exist_ok=True)
        meta = dict(name=sf.name, up=sf.up, views=[[*v.eye, *v.target, v.fov] for v in sf.views],
                    point_light=sf.point_light, area_light=sf.area_light, cull_backfaces=sf.cull_backfaces,
                    light_intensity=sf.light_intensity, background=sf.background, path=sf.path)
        arrays = ps.to_arrays()
        arrays.update(scene_pos=sf.pos, scene_tris=sf.tris, tri_mat=sf.tri_mat, mat_color=sf.mat_color,
                      meta=np.array(json.dumps(meta)))
        tmp = self._file(key) + f".{os.getpid()}.{threading.get_ident()}.tmp"
        with open(tmp, "wb") as f:
            np.savez(f, **arrays)
        os.replace(tmp, self._file(key))

    def _load(self, key: str, path: str):
        from .renderer import PreparedScene
        fn = self._file(key)
        if not os.path.exists(fn):
            return None
        try:
            with np.load(fn, allow_pickle=False) as z:
                d = {k: z[k] for k in z.files}
            meta = json.loads(str(d["meta"]))
            ps = PreparedScene.from_arrays(d)
        except (OSError, ValueError, KeyError):
            return None  # a damaged entry is rebuilt
        views = [View(tuple(v[:3]), tuple(v[3:6]), float(v[6])) for v in meta["views"]]
        sf = SceneFile(name=meta["name"], pos=d["scene_pos"], tris=d["scene_tris"], up=tuple(meta["up"]),
                       views=views,
                       point_light=tuple(meta["point_light"]) if meta["point_light"] is not None else None,
                       area_light=tuple(tuple(x) for x in meta["area_light"]) if meta["area_light"] else None,
                       tri_mat=d["tri_mat"], mat_color=d["mat_color"], cull_backfaces=bool(meta["cull_backfaces"]),
                       light_intensity=float(meta["light_intensity"]), background=tuple(meta["background"]),
                       path=path)
        return sf, ps

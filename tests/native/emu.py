"""ctypes wrapper of the host emulator (test infrastructure only)."""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import build_emu  # noqa: E402

from beamtrace2007_b200 import _native as N  # noqa: E402
from beamtrace2007_b200.renderer import PolyList  # noqa: E402

_P = C.c_void_p


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Emulator:
    def __init__(self, prepared):
        self.lib = C.CDLL(build_emu.build())
        self.lib.emu_create.restype = _P
        self.lib.emu_create.argtypes = [C.POINTER(N.SceneDesc), C.POINTER(N.KdDesc)]
        self.lib.emu_primary_tiles.restype = C.c_int64
        self.lib.emu_point.restype = C.c_int64
        self.prepared = prepared
        sd, kd = prepared.descs()
        self.h = self.lib.emu_create(C.byref(sd), C.byref(kd))

    def __del__(self):
        try:
            self.lib.emu_destroy(_P(self.h))
        except Exception:
            pass

    def soft_points(self, light, offset, tri, X, N_, exact=False):
        tri = np.ascontiguousarray(tri, np.int32)
        X = np.ascontiguousarray(X, np.float32)
        N_ = np.ascontiguousarray(N_, np.float32)
        light = np.ascontiguousarray(light, np.float32)
        n = len(tri)
        vis, G = np.zeros(n), np.zeros(n)
        st = np.zeros(11, np.uint64)
        self.lib.emu_soft_points(_P(self.h), _p(light), C.c_float(offset), C.c_int64(n), _p(tri), _p(X), _p(N_),
                                 int(exact), _p(vis), _p(G), _p(st))
        return vis, G, st

    def primary_tiles(self, cam, cull=False, tile=16, cap=1 << 20):
        p = PolyList.alloc(cap)
        st = np.zeros(11, np.uint64)
        k = self.lib.emu_primary_tiles(_P(self.h), C.byref(cam), int(cull), int(tile), C.c_int64(cap), _p(p.x),
                                       _p(p.y), _p(p.n), _p(p.tri), _p(p.area), _p(p.root), _p(st))
        assert k <= cap
        return p.head(k), st

    def point(self, cam, light, hits, cap=1 << 20):
        p = PolyList.alloc(cap)
        st = np.zeros(11, np.uint64)
        light = np.ascontiguousarray(light, np.float32)
        k = self.lib.emu_point(_P(self.h), C.byref(cam), _p(light), C.c_int64(len(hits)),
                               _p(np.ascontiguousarray(hits.x, np.float32)), _p(np.ascontiguousarray(hits.y, np.float32)),
                               _p(np.ascontiguousarray(hits.n, np.int32)), _p(np.ascontiguousarray(hits.tri, np.int32)),
                               C.c_int64(cap), _p(p.x), _p(p.y), _p(p.n), _p(p.tri), _p(p.area), _p(p.root), _p(st))
        assert k <= cap
        return p.head(k), st

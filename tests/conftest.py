"""Shared fixtures.  CPU tests check the oracle, the host code and the
emulated per-lane engine against the reference; `-m gpu` tests check the
CUDA engine through the C-ABI."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests", "native"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def native_lib():
    from beamtrace2007_b200 import build
    build.build()
    from beamtrace2007_b200 import _native
    return _native.lib()


@pytest.fixture(scope="session")
def oracle_ready():
    """The reference compiled from its sources (oracle/_ref); built here when
    the sources are present, prebuilt libraries are used elsewhere."""
    from ref import ref_available
    if not (ref_available("f") and ref_available("d")):
        # builds the reference where its sources are present (the Makefile's
        # `all` is empty elsewhere)
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8", "all"], capture_output=True)
    if not (ref_available("f") and ref_available("d")):
        pytest.skip("oracle/_ref not built")
    return True


@pytest.fixture(scope="session")
def gpu(native_lib):
    from beamtrace2007_b200.renderer import gpu_available
    info = gpu_available()
    if info is None:
        pytest.skip("no CUDA device")
    return info


_SCENES = {}


def scene(name, **kw):
    from beamtrace2007_b200 import scenes
    from beamtrace2007_b200.renderer import PreparedScene
    key = (name, tuple(sorted(kw.items())))
    if key not in _SCENES:
        s = scenes.SCENES[name](**kw) if name in scenes.SCENES else getattr(scenes, name)(**kw)
        _SCENES[key] = (s, PreparedScene(s.pos, s.tris))
    return _SCENES[key]


def piece_keys(p, with_area=False):
    """Order-free identity of a piece list: (root, n, tri, corner bits)."""
    x = np.ascontiguousarray(p.x, np.float32).view(np.uint32)
    y = np.ascontiguousarray(p.y, np.float32).view(np.uint32)
    cols = [np.asarray(p.root, np.int64), np.asarray(p.n, np.int64), np.asarray(p.tri, np.int64)]
    rows = np.concatenate([np.stack(cols, 1), x.astype(np.int64), y.astype(np.int64)], 1)
    if with_area:
        rows = np.concatenate([rows, np.ascontiguousarray(p.area, np.float32).view(np.uint32).astype(np.int64)[:, None]], 1)
    order = np.lexsort(rows.T[::-1])
    return rows[order]


def to_f32(p):
    from beamtrace2007_b200.renderer import PolyList
    return PolyList(np.ascontiguousarray(p.x, np.float32), np.ascontiguousarray(p.y, np.float32),
                    np.asarray(p.n, np.int32), np.asarray(p.tri, np.int32), np.ascontiguousarray(p.area, np.float32),
                    np.asarray(p.root, np.int32))

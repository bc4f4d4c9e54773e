"""The clip's polygon steps -- fuzzy split by a line, then clean-up -- as
this package compiles them (beam_math.cuh, built for the host by
tests/native/emu.cpp), against the reference's own splitPoly/cleanPoly
(src/beam/beam_geom.h:83-150, its float build) on 20,000 random convex
triangles and quads over six orders of magnitude, with lines through
vertices, inside and just outside the fuzzy band, and anywhere: bitwise the
same pieces.  And the reference's own invariants of the split
(tests/test_geometry.cpp:54-110): the pieces stay convex, their areas add
up to the polygon's, and splitting by L and by -L gives the same two pieces
the other way round, bit for bit (neighbouring beams agree on their shared
edge)."""
import ctypes as C

import numpy as np
import pytest

CASES = 20_000


def _emu():
    import build_emu
    lib = C.CDLL(build_emu.build())
    f = C.POINTER(C.c_float)
    i = C.POINTER(C.c_int)
    lib.emu_split_clean.restype = C.c_int
    lib.emu_split_clean.argtypes = [f, f, C.c_int, f, C.c_float, f, f, i, f, f, i]
    lib.emu_poly_area.restype = C.c_float
    lib.emu_poly_area.argtypes = [f, f, C.c_int]
    return lib


def _cases(seed=5):
    rng = np.random.default_rng(seed)
    for _ in range(CASES):
        n = int(rng.integers(3, 5))
        ext = np.float32(10.0 ** rng.uniform(-3, 3))
        ang = np.sort(rng.uniform(0, 2 * np.pi, n))
        r = ext * rng.uniform(0.5, 1.0)
        cx, cy = rng.uniform(-2, 2, 2) * ext
        px = (cx + r * np.cos(ang)).astype(np.float32)
        py = (cy + r * np.sin(ang)).astype(np.float32)
        t = rng.uniform(0, 2 * np.pi)
        a, b = np.float32(np.cos(t)), np.float32(np.sin(t))
        eps = np.float32(ext * np.float32(2e-5))
        k = int(rng.integers(n))
        mode = int(rng.integers(5))
        off = [0.0, 0.5 * eps, -0.5 * eps, 2.0 * eps, float(rng.uniform(-1, 1) * ext)][mode]
        c = np.float32(-(a * px[k] + b * py[k]) + off)
        yield px, py, np.array([a, b, c], np.float32), eps


def _ours(lib, px, py, line, eps):
    f = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    bufs = [np.zeros(8, np.float32) for _ in range(4)]
    ni, no = C.c_int(0), C.c_int(0)
    ok = lib.emu_split_clean(f(px), f(py), len(px), f(line), C.c_float(eps), f(bufs[0]), f(bufs[1]), C.byref(ni),
                             f(bufs[2]), f(bufs[3]), C.byref(no))
    return ok, (bufs[0][:ni.value], bufs[1][:ni.value]), (bufs[2][:no.value], bufs[3][:no.value])


def _ref(lib, px, py, line, eps):
    d = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    bufs = [np.zeros(8) for _ in range(4)]
    ni, no = C.c_int(0), C.c_int(0)
    ok = lib.btr_split_clean(d(px.astype(np.float64)), d(py.astype(np.float64)), len(px),
                             d(line.astype(np.float64)), C.c_double(float(eps)), d(bufs[0]), d(bufs[1]),
                             C.byref(ni), d(bufs[2]), d(bufs[3]), C.byref(no))
    return ok, (bufs[0][:ni.value], bufs[1][:ni.value]), (bufs[2][:no.value], bufs[3][:no.value])


def _same(a, b):
    return len(a[0]) == len(b[0]) and np.array_equal(np.asarray(a[0], np.float32), np.asarray(b[0], np.float32)) \
        and np.array_equal(np.asarray(a[1], np.float32), np.asarray(b[1], np.float32))


def test_split_and_clean_match_the_reference_bitwise(oracle_ready):
    from ref import _lib
    ref = _lib("f")
    ref.btr_split_clean.restype = C.c_int
    emu = _emu()
    splits = 0
    for px, py, line, eps in _cases():
        ok1, in1, out1 = _ours(emu, px, py, line, eps)
        ok2, in2, out2 = _ref(ref, px, py, line, eps)
        assert ok1 == ok2 == 1
        assert _same(in1, in2) and _same(out1, out2), (px, py, line, eps)
        splits += len(in1[0]) >= 3 and len(out1[0]) >= 3
    assert splits > CASES // 10  # the lines do cut many polygons


def test_split_invariants():
    emu = _emu()
    f = lambda a: np.ascontiguousarray(a, np.float32).ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    for px, py, line, eps in _cases(seed=9):
        ok, pin, pout = _ours(emu, px, py, line, eps)
        assert ok == 1
        okn, nin, nout = _ours(emu, px, py, -line, eps)
        assert okn == 1
        # L and -L: the same pieces, exchanged
        assert _same(pin, nout) and _same(pout, nin)
        # the pieces stay convex: no turn against the polygon's orientation
        # beyond rounding (cleanPoly has welded near-collinear corners)
        for x, y in (pin, pout):
            if len(x) >= 3:
                xd, yd = np.asarray(x, np.float64), np.asarray(y, np.float64)
                ex, ey = np.roll(xd, -1) - xd, np.roll(yd, -1) - yd
                turn = ex * np.roll(ey, -1) - ey * np.roll(ex, -1)
                scale = float(np.max(np.hypot(ex, ey))) ** 2
                assert np.all(turn >= -1e-5 * scale), turn
        # the areas add up (the pieces share the crossing points)
        A = float(emu.emu_poly_area(f(px), f(py), len(px)))
        parts = sum(float(emu.emu_poly_area(f(x), f(y), len(x))) for x, y in (pin, pout) if len(x) >= 3)
        ext = float(max(np.ptp(px), np.ptp(py)))
        assert abs(parts - A) <= 1e-4 * abs(A) + 4 * float(eps) * ext

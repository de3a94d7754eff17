"""The pure-Python hull builder (bounce_b200/hull.py) against the native one
(b3g_hull_from_points / b3g_hull_box in the library): the same arrays bit for
bit, so a process that builds its scene without the library (the reference
arm of the benchmark) collides the same hulls as the device arm."""
import ctypes

import numpy as np

from bounce_b200 import _native as N
from bounce_b200 import hull as H
from bounce_b200 import scene as S


def _native_hull(lib, pts):
    pts = np.ascontiguousarray(pts, np.float32)
    n = len(pts)
    v = np.zeros(3 * n, np.float32)
    e = np.zeros(30 * n, np.uint32)
    f = np.zeros(2 * n, np.uint32)
    p = np.zeros(8 * n, np.float32)
    c = np.zeros(3, np.float32)
    cnt = np.zeros(3, np.uint32)
    rc = lib.b3g_hull_from_points(N.ptr(pts, ctypes.c_float), n, N.ptr(v, ctypes.c_float), N.ptr(e, ctypes.c_uint32),
                                  N.ptr(f, ctypes.c_uint32), N.ptr(p, ctypes.c_float), N.ptr(c, ctypes.c_float),
                                  N.ptr(cnt, ctypes.c_uint32))
    if rc:
        return None
    nv, ne, nf = (int(x) for x in cnt)
    return v[:3 * nv], e[:5 * ne], f[:nf], p[:4 * nf], c, (nv, ne, nf)


def test_points_match_native():
    lib = N.load()
    rng = np.random.default_rng(12)
    built = 0
    for k in range(600):
        m = int(rng.integers(4, 65))
        pts = S.ellipsoid_points(rng, m, rng.uniform(0.3, 1.2, 3))
        if k % 5 == 0:
            pts = (np.round(pts * 4) / 4).astype(np.float32)  # repeated and coplanar points
        if k % 97 == 0:
            pts[:, 2] = 0.25  # all coplanar: rejected by both
        a = _native_hull(lib, pts)
        try:
            b = H.hull_from_points(pts)
        except ValueError:
            b = None
        assert (a is None) == (b is None), k
        if a is None:
            continue
        built += 1
        assert a[5] == b[5], k
        for x, y in zip(a[:5], b[:5]):
            assert x.dtype == y.dtype and np.array_equal(x, y), k
    assert built > 500


def test_box_matches_native():
    lib = N.load()
    for ext in [(0.5, 0.5, 0.5), (50.0, 0.5, 50.0), (0.1, 2.0, 0.7)]:
        v = np.zeros(24, np.float32)
        e = np.zeros(120, np.uint32)
        f = np.zeros(6, np.uint32)
        p = np.zeros(24, np.float32)
        c = np.zeros(3, np.float32)
        cnt = np.zeros(3, np.uint32)
        lib.b3g_hull_box(np.float32(ext[0]), np.float32(ext[1]), np.float32(ext[2]), N.ptr(v, ctypes.c_float),
                         N.ptr(e, ctypes.c_uint32), N.ptr(f, ctypes.c_uint32), N.ptr(p, ctypes.c_float),
                         N.ptr(c, ctypes.c_float), N.ptr(cnt, ctypes.c_uint32))
        hv, he, hf, hp, hc, counts = H.hull_box(*ext)
        assert counts == tuple(int(x) for x in cnt)
        for x, y in [(v, hv), (e, he), (f, hf), (p, hp), (c, hc)]:
            assert np.array_equal(x, y)


def test_scene_same_with_either_builder():
    a = S.mixed_scene(seed=21, n=400, side=8.0).finalize()
    S.NATIVE_HULLS = False
    try:
        b = S.mixed_scene(seed=21, n=400, side=8.0).finalize()
    finally:
        S.NATIVE_HULLS = True
    for k in a.hull_arrays:
        assert np.array_equal(a.hull_arrays[k], b.hull_arrays[k]), k
    assert np.array_equal(a.local_center, b.local_center)

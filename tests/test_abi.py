"""CPU checks of the boundary: the C-ABI library loads and exports every entry
point the headers declare, and its manifold record is the reference's
b3Manifold layout."""
import ctypes
import os
import re

import numpy as np

from bounce_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("b3g.h", "b3g_hull.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(b3g_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_entry_point():
    lib = N.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"
    assert set(N.EXPORTED) == names


def test_manifold_layout_matches_reference(oracle_mod):
    L = oracle_mod.lib(32)
    L.ref_manifold_layout.argtypes = [ctypes.POINTER(ctypes.c_uint32)]
    o = np.zeros(16, np.uint32)
    L.ref_manifold_layout(o.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    p, m = N.POINT_DTYPE, N.MANIFOLD_DTYPE
    assert o[0] == p.itemsize and o[9] == m.itemsize
    assert list(o[1:9]) == [p.fields[k][1] for k in ("n", "p1", "p2", "normalImpulse", "triangleKey", "key",
                                                      "persisting", "edgeContact")]
    assert list(o[10:16]) == [m.fields[k][1] for k in ("pointCount", "tangentImpulse", "motorImpulse", "motorSpeed",
                                                       "tangentSpeed1", "tangentSpeed2")]


def test_invalid_arguments_are_rejected_without_gpu_work():
    lib = N.load()
    # Null config: rejected before any CUDA call.
    assert lib.b3g_create(None, ctypes.byref(ctypes.c_void_p())) == N.B3G_E_INVALID
    assert lib.b3g_last_error(None) == b"null context"

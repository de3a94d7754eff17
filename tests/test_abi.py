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


# The records of include/b3g.h that cross the boundary, with the numpy dtypes
# the Python binding reads them with (C field name -> dtype field name).
STRUCTS = {
    "b3g_solver_body": ("SOLVER_BODY_DTYPE", {"x": "x", "q": "q", "v": "v", "w": "w", "inv_mass": "invMass",
                                              "local_center": "localCenter", "inv_i": "invI"}),
    "b3g_contact_constraint": ("CONTACT_CONSTRAINT_DTYPE", {
        "index_a": "indexA", "index_b": "indexB", "manifold_start": "manifoldStart",
        "manifold_count": "manifoldCount", "inv_mass_a": "invMassA", "inv_mass_b": "invMassB",
        "friction": "friction", "restitution": "restitution", "inv_i_a": "invIA", "inv_i_b": "invIB",
        "radius_a": "radiusA", "radius_b": "radiusB", "contact": "contact"}),
    "b3g_manifold_constraint": ("MANIFOLD_CONSTRAINT_DTYPE", {
        "r_a": "rA", "r_b": "rB", "normal": "normal", "tangent1": "tangent1", "tangent2": "tangent2",
        "tangent_speed1": "tangentSpeed1", "tangent_speed2": "tangentSpeed2", "tangent_mass": "tangentMass",
        "tangent_impulse": "tangentImpulse", "motor_impulse": "motorImpulse", "motor_mass": "motorMass",
        "motor_speed": "motorSpeed", "point_count": "pointCount", "constraint": "constraint",
        "points": "points", "position_points": "positionPoints"}),
    "b3g_shape_cast_input": ("SHAPE_CAST_DTYPE", {
        "shape_type": "type", "hull": "hull", "world": "world", "params": "params", "position": "position",
        "rotation": "rotation", "displacement": "displacement"}),
    "b3g_toi_input": ("TOI_INPUT_DTYPE", {
        "type_a": "type_a", "hull_a": "hull_a", "type_b": "type_b", "hull_b": "hull_b", "params_a": "params_a",
        "params_b": "params_b", "sweep_a": "sweep_a", "sweep_b": "sweep_b", "t_max": "t_max"}),
    "b3g_gjk_cast_input": ("GJK_CAST_DTYPE", {
        "type_a": "type_a", "hull_a": "hull_a", "type_b": "type_b", "hull_b": "hull_b", "params_a": "params_a",
        "params_b": "params_b", "xf_a": "xf_a", "xf_b": "xf_b", "translation_b": "translation_b"}),
}


def test_record_layouts_match_the_header(tmp_path):
    """Sizes and field offsets of the header's records, as the C compiler
    lays them out, equal the binding's numpy dtypes."""
    import subprocess

    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "b3g.h"', "int main(void) {"]
    for struct, (_, fields) in STRUCTS.items():
        lines.append(f'printf("{struct} size %zu\\n", sizeof({struct}));')
        for f in fields:
            lines.append(f'printf("{struct} {f} %zu\\n", offsetof({struct}, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        struct, field, value = line.split()
        got[(struct, field)] = int(value)
    for struct, (dtype_name, fields) in STRUCTS.items():
        dt = getattr(N, dtype_name)
        assert got[(struct, "size")] == dt.itemsize, struct
        for c_field, np_field in fields.items():
            assert got[(struct, c_field)] == dt.fields[np_field][1], (struct, c_field)

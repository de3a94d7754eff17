"""Loader for the in-tree CUDA library ``bounce_b200/libb3g.so`` (include/b3g.h).

The product path has no CPU fallback: if the library is missing or a call
fails, an exception is raised.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libb3g.so")

B3G_OK = 0
B3G_E_INVALID = -1
B3G_E_CAPACITY = -2
B3G_E_CUDA = -3
B3G_E_TIMEOUT = -4
B3G_E_STATE = -5

SHAPE_SPHERE, SHAPE_CAPSULE, SHAPE_TRIANGLE, SHAPE_HULL, SHAPE_MESH = 0, 1, 2, 3, 4
BODY_STATIC, BODY_KINEMATIC, BODY_DYNAMIC = 0, 1, 2
FLAG_WARM_STARTING = 1
FLAG_CONVEX_CACHE = 2
FLAG_GRAPH = 4
FLAG_CONTACT_FILTER = 8
TUNE_CONVEX, TUNE_PROBE, TUNE_SAT_WARPS, TUNE_SAT_BLOCKS, TUNE_TRAVERSE, TUNE_COUNT = 0, 9, 10, 11, 12, 13
FIXTURE_SENSOR = 1


class B3GError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"b3g error {code}: {msg}")
        self.code = code


class Config(ctypes.Structure):
    _fields_ = [
        ("max_proxies", ctypes.c_uint32),
        ("max_contacts", ctypes.c_uint32),
        ("max_hull_data", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("device", ctypes.c_int32),
    ]


class Counts(ctypes.Structure):
    _fields_ = [
        ("contacts", ctypes.c_uint32),
        ("begun", ctypes.c_uint32),
        ("ended", ctypes.c_uint32),
        ("touching", ctypes.c_uint32),
        ("manifolds", ctypes.c_uint32),
        ("points", ctypes.c_uint32),
        ("moved", ctypes.c_uint32),
        ("status", ctypes.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# b3ManifoldPoint / b3Manifold (include/bounce/collision/collision.h:97-128), 72 / 320 bytes.
POINT_DTYPE = np.dtype(
    [
        ("n", "<f4", 3),
        ("p1", "<f4", 3),
        ("p2", "<f4", 3),
        ("normalImpulse", "<f4"),
        ("triangleKey", "<u4"),
        ("pad0", "<u4"),
        ("key", "<u4", 4),
        ("persisting", "u1"),
        ("edgeContact", "u1"),
        ("pad1", "u1", 6),
    ]
)
MANIFOLD_DTYPE = np.dtype(
    [
        ("points", POINT_DTYPE, 4),
        ("pointCount", "<u4"),
        ("tangentImpulse", "<f4", 2),
        ("motorImpulse", "<f4"),
        ("motorSpeed", "<f4"),
        ("tangentSpeed1", "<f4"),
        ("tangentSpeed2", "<f4"),
        ("pad", "<u4"),
    ]
)
assert POINT_DTYPE.itemsize == 72 and MANIFOLD_DTYPE.itemsize == 320

# Solver input records (include/b3g.h): b3g_solver_body (b3Position /
# b3Velocity entries and body fields, island.cpp:130-134), b3g_contact_constraint
# (b3ContactVelocityConstraint, contact_solver.h:93-105) and
# b3g_manifold_constraint (b3VelocityConstraintManifold with its points and the
# b3PositionConstraintPoints, contact_solver.h:31-91).
SOLVER_BODY_DTYPE = np.dtype(
    [
        ("x", "<f4", 3),
        ("q", "<f4", 4),
        ("v", "<f4", 3),
        ("w", "<f4", 3),
        ("invMass", "<f4"),
        ("localCenter", "<f4", 3),
        ("invI", "<f4", 9),
        ("pad", "<f4", 2),
    ]
)
CONTACT_CONSTRAINT_DTYPE = np.dtype(
    [
        ("indexA", "<u4"),
        ("indexB", "<u4"),
        ("manifoldStart", "<u4"),
        ("manifoldCount", "<u4"),
        ("invMassA", "<f4"),
        ("invMassB", "<f4"),
        ("friction", "<f4"),
        ("restitution", "<f4"),
        ("invIA", "<f4", 9),
        ("invIB", "<f4", 9),
        ("radiusA", "<f4"),
        ("radiusB", "<f4"),
        ("contact", "<u4"),
        ("pad", "<u4", 3),
    ]
)
VELOCITY_POINT_DTYPE = np.dtype(
    [
        ("rA", "<f4", 3),
        ("rB", "<f4", 3),
        ("normal", "<f4", 3),
        ("normalMass", "<f4"),
        ("normalImpulse", "<f4"),
        ("velocityBias", "<f4"),
    ]
)
POSITION_POINT_DTYPE = np.dtype([("localNormalA", "<f4", 3), ("localPointA", "<f4", 3), ("localPointB", "<f4", 3)])
MANIFOLD_CONSTRAINT_DTYPE = np.dtype(
    [
        ("rA", "<f4", 3),
        ("rB", "<f4", 3),
        ("normal", "<f4", 3),
        ("tangent1", "<f4", 3),
        ("tangent2", "<f4", 3),
        ("tangentSpeed1", "<f4"),
        ("tangentSpeed2", "<f4"),
        ("tangentMass", "<f4", 4),
        ("tangentImpulse", "<f4", 2),
        ("motorImpulse", "<f4"),
        ("motorMass", "<f4"),
        ("motorSpeed", "<f4"),
        ("pointCount", "<u4"),
        ("constraint", "<u4"),
        ("pad", "<u4", 4),
        ("points", VELOCITY_POINT_DTYPE, 4),
        ("positionPoints", POSITION_POINT_DTYPE, 4),
    ]
)
# b3g_shape_cast_input: a convex shape at a transform swept along a
# displacement (b3World::ShapeCast's arguments, world.cpp:752-753).
SHAPE_CAST_DTYPE = np.dtype(
    [
        ("type", "<u4"),
        ("hull", "<u4"),
        ("world", "<u4"),
        ("pad", "<u4"),
        ("params", "<f4", 12),
        ("position", "<f4", 3),
        ("rotation", "<f4", 4),
        ("displacement", "<f4", 3),
        ("pad2", "<f4", 2),
    ]
)
assert SHAPE_CAST_DTYPE.itemsize == 112

# b3g_toi_input (b3TOIInput) and b3g_gjk_cast_input (b3ShapeCast's arguments).
SWEEP_FIELDS = 18  # localCenter, orientation0, worldCenter0, t0, orientation, worldCenter
TOI_INPUT_DTYPE = np.dtype(
    [
        ("type_a", "<u4"), ("hull_a", "<u4"), ("type_b", "<u4"), ("hull_b", "<u4"),
        ("params_a", "<f4", 12), ("params_b", "<f4", 12),
        ("sweep_a", "<f4", SWEEP_FIELDS), ("sweep_b", "<f4", SWEEP_FIELDS),
        ("t_max", "<f4"), ("pad", "<f4", 3),
    ]
)
GJK_CAST_DTYPE = np.dtype(
    [
        ("type_a", "<u4"), ("hull_a", "<u4"), ("type_b", "<u4"), ("hull_b", "<u4"),
        ("params_a", "<f4", 12), ("params_b", "<f4", 12),
        ("xf_a", "<f4", 7), ("xf_b", "<f4", 7), ("translation_b", "<f4", 3), ("pad", "<f4", 3),
    ]
)
assert TOI_INPUT_DTYPE.itemsize == 272 and GJK_CAST_DTYPE.itemsize == 192
assert SOLVER_BODY_DTYPE.itemsize == 112 and CONTACT_CONSTRAINT_DTYPE.itemsize == 128
assert MANIFOLD_CONSTRAINT_DTYPE.itemsize == 464

EXPORTED = [
    "b3g_create",
    "b3g_destroy",
    "b3g_last_error",
    "b3g_set_hulls",
    "b3g_set_bodies",
    "b3g_set_fixtures",
    "b3g_set_awake",
    "b3g_set_triangle_wings",
    "b3g_set_meshes",
    "b3g_mesh_wings",
    "b3g_collide",
    "b3g_get_counts",
    "b3g_get_pass_stats",
    "b3g_set_walk_limit",
    "b3g_set_tree_rebuild_interval",
    "b3g_set_joint_pairs",
    "b3g_set_contact_veto",
    "b3g_fetch_new_pairs",
    "b3g_finish_pass",
    "b3g_fetch_contacts",
    "b3g_fetch_manifolds",
    "b3g_fetch_touching",
    "b3g_fetch_ended",
    "b3g_fetch_fixture_contacts",
    "b3g_fetch_results_async",
    "b3g_fetch_results_packed_async",
    "b3g_wait_results",
    "b3g_fetch_awake",
    "b3g_fetch_caches",
    "b3g_fetch_fat_aabbs",
    "b3g_load_impulses",
    "b3g_load_mesh_impulses",
    "b3g_device_results",
    "b3g_get_totals",
    "b3g_set_profiling",
    "b3g_get_profile",
    "b3g_stage_name",
    "b3g_collide_pairs",
    "b3g_find_pairs_static",
    "b3g_query_aabb",
    "b3g_ray_cast",
    "b3g_ray_cast_single",
    "b3g_ray_cast_single_device",
    "b3g_shape_cast",
    "b3g_shape_cast_single",
    "b3g_shape_cast_single_device",
    "b3g_time_of_impact",
    "b3g_time_of_impact_device",
    "b3g_time_of_impact_aabb",
    "b3g_gjk_shape_cast",
    "b3g_set_materials",
    "b3g_contact_constraints",
    "b3g_contact_constraints_device",
    "b3g_autotune",
    "b3g_update_scene",
    "b3g_update_scene_device",
    "b3g_set_active",
    "b3g_world_counts",
    "b3g_kinematic_step",
    "b3g_set_tuning",
    "b3g_get_tuning",
    "b3g_hull_from_points",
    "b3g_hull_box",
]

_lib = None


def _p(t):
    return ctypes.POINTER(t)


def load():
    """Load libb3g.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
            "(make -C bounce_b200/csrc); there is no CPU fallback"
        )
    lib = ctypes.CDLL(LIB_PATH)
    u32p, f32p, u8p, vp = _p(ctypes.c_uint32), _p(ctypes.c_float), _p(ctypes.c_uint8), ctypes.c_void_p
    ctx = ctypes.c_void_p
    sig = {
        "b3g_create": ([_p(Config), _p(ctypes.c_void_p)], ctypes.c_int),
        "b3g_destroy": ([ctx], None),
        "b3g_last_error": ([ctx], ctypes.c_char_p),
        "b3g_set_hulls": ([ctx, ctypes.c_uint32, u32p, f32p, u32p, u32p, f32p, f32p], ctypes.c_int),
        "b3g_set_bodies": ([ctx, ctypes.c_uint32, u32p, u32p, u8p], ctypes.c_int),
        "b3g_set_fixtures": ([ctx, ctypes.c_uint32, u32p, u32p, u32p, f32p, u32p, u32p], ctypes.c_int),
        "b3g_set_awake": ([ctx, u8p], ctypes.c_int),
        "b3g_set_triangle_wings": ([ctx, ctypes.c_uint32, u32p, f32p], ctypes.c_int),
        "b3g_set_meshes": ([ctx, ctypes.c_uint32, u32p, f32p, u32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_mesh_wings": ([ctx, ctypes.c_uint32, u32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_collide": ([ctx, vp, ctypes.c_int, vp], ctypes.c_int),
        "b3g_get_counts": ([ctx, _p(Counts)], ctypes.c_int),
        "b3g_get_pass_stats": ([ctx, _p(ctypes.c_uint32), ctypes.c_uint32], ctypes.c_int),
        "b3g_set_walk_limit": ([ctx, ctypes.c_uint32], ctypes.c_int),
        "b3g_set_tree_rebuild_interval": ([ctx, ctypes.c_uint32], ctypes.c_int),
        "b3g_set_joint_pairs": ([ctx, ctypes.c_uint32, _p(ctypes.c_uint32)], ctypes.c_int),
        "b3g_set_contact_veto": ([ctx, ctypes.c_uint32, _p(ctypes.c_uint8)], ctypes.c_int),
        "b3g_fetch_new_pairs": ([ctx, _p(ctypes.c_uint32), ctypes.c_uint32], ctypes.c_int),
        "b3g_finish_pass": ([ctx, _p(ctypes.c_uint8), ctypes.c_uint32], ctypes.c_int),
        "b3g_fetch_contacts": ([ctx, u32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_fetch_manifolds": ([ctx, vp, ctypes.c_uint32], ctypes.c_int),
        "b3g_fetch_touching": ([ctx, u32p, vp, ctypes.c_uint32], ctypes.c_int),
        "b3g_fetch_ended": ([ctx, u32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_fetch_fixture_contacts": ([ctx, u32p, u32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_fetch_results_async": ([ctx, vp, ctypes.c_uint32, vp, vp, ctypes.c_uint32, _p(Counts)], ctypes.c_int),
        "b3g_fetch_results_packed_async": ([ctx, vp, ctypes.c_uint32, vp, vp, ctypes.c_uint32, ctypes.c_uint64,
                                            _p(Counts)], ctypes.c_int),
        "b3g_wait_results": ([ctx], ctypes.c_int),
        "b3g_fetch_awake": ([ctx, u8p, ctypes.c_uint32], ctypes.c_int),
        "b3g_fetch_caches": ([ctx, u32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_fetch_fat_aabbs": ([ctx, f32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_load_impulses": ([ctx, f32p, f32p, f32p], ctypes.c_int),
        "b3g_load_mesh_impulses": ([ctx, f32p, f32p, f32p], ctypes.c_int),
        "b3g_device_results": ([ctx, _p(ctypes.c_void_p), _p(ctypes.c_void_p)], ctypes.c_int),
        "b3g_get_totals": ([ctx, _p(ctypes.c_uint64), ctypes.c_int], ctypes.c_int),
        "b3g_set_profiling": ([ctx, ctypes.c_int], ctypes.c_int),
        "b3g_get_profile": ([ctx, _p(ctypes.c_double), u32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_stage_name": ([ctypes.c_uint32], ctypes.c_char_p),
        "b3g_collide_pairs": (
            [ctx, ctypes.c_uint32, u32p, u32p, f32p, f32p, f32p, f32p, u32p, vp],
            ctypes.c_int,
        ),
        "b3g_find_pairs_static": ([vp, ctypes.c_uint32, vp, ctypes.c_uint32, vp, vp], ctypes.c_int),
        "b3g_autotune": ([ctx, ctypes.c_uint32, vp, u32p], ctypes.c_int),
        "b3g_query_aabb": ([ctx, ctypes.c_uint32, f32p, u32p, u32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_ray_cast": ([ctx, ctypes.c_uint32, f32p, u32p, u32p, f32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_ray_cast_single": ([ctx, ctypes.c_uint32, f32p, u32p, u32p, f32p], ctypes.c_int),
        "b3g_ray_cast_single_device": ([ctx, ctypes.c_uint32, vp, vp, vp, vp, vp], ctypes.c_int),
        "b3g_shape_cast": ([ctx, ctypes.c_uint32, vp, u32p, f32p, ctypes.c_uint32], ctypes.c_int),
        "b3g_shape_cast_single": ([ctx, ctypes.c_uint32, vp, u32p, f32p], ctypes.c_int),
        "b3g_shape_cast_single_device": ([ctx, ctypes.c_uint32, vp, vp, vp, vp], ctypes.c_int),
        "b3g_time_of_impact": ([ctx, ctypes.c_uint32, vp, u32p], ctypes.c_int),
        "b3g_time_of_impact_device": ([ctx, ctypes.c_uint32, vp, vp, vp], ctypes.c_int),
        "b3g_time_of_impact_aabb": ([ctx, ctypes.c_uint32, f32p, u32p], ctypes.c_int),
        "b3g_gjk_shape_cast": ([ctx, ctypes.c_uint32, vp, f32p], ctypes.c_int),
        "b3g_set_materials": ([ctx, f32p, f32p], ctypes.c_int),
        "b3g_contact_constraints": ([ctx, ctypes.c_uint32, u32p, vp, ctypes.c_float, ctypes.c_int, vp,
                                     ctypes.c_uint32, vp, ctypes.c_uint32, u32p], ctypes.c_int),
        "b3g_contact_constraints_device": ([ctx, ctypes.c_uint32, vp, vp, ctypes.c_float, ctypes.c_int, vp,
                                            ctypes.c_uint32, vp, ctypes.c_uint32, vp, vp], ctypes.c_int),
        "b3g_update_scene": ([ctx, ctypes.c_uint32, u32p, u32p, u32p, u8p, ctypes.c_uint32, u32p, u32p, u32p, u32p,
                              f32p, u32p, ctypes.c_uint32, u32p, vp], ctypes.c_int),
        "b3g_update_scene_device": ([ctx, ctypes.c_uint32, vp, vp, vp, ctypes.c_uint32, vp, vp, vp, vp, vp, vp,
                                     ctypes.c_uint32, vp, vp], ctypes.c_int),
        "b3g_set_active": ([ctx, ctypes.c_uint32, ctypes.c_uint32], ctypes.c_int),
        "b3g_world_counts": ([ctx, ctypes.c_uint32, vp, vp], ctypes.c_int),
        "b3g_kinematic_step": ([vp, vp, ctypes.c_uint32, ctypes.c_float, vp], ctypes.c_int),
        "b3g_set_tuning": ([ctx, u32p], ctypes.c_int),
        "b3g_get_tuning": ([ctx, u32p], ctypes.c_int),
        "b3g_hull_from_points": ([f32p, ctypes.c_uint32, f32p, u32p, u32p, f32p, f32p, u32p], ctypes.c_int),
        "b3g_hull_box": (
            [ctypes.c_float, ctypes.c_float, ctypes.c_float, f32p, u32p, u32p, f32p, f32p, u32p],
            ctypes.c_int,
        ),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def ptr(a, t):
    """ctypes pointer into a C-contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(ctypes.POINTER(t))

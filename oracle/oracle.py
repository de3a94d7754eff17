"""ctypes driver for the reference build in oracle/_ref (see Makefile and
ref_harness.cpp).

TEST INFRASTRUCTURE ONLY. Imported by tests/, by __graft_entry__.smoke() as
the checker and by bench.py's CPU-baseline leg; never by the product.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# The reference checkout (Bounce sources) the oracle is compiled from: the
# BOUNCE_REF_SRC environment variable, else the checkout's usual location.
REFERENCE_SRC = os.environ.get("BOUNCE_REF_SRC", "/root/reference")

# Harness dump records (ref_harness.cpp DumpPoint / DumpManifold / DumpContact).
DPOINT = np.dtype(
    [
        ("n", "<f8", 3),
        ("p1", "<f8", 3),
        ("p2", "<f8", 3),
        ("normalImpulse", "<f8"),
        ("triangleKey", "<u4"),
        ("key", "<u4", 4),
        ("persisting", "<u4"),
        ("edgeContact", "<u4"),
        ("pad", "<u4"),
    ]
)
DMANIFOLD = np.dtype(
    [("pointCount", "<u4"), ("pad", "<u4"), ("tangentImpulse", "<f8", 2), ("motorImpulse", "<f8"), ("points", DPOINT, 4)]
)
DCONTACT = np.dtype(
    [
        ("fixtureA", "<u4"),
        ("fixtureB", "<u4"),
        ("flags", "<u4"),
        ("manifoldCount", "<u4"),
        ("cache", "<u4", 4),
        ("manifolds", DMANIFOLD, 3),
    ]
)


def build(quiet=True):
    """Compile oracle/_ref from the reference sources at REFERENCE_SRC."""
    if not os.path.isdir(REFERENCE_SRC):
        return False
    cmd = ["make", "-C", HERE, "-j8", f"REF={REFERENCE_SRC}"]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)
    return True


def available(precision=32):
    return os.path.exists(os.path.join(REF_DIR, f"libb3ref{precision}.so"))


_libs = {}


def lib(precision=32):
    """The reference build: 32 (FP32), 64 (the FP64 rerun) or "shim" (FP32
    with the GPU contact manager of bounce_b200/shim in place of the
    reference's, linked to the library)."""
    if precision in _libs:
        return _libs[precision]
    name = "libb3shim.so" if precision == "shim" else f"libb3ref{precision}.so"
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        raise RuntimeError(f"{path} missing: build the oracle with make -C oracle")
    L = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    vp, u32p, f32p, f64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
    sig = {
        "refh_create": ([ctypes.c_uint32, u32p, f32p, u32p, u32p, f32p, f32p], vp),
        "refh_destroy": ([vp], None),
        "refh_add_meshes": ([vp, ctypes.c_uint32, u32p, f32p, u32p], None),
        "refh_mesh_wings": ([vp, ctypes.c_uint32, u32p], None),
        "refw_create": (
            [vp, ctypes.c_uint32, u32p, f32p, ctypes.c_uint32, u32p, u32p, u32p, f32p, u32p, ctypes.c_uint32],
            vp,
        ),
        "refw_destroy": ([vp], None),
        "refw_get_bodies": ([vp, f32p], None),
        "refw_set_sweeps": ([vp, f32p], None),
        "refw_set_local_centers": ([vp, f32p], None),
        "refw_add_joints": ([vp, ctypes.c_uint32, u32p], None),
        "refw_clear_joints": ([vp], None),
        "refw_set_filter": ([vp, ctypes.c_uint32, ctypes.c_uint32], None),
        "refw_filter_calls": ([vp, u32p, ctypes.c_uint32], ctypes.c_uint32),
        "ref_filter_rejects": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32], ctypes.c_uint32),
        "refw_set_awake": ([vp, ctypes.POINTER(ctypes.c_uint8)], None),
        "refw_get_awake": ([vp, ctypes.POINTER(ctypes.c_uint8)], None),
        "refw_set_triangle_wings": ([vp, ctypes.c_uint32, u32p, f32p], None),
        "refw_pass_sleep": ([vp, ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint8), f64p], None),
        "refw_set_convex_cache": ([ctypes.c_uint32], None),
        "refw_first_pass": ([vp, f64p], None),
        "refw_pass": ([vp, f64p], None),
        "refw_contact_count": ([vp], ctypes.c_uint32),
        "refw_touching_count": ([vp, u32p, u32p], ctypes.c_uint32),
        "refw_fat_aabbs": ([vp, f32p], None),
        "refw_proxy_ids": ([vp, u32p], None),
        "refw_dump_pairs": ([vp, u32p], ctypes.c_uint32),
        "refw_dump_contacts": ([vp, ctypes.c_uint32, ctypes.c_uint32, vp], ctypes.c_uint32),
        "refw_load_impulses": ([vp, vp], None),
        "refw_query_aabb": ([vp, f32p, u32p, ctypes.c_uint32], ctypes.c_uint32),
        "refw_fixture_edges": ([vp, u32p, u32p, ctypes.c_uint32], ctypes.c_uint32),
        "refw_contact_solver": (
            [vp, ctypes.c_uint32, u32p, f32p, f32p, f32p, ctypes.c_float, ctypes.c_uint32, u32p, u32p, u32p, f64p],
            ctypes.c_uint32,
        ),
        "refw_mass_data": ([vp, f32p], None),
        "refw_ray_cast": ([vp, f32p, u32p, f64p, ctypes.c_uint32], ctypes.c_uint32),
        "refw_ray_cast_single": ([vp, f32p, u32p, f64p], ctypes.c_uint32),
        "refw_ray_cast_single_batch": ([vp, f32p, ctypes.c_uint32, u32p], ctypes.c_double),
        "refw_shape_cast": ([vp, f32p, u32p, f64p, ctypes.c_uint32], ctypes.c_uint32),
        "refw_shape_cast_single": ([vp, f32p, u32p, f64p], ctypes.c_uint32),
        "refw_shape_cast_single_batch": ([vp, f32p, ctypes.c_uint32, u32p, f32p], ctypes.c_double),
        "ref_sizeof_dump_contact": ([], ctypes.c_uint32),
        "ref_sizeof_scalar": ([], ctypes.c_uint32),
        "ref_collide": (
            [vp, ctypes.c_uint32, f32p, ctypes.c_uint32, ctypes.c_uint32, f32p, ctypes.c_uint32, f32p, f32p, f32p, f32p,
             u32p, vp],
            ctypes.c_int,
        ),
        "ref_collide_wings": (
            [vp, ctypes.c_uint32, f32p, ctypes.c_uint32, ctypes.c_uint32, f32p, ctypes.c_uint32, f32p, f32p, f32p, f32p,
             u32p, vp, f32p, f32p],
            ctypes.c_int,
        ),
        "ref_sweep_xf0": ([f32p, f32p, f32p, f32p, f32p], None),
        "refh_toi": ([vp, ctypes.c_uint32, f32p, u32p], None),
        "refh_toi_aabb": ([ctypes.c_uint32, f32p, u32p], None),
        "refh_gjk_cast": ([vp, ctypes.c_uint32, f32p, f32p], None),
    }
    sig["stepw_create"] = ([vp, ctypes.c_uint32, u32p, f32p, f32p, ctypes.c_uint32, u32p, u32p, u32p, f32p, u32p, f32p],
                           vp)
    sig["stepw_step"] = ([vp, ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32], None)
    if precision == "shim":
        sig["b3g_shim_failures"] = ([], ctypes.c_uint32)
    if precision == 64:
        sig["refc_reset"] = ([], None)
        sig["refc_read"] = ([f64p, ctypes.c_uint32], ctypes.c_uint32)
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    assert L.ref_sizeof_dump_contact() == DCONTACT.itemsize, "dump layout mismatch"
    _libs[precision] = L
    return L


# Counters of flop_count.cpp (FP64 build), in its RC_* order.
FLOP_COUNTERS = ("flops", "spheres", "capsule_sphere", "capsules", "hull_sphere", "hull_capsule", "hulls",
                 "face_queries", "face_trips", "edge_queries", "edge_pairs", "edge_qualified", "gjk_calls",
                 "gjk_iters", "clip_planes", "clip_vertices", "cache_reads", "hull_sphere_planes", "flops_sat",
                 "flops_gjk", "flops_clip")


def filter_rejects(ia, ib, modulus, salt):
    """The seeded contact filter's rule (vectorised): reject when a hash of
    (smaller, larger fixture index, salt) is 0 modulo `modulus`."""
    ia = np.asarray(ia, np.uint64)
    ib = np.asarray(ib, np.uint64)
    lo, hi = np.minimum(ia, ib), np.maximum(ia, ib)
    h = (lo * np.uint64(2654435761) + hi * np.uint64(40503) + np.uint64(salt) * np.uint64(97)) & np.uint64(0xFFFFFFFF)
    if modulus == 0:
        return np.zeros(h.shape, bool)
    return ((h >> np.uint64(8)) % np.uint64(modulus)) == 0


def flop_counts(reset=False):
    """The narrowphase trip and flop counters of the FP64 reference build
    since the last reset (oracle/flop_count.cpp, constants in flops.h)."""
    L = lib(64)
    out = np.zeros(len(FLOP_COUNTERS), np.float64)
    n = L.refc_read(out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(out))
    assert n == len(out), n
    if reset:
        L.refc_reset()
    return dict(zip(FLOP_COUNTERS, out.tolist()))


def _p(a, t):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(t))


class RefHulls:
    """Hulls and, when given, triangle meshes (mesh_arrays: desc, verts, tris)."""

    def __init__(self, hull_arrays, precision=32, mesh_arrays=None):
        self.L = lib(precision)
        h = hull_arrays
        self._keep = (h, mesh_arrays)
        nh = len(h["desc"]) // 6
        self.h = self.L.refh_create(
            nh, _p(h["desc"], ctypes.c_uint32), _p(h["verts"], ctypes.c_float), _p(h["edges"], ctypes.c_uint32),
            _p(h["faces"], ctypes.c_uint32), _p(h["planes"], ctypes.c_float), _p(h["centroids"], ctypes.c_float),
        )
        if mesh_arrays is not None:
            m = mesh_arrays
            self.L.refh_add_meshes(self.h, len(m["desc"]) // 4, _p(m["desc"], ctypes.c_uint32),
                                   _p(m["verts"], ctypes.c_float), _p(m["tris"], ctypes.c_uint32))

    def time_of_impact(self, queries):
        """b3TimeOfImpact(b3TOIInput) per query ((n, 68) float32 words in the
        b3g_toi_input layout): (n, 4) u32 state, t bits, iterations, 0."""
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, 68)
        out = np.zeros((max(len(q), 1), 4), np.uint32)
        self.L.refh_toi(self.h, len(q), _p(q, ctypes.c_float), _p(out, ctypes.c_uint32))
        return out[:len(q)]

    def gjk_shape_cast(self, queries):
        """b3ShapeCast per query ((n, 48) words, b3g_gjk_cast_input layout):
        (n, 9) float32 words hit, t, point, normal, iterations."""
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, 48)
        out = np.zeros((max(len(q), 1), 9), np.float32)
        self.L.refh_gjk_cast(self.h, len(q), _p(q, ctypes.c_float), _p(out, ctypes.c_float))
        return out[:len(q)]

    def mesh_wings(self, m, n_triangles):
        out = np.zeros(3 * n_triangles, np.uint32)
        self.L.refh_mesh_wings(self.h, m, _p(out, ctypes.c_uint32))
        return out.reshape(-1, 3)

    def __del__(self):
        try:
            self.L.refh_destroy(self.h)
        except Exception:
            pass


class RefWorld:
    """One reference b3World built from a bounce_b200.scene.Scene."""

    def __init__(self, scene, precision=32, warm_starting=True, hulls=None):
        self.L = lib(precision)
        self.precision = precision
        self.scene = scene
        self.hulls = hulls or RefHulls(scene.hull_arrays, precision, getattr(scene, "mesh_arrays", None))
        s = scene
        self.w = self.L.refw_create(
            self.hulls.h, s.n_bodies, _p(s.body_type, ctypes.c_uint32), _p(s.body_pose, ctypes.c_float),
            s.n_fixtures, _p(s.fix_body, ctypes.c_uint32), _p(s.fix_type, ctypes.c_uint32),
            _p(s.fix_hull, ctypes.c_uint32), _p(s.fix_params, ctypes.c_float), _p(s.fix_flags, ctypes.c_uint32),
            1 if warm_starting else 0,
        )
        self.times = np.zeros(2)
        wings = getattr(scene, "tri_wings", None)
        if wings is not None and len(wings):
            self.set_triangle_wings(scene.tri_fixtures, wings)

    def close(self):
        if self.w:
            self.L.refw_destroy(self.w)
            self.w = None

    @classmethod
    def stepping(cls, scene, build=32, gravity=(0.0, -9.8, 0.0)):
        """A world for whole b3World::Step calls (solver, islands, sleep): the
        scene's bodies with their velocities, gravity and sleeping on. build:
        32 (the reference) or "shim" (the reference with the GPU contact
        manager)."""
        self = cls.__new__(cls)
        self.L = lib(build)
        self.precision = 32
        self.scene = scene
        self.hulls = RefHulls(scene.hull_arrays, build, getattr(scene, "mesh_arrays", None))
        s = scene
        vel = np.ascontiguousarray(np.concatenate([s.body_lin, s.body_ang], axis=1), np.float32)
        g = np.asarray(gravity, np.float32)
        self._keep = (vel, g)
        self.w = self.L.stepw_create(
            self.hulls.h, s.n_bodies, _p(s.body_type, ctypes.c_uint32), _p(s.body_pose, ctypes.c_float),
            _p(vel, ctypes.c_float), s.n_fixtures, _p(s.fix_body, ctypes.c_uint32), _p(s.fix_type, ctypes.c_uint32),
            _p(s.fix_hull, ctypes.c_uint32), _p(s.fix_params, ctypes.c_float), _p(s.fix_flags, ctypes.c_uint32),
            _p(g, ctypes.c_float))
        self.times = np.zeros(2)
        return self

    def step(self, dt=1.0 / 60.0, velocity_iterations=8, position_iterations=2):
        self.L.stepw_step(self.w, dt, velocity_iterations, position_iterations)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bodies17(self):
        out = np.zeros(17 * self.scene.n_bodies, np.float32)
        self.L.refw_get_bodies(self.w, _p(out, ctypes.c_float))
        return out

    def local_centers(self):
        return self.bodies17().reshape(-1, 17)[:, 14:17].copy()

    def set_local_centers(self, lc):
        """Use the caller's centres of mass (n x 3, body frame) for the
        dynamic bodies instead of the ones the reference computed."""
        a = np.ascontiguousarray(lc, np.float32).reshape(-1)
        assert len(a) == 3 * self.scene.n_bodies
        self.L.refw_set_local_centers(self.w, _p(a, ctypes.c_float))

    def add_joints(self, body_pairs):
        """A joint with collideConnected = false between each body pair."""
        a = np.ascontiguousarray(body_pairs, np.uint32).reshape(-1)
        self.L.refw_add_joints(self.w, len(a) // 2, _p(a, ctypes.c_uint32))

    def clear_joints(self):
        self.L.refw_clear_joints(self.w)

    def set_filter(self, modulus, salt=0):
        """The seeded contact filter (filter_rejects); modulus 0 removes it."""
        self.L.refw_set_filter(self.w, modulus, salt)

    def filter_calls(self):
        """Fixture pairs the filter was asked about by AddPair in the last
        pass, in call order."""
        out = np.zeros(2 * 4_000_000, np.uint32)
        n = self.L.refw_filter_calls(self.w, _p(out, ctypes.c_uint32), len(out) // 2)
        return out[:2 * n].reshape(-1, 2).copy()

    def set_sweeps(self, sweeps14):
        a = np.ascontiguousarray(sweeps14, np.float32)
        self.L.refw_set_sweeps(self.w, _p(a, ctypes.c_float))

    def set_awake(self, awake):
        a = np.ascontiguousarray(awake, np.uint8)
        self.L.refw_set_awake(self.w, _p(a, ctypes.c_uint8))

    def first_pass(self):
        t = np.zeros(2)
        self.L.refw_first_pass(self.w, _p(t, ctypes.c_double))
        self.times = t
        return t

    def step_pass(self):
        t = np.zeros(2)
        self.L.refw_pass(self.w, _p(t, ctypes.c_double))
        self.times = t
        return t

    def step_pass_sleep(self, moved, awake):
        """A pass whose synchronised bodies are `moved` and whose
        UpdateContacts starts with the awake flags `awake`."""
        t = np.zeros(2)
        m = np.ascontiguousarray(moved, np.uint8)
        a = np.ascontiguousarray(awake, np.uint8)
        self.L.refw_pass_sleep(self.w, _p(m, ctypes.c_uint8), _p(a, ctypes.c_uint8), _p(t, ctypes.c_double))
        self.times = t
        return t

    def set_triangle_wings(self, fixtures, wings):
        f = np.ascontiguousarray(fixtures, np.uint32)
        w = np.ascontiguousarray(wings, np.float32).reshape(-1)
        self.L.refw_set_triangle_wings(self.w, len(f), _p(f, ctypes.c_uint32), _p(w, ctypes.c_float))

    def awake(self):
        out = np.zeros(len(self.bodies17()) // 17, np.uint8)
        self.L.refw_get_awake(self.w, _p(out, ctypes.c_uint8))
        return out

    def contact_count(self):
        return self.L.refw_contact_count(self.w)

    def fixture_edges(self):
        """Each fixture's contact edge list: (offsets (fixtures + 1,), (edges, 2)
        fixtureA, fixtureB of the edge's contact)."""
        nf = self.scene.n_fixtures
        offsets = np.zeros(nf + 1, np.uint32)
        cap = 2 * self.contact_count()
        pairs = np.zeros((max(cap, 1), 2), np.uint32)
        k = self.L.refw_fixture_edges(self.w, _p(offsets, ctypes.c_uint32), _p(pairs, ctypes.c_uint32), cap)
        return offsets, pairs[:k]

    def mass_data(self):
        """Per body as the reference computed it from the fixtures: m_invMass
        (n,), m_invI (n, 9) and m_worldInvI (n, 9), matrices by columns."""
        nb = self.scene.n_bodies
        out = np.zeros((max(nb, 1), 19), np.float32)
        self.L.refw_mass_data(self.w, _p(out, ctypes.c_float))
        return out[:nb, 0].copy(), out[:nb, 1:10].copy(), out[:nb, 10:19].copy()

    def contact_solver(self, bodies, friction, restitution, dt_ratio=1.0, warm=True, contacts=None, timed=False):
        """The reference's b3ContactSolver constructor and
        InitializeVelocityConstraints on this world's contacts (the listed
        contact-list positions, or every touching non-sensor contact in list
        order). bodies: (n, 28) float32 in the b3g_solver_body layout;
        friction, restitution per fixture. Returns the raw records:
        constraints (k, 32) and manifolds (m, 116) as uint32 words (and, with
        timed, the seconds of the constructor and InitializeVelocityConstraints)."""
        b = np.ascontiguousarray(bodies, np.float32).reshape(-1, 28)
        fr = np.ascontiguousarray(friction, np.float32)
        re = np.ascontiguousarray(restitution, np.float32)
        lst = None if contacts is None else np.ascontiguousarray(contacts, np.uint32)
        count = self.contact_count() if lst is None else len(lst)
        con = np.zeros((max(count, 1), 32), np.uint32)
        man = np.zeros((max(3 * count, 1), 116), np.uint32)
        mc = ctypes.c_uint32()
        secs = ctypes.c_double()
        k = self.L.refw_contact_solver(self.w, 0 if lst is None else len(lst), _p(lst, ctypes.c_uint32),
                                       _p(b, ctypes.c_float), _p(fr, ctypes.c_float), _p(re, ctypes.c_float),
                                       float(dt_ratio), 1 if warm else 0, _p(con, ctypes.c_uint32),
                                       _p(man, ctypes.c_uint32), ctypes.byref(mc), ctypes.byref(secs))
        if timed:
            return con[:k], man[:mc.value], secs.value
        return con[:k], man[:mc.value]

    def query_aabb(self, box):
        """b3World::QueryAABB: indices of the fixtures reported (report order)."""
        b = np.ascontiguousarray(box, np.float32)
        cap = self.scene.n_fixtures
        out = np.zeros(max(cap, 1), np.uint32)
        n = self.L.refw_query_aabb(self.w, _p(b, ctypes.c_float), _p(out, ctypes.c_uint32), cap)
        return out[:n]

    def ray_cast(self, ray):
        """b3World::RayCast keeping every hit: (fixtures, hits (k, 7): point, normal, fraction)."""
        r = np.ascontiguousarray(ray, np.float32)
        cap = self.scene.n_fixtures
        fix = np.zeros(max(cap, 1), np.uint32)
        hit = np.zeros((max(cap, 1), 7), np.float64)
        n = self.L.refw_ray_cast(self.w, _p(r, ctypes.c_float), _p(fix, ctypes.c_uint32),
                                 hit.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap)
        return fix[:n], hit[:n]

    def ray_cast_single(self, ray):
        """b3World::RayCastSingle: (fixture, hit (7,)) or (None, None)."""
        r = np.ascontiguousarray(ray, np.float32)
        fix = np.zeros(1, np.uint32)
        hit = np.zeros(7, np.float64)
        if not self.L.refw_ray_cast_single(self.w, _p(r, ctypes.c_float), _p(fix, ctypes.c_uint32),
                                           hit.ctypes.data_as(ctypes.POINTER(ctypes.c_double))):
            return None, None
        return int(fix[0]), hit

    def ray_cast_single_batch(self, rays):
        """RayCastSingle for each ray, timed inside the harness: (fixtures, seconds)."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        fix = np.zeros(max(len(r), 1), np.uint32)
        t = self.L.refw_ray_cast_single_batch(self.w, _p(r, ctypes.c_float), len(r), _p(fix, ctypes.c_uint32))
        return fix[:len(r)], t

    def shape_cast(self, cast):
        """b3World::ShapeCast keeping every hit; cast is 28 float32 words in
        the b3g_shape_cast_input layout: (fixtures, hits (k, 7): point, normal,
        fraction)."""
        c = np.ascontiguousarray(cast, np.float32).reshape(28)
        cap = 4 * self.scene.n_fixtures + 64
        fix = np.zeros(cap, np.uint32)
        hit = np.zeros((cap, 7), np.float64)
        n = self.L.refw_shape_cast(self.w, _p(c, ctypes.c_float), _p(fix, ctypes.c_uint32),
                                   hit.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap)
        assert n <= cap
        return fix[:n], hit[:n]

    def shape_cast_single(self, cast):
        """b3World::ShapeCastSingle: (fixture, hit (7,)) or (None, None)."""
        c = np.ascontiguousarray(cast, np.float32).reshape(28)
        fix = np.zeros(1, np.uint32)
        hit = np.zeros(7, np.float64)
        if not self.L.refw_shape_cast_single(self.w, _p(c, ctypes.c_float), _p(fix, ctypes.c_uint32),
                                             hit.ctypes.data_as(ctypes.POINTER(ctypes.c_double))):
            return None, None
        return int(fix[0]), hit

    def shape_cast_single_batch(self, casts):
        """ShapeCastSingle for each cast, timed inside the harness:
        (fixtures, fractions, seconds)."""
        c = np.ascontiguousarray(casts, np.float32).reshape(-1, 28)
        fix = np.zeros(max(len(c), 1), np.uint32)
        frac = np.zeros(max(len(c), 1), np.float32)
        t = self.L.refw_shape_cast_single_batch(self.w, _p(c, ctypes.c_float), len(c), _p(fix, ctypes.c_uint32),
                                                _p(frac, ctypes.c_float))
        return fix[:len(c)], frac[:len(c)], t

    def load_impulses(self, normal, tangent, motor):
        """The solver's impulses for every contact in list order, per manifold
        (B3_MAX_MANIFOLDS = 3): normal (n, 3, 4), tangent (n, 3, 2), motor (n, 3)."""
        n = self.contact_count()
        rec = np.zeros(max(n, 1), DCONTACT)
        rec["manifolds"]["points"]["normalImpulse"][:n] = np.asarray(normal, np.float64)[:n]
        rec["manifolds"]["tangentImpulse"][:n] = np.asarray(tangent, np.float64)[:n]
        rec["manifolds"]["motorImpulse"][:n] = np.asarray(motor, np.float64)[:n]
        self.L.refw_load_impulses(self.w, ctypes.c_void_p(rec.ctypes.data))

    def touching(self):
        m, p = ctypes.c_uint32(), ctypes.c_uint32()
        t = self.L.refw_touching_count(self.w, ctypes.byref(m), ctypes.byref(p))
        return t, m.value, p.value

    def pairs(self):
        n = self.contact_count()
        out = np.zeros((max(n, 1), 3), np.uint32)
        self.L.refw_dump_pairs(self.w, _p(out, ctypes.c_uint32))
        return out[:n]

    def contacts(self, start=0, count=None):
        n = self.contact_count()
        if count is None:
            count = n - start
        out = np.zeros(max(count, 1), DCONTACT)
        m = self.L.refw_dump_contacts(self.w, start, count, ctypes.c_void_p(out.ctypes.data))
        return out[:m]

    def fat_aabbs(self):
        out = np.zeros((self.scene.n_fixtures, 6), np.float32)
        self.L.refw_fat_aabbs(self.w, _p(out, ctypes.c_float))
        return out

    def proxy_ids(self):
        out = np.zeros(self.scene.n_fixtures, np.uint32)
        self.L.refw_proxy_ids(self.w, _p(out, ctypes.c_uint32))
        return out


_restate = None


def time_of_impact_aabb(queries, precision=32):
    """b3TimeOfImpact(aabb1, d1, aabb2, d2) per query ((n, 18) float32):
    (n, 4) u32 state, t bits, iterations, 0."""
    L = lib(precision)
    q = np.ascontiguousarray(queries, np.float32).reshape(-1, 18)
    out = np.zeros((max(len(q), 1), 4), np.uint32)
    L.refh_toi_aabb(len(q), _p(q, ctypes.c_float), _p(out, ctypes.c_uint32))
    return out[:len(q)]


def restate():
    """The C restatement of the broadphase front end (restate.c)."""
    global _restate
    if _restate is None:
        path = os.path.join(REF_DIR, "librestate.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: build the oracle with make -C oracle")
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.rs_sync.argtypes = [ctypes.c_int, ctypes.c_uint32] + [vp] * 11
        L.rs_sync.restype = None
        L.rs_pairs.argtypes = [ctypes.c_uint32, vp, vp, vp, vp, vp, vp, ctypes.c_uint32]
        L.rs_pairs.restype = ctypes.c_uint32
        _restate = L
    return _restate


def restate_sync(scene, state17, fat, awake=None, creation=False):
    """Fat-AABB update of every fixture (in place on fat, 6 floats each); returns moved flags."""
    L = restate()
    nf = scene.n_fixtures
    aw = np.ascontiguousarray(np.ones(scene.n_bodies, np.uint8) if awake is None else awake, np.uint8)
    moved = np.zeros(nf, np.uint8)
    st = np.ascontiguousarray(state17, np.float32)
    ha = scene.hull_arrays
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    L.rs_sync(1 if creation else 0, nf, p(scene.fix_body), p(scene.fix_type), p(scene.fix_hull), p(scene.fix_params),
              p(scene.body_type), p(aw), p(st), p(ha["desc"]), p(ha["verts"]), p(fat), p(moved))
    return moved


def restate_pairs(scene, fat, keys=None):
    """Contact set (fixture A, fixture B) of the fat AABBs, sorted by pair."""
    L = restate()
    nf = scene.n_fixtures
    k = np.ascontiguousarray(np.arange(nf, dtype=np.uint32) if keys is None else keys, np.uint32)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    cap = 64 * nf + 1024
    out = np.zeros((cap, 2), np.uint32)
    n = L.rs_pairs(nf, p(fat), p(scene.fix_body), p(scene.body_type), p(scene.fix_type), p(k), p(out), cap)
    assert n <= cap
    out = out[:n]
    order = np.argsort((out[:, 0].astype(np.uint64) << 32) | out[:, 1])
    return out[order]


def set_convex_cache(on, precision=32):
    lib(precision).refw_set_convex_cache(1 if on else 0)


def collide(hulls, typeA, pA, hullA, typeB, pB, hullB, xfA, xfB, xf0A=None, xf0B=None, cache=None, precision=32,
            wingsA=None, wingsB=None):
    """One b3Collide* call of the reference (ref_collide in ref_harness.cpp);
    wingsA / wingsB: 12 floats of triangle edge wings."""
    L = lib(precision)
    f = lambda a: np.ascontiguousarray(a, np.float32)
    pa, pb = f(np.pad(np.asarray(pA, np.float32), (0, 12 - len(pA)))), f(np.pad(np.asarray(pB, np.float32), (0, 12 - len(pB))))
    xa, xb = f(xfA), f(xfB)
    x0a = f(xf0A if xf0A is not None else xfA)
    x0b = f(xf0B if xf0B is not None else xfB)
    c = np.ascontiguousarray(cache if cache is not None else np.array([0, 1, 0, 0]), np.uint32)
    out = np.zeros(1, DMANIFOLD)
    wa = None if wingsA is None else f(wingsA)
    wb = None if wingsB is None else f(wingsB)
    rc = L.ref_collide_wings(
        hulls.h, typeA, _p(pa, ctypes.c_float), hullA, typeB, _p(pb, ctypes.c_float), hullB, _p(xa, ctypes.c_float),
        _p(xb, ctypes.c_float), _p(x0a, ctypes.c_float), _p(x0b, ctypes.c_float), _p(c, ctypes.c_uint32),
        ctypes.c_void_p(out.ctypes.data), None if wa is None else _p(wa, ctypes.c_float),
        None if wb is None else _p(wb, ctypes.c_float),
    )
    if rc != 0:
        raise ValueError("unsupported shape pair")
    if cache is not None:
        cache[...] = c
    return out[0]

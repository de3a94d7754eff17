"""Python host mirror of the pipeline's C ABI (include/b3g.h).

``CollisionPipeline`` plays the role of Bounce's b3ContactManager +
b3BroadPhase for one context: ``collide()`` is one collision pass (the fixture
sync and FindNewContacts of the "Find New Pairs" block, world.cpp:424-449,
then UpdateContacts, contact_manager.cpp:225-287), and the fetch methods read
the contact list, the b3Manifold records and the destroyed contacts back.
Errors raise ``B3GError`` with the library's message; there is no CPU path.
"""
import ctypes

import numpy as np

from . import _native as N

u32, f32 = ctypes.c_uint32, ctypes.c_float


class CollisionPipeline:
    def __init__(self, scene, max_contacts=None, warm_starting=True, convex_cache=True, device=0, graph=False,
                 contact_filter=False):
        self.lib = N.load()
        self.scene = scene
        nf = scene.n_fixtures
        if max_contacts is None:
            max_contacts = max(1024, 32 * nf)
        ha = scene.hull_arrays
        cfg = N.Config(
            max_proxies=max(nf, 1),
            max_contacts=int(max_contacts),
            max_hull_data=0,
            flags=(N.FLAG_WARM_STARTING if warm_starting else 0) | (N.FLAG_CONVEX_CACHE if convex_cache else 0)
            | (N.FLAG_GRAPH if graph else 0) | (N.FLAG_CONTACT_FILTER if contact_filter else 0),
            device=device,
        )
        h = ctypes.c_void_p()
        rc = self.lib.b3g_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != 0:
            raise N.B3GError(rc, "b3g_create failed")
        self.ctx = h
        self.max_contacts = int(max_contacts)
        self.n_bodies = int(scene.n_bodies)
        nh = len(ha["desc"]) // 6
        self._check(
            self.lib.b3g_set_hulls(
                self.ctx, nh, N.ptr(ha["desc"], u32), N.ptr(ha["verts"], f32), N.ptr(ha["edges"], u32),
                N.ptr(ha["faces"], u32), N.ptr(ha["planes"], f32), N.ptr(ha["centroids"], f32),
            )
        )
        meshes = getattr(scene, "mesh_arrays", None)
        if meshes is not None:
            self._check(self.lib.b3g_set_meshes(
                self.ctx, len(meshes["desc"]) // 4, N.ptr(meshes["desc"], u32), N.ptr(meshes["verts"], f32),
                N.ptr(meshes["tris"], u32), int(meshes.get("max_pairs", 0))))
        awake = np.ones(scene.n_bodies, np.uint8)
        self._check(
            self.lib.b3g_set_bodies(
                self.ctx, scene.n_bodies, N.ptr(scene.body_world, u32), N.ptr(scene.body_type, u32),
                N.ptr(awake, ctypes.c_uint8),
            )
        )
        self._check(
            self.lib.b3g_set_fixtures(
                self.ctx, nf, N.ptr(scene.fix_body, u32), N.ptr(scene.fix_type, u32), N.ptr(scene.fix_hull, u32),
                N.ptr(scene.fix_params, f32), N.ptr(scene.fix_flags, u32), None,
            )
        )
        wings = getattr(scene, "tri_wings", None)
        if wings is not None and len(wings):
            fx = np.ascontiguousarray(scene.tri_fixtures, np.uint32)
            w = np.ascontiguousarray(wings, np.float32).reshape(-1)
            self._check(self.lib.b3g_set_triangle_wings(self.ctx, len(fx), N.ptr(fx, u32), N.ptr(w, f32)))

    def _check(self, rc):
        if rc < 0:
            msg = self.lib.b3g_last_error(self.ctx)
            raise N.B3GError(rc, msg.decode() if msg else "")
        return rc

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.b3g_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- pass -------------------------------------------------------------

    def set_awake(self, awake):
        a = np.ascontiguousarray(awake, np.uint8)
        self._check(self.lib.b3g_set_awake(self.ctx, N.ptr(a, ctypes.c_uint8)))

    def collide(self, state17, on_device=False, stream=None):
        """One collision pass. state17: host float32 array (17 per body) or,
        with on_device=True, a device pointer (int) to the same layout."""
        if on_device:
            p = ctypes.c_void_p(int(state17))
        else:
            assert state17.dtype == np.float32 and state17.flags["C_CONTIGUOUS"]
            p = ctypes.c_void_p(state17.ctypes.data)
        self._check(self.lib.b3g_collide(self.ctx, p, 1 if on_device else 0, ctypes.c_void_p(stream or 0)))

    # -- collision filters (b3g_set_joint_pairs and the contact filter) ------

    def set_joint_pairs(self, body_pairs):
        """Body pairs of the joints with collideConnected = false."""
        a = np.ascontiguousarray(body_pairs, np.uint32).reshape(-1)
        self._check(self.lib.b3g_set_joint_pairs(self.ctx, len(a) // 2, N.ptr(a, u32) if len(a) else None))

    def set_contact_veto(self, veto):
        """The contact filter's rejections of the last pass's contacts, in list order."""
        v = np.ascontiguousarray(veto, np.uint8)
        self._check(self.lib.b3g_set_contact_veto(self.ctx, len(v), N.ptr(v, ctypes.c_uint8) if len(v) else None))

    def new_pairs(self):
        """The new pairs the contact filter decides this pass (after collide
        with contact_filter=True), in AddPair order: (n, 2) fixtures."""
        n = self._check(self.lib.b3g_fetch_new_pairs(self.ctx, None, 0))
        out = np.zeros((max(n, 1), 2), np.uint32)
        n = self._check(self.lib.b3g_fetch_new_pairs(self.ctx, N.ptr(out, u32), n))
        return out[:n]

    def finish_pass(self, keep=None):
        """Rest of the pass with the filter's answers (None keeps every new pair)."""
        if keep is None:
            self._check(self.lib.b3g_finish_pass(self.ctx, None, 0))
        else:
            k = np.ascontiguousarray(keep, np.uint8)
            self._check(self.lib.b3g_finish_pass(self.ctx, N.ptr(k, ctypes.c_uint8) if len(k) else None, len(k)))

    def set_walk_limit(self, max_nodes):
        """Node visits allowed per broadphase walk (0: the depth-first bound)."""
        self._check(self.lib.b3g_set_walk_limit(self.ctx, int(max_nodes)))

    def set_tree_rebuild_interval(self, passes):
        """Passes between LBVH rebuilds (the tree is refit in between; 1
        rebuilds every pass). Results do not depend on it."""
        self._check(self.lib.b3g_set_tree_rebuild_interval(self.ctx, int(passes)))

    def counts(self):
        c = N.Counts()
        self._check(self.lib.b3g_get_counts(self.ctx, ctypes.byref(c)))
        return c.as_dict()

    STAT_NAMES = ("raw_pairs", "kept", "hull_miss", "trav_overflow", "mesh_items", "wake_events", "wake_activated",
                  "late_destroyed", "asleep")
    BUCKET_NAMES = ("spheres", "capsule_sphere", "capsules", "triangle_sphere", "triangle_capsule", "hull_sphere",
                    "hull_capsule", "hull_triangle", "hulls", "mesh", "sensor", "inactive", "apart")

    def pass_stats(self):
        """Inner counters of the last pass (b3g_get_pass_stats): named
        statistics plus a 'buckets' dict of narrowphase bucket sizes."""
        n = len(self.STAT_NAMES) + len(self.BUCKET_NAMES)
        out = np.zeros(n, np.uint32)
        k = self._check(self.lib.b3g_get_pass_stats(self.ctx, N.ptr(out, ctypes.c_uint32), n))
        assert k == n, k
        d = {name: int(out[i]) for i, name in enumerate(self.STAT_NAMES)}
        d["buckets"] = {name: int(out[len(self.STAT_NAMES) + i]) for i, name in enumerate(self.BUCKET_NAMES)}
        return d

    # -- results ----------------------------------------------------------

    def contacts(self):
        n = self.counts()["contacts"]
        out = np.zeros((max(n, 1), 3), np.uint32)
        m = self._check(self.lib.b3g_fetch_contacts(self.ctx, N.ptr(out, u32), n))
        return out[:m]

    def manifolds(self):
        n = self.counts()["contacts"]
        out = np.zeros(max(n, 1), N.MANIFOLD_DTYPE)
        m = self._check(self.lib.b3g_fetch_manifolds(self.ctx, ctypes.c_void_p(out.ctypes.data), n))
        return out[:m]

    def touching(self):
        n = self.counts()["manifolds"]
        idx = np.zeros(max(n, 1), np.uint32)
        man = np.zeros(max(n, 1), N.MANIFOLD_DTYPE)
        m = self._check(self.lib.b3g_fetch_touching(self.ctx, N.ptr(idx, u32), ctypes.c_void_p(man.ctypes.data), n))
        return idx[:m], man[:m]

    def fetch_results_async(self, contacts, index, manifolds):
        """Starts the copies of the last pass's contact records and touching
        output into the given host arrays ((C, 3) u32, (T,) u32, (T,)
        MANIFOLD_DTYPE); returns the pass counts. Read the arrays after
        wait_results()."""
        c = N.Counts()
        self._check(self.lib.b3g_fetch_results_async(
            self.ctx, ctypes.c_void_p(contacts.ctypes.data), len(contacts), ctypes.c_void_p(index.ctypes.data),
            ctypes.c_void_p(manifolds.ctypes.data), min(len(index), len(manifolds)), ctypes.byref(c)))
        return c.as_dict()

    def fetch_results_packed_async(self, contacts, index, packed):
        """As fetch_results_async with the touching output packed into the
        byte array `packed` (see unpack_manifolds)."""
        c = N.Counts()
        self._check(self.lib.b3g_fetch_results_packed_async(
            self.ctx, ctypes.c_void_p(contacts.ctypes.data), len(contacts), ctypes.c_void_p(index.ctypes.data),
            ctypes.c_void_p(packed.ctypes.data), len(index), packed.nbytes, ctypes.byref(c)))
        return c.as_dict()

    @staticmethod
    def unpack_manifolds(packed, count):
        """b3Manifold records (MANIFOLD_DTYPE) from `count` packed records;
        point slots past pointCount are zero."""
        out = np.zeros(count, N.MANIFOLD_DTYPE)
        raw = out.view(np.uint8).reshape(count, 320)
        src = np.asarray(packed).view(np.uint8).reshape(-1)
        off = 0
        for k in range(count):
            raw[k, 288:320] = src[off:off + 32]
            pc = int(src[off:off + 4].view(np.uint32)[0])
            raw[k, 0:72 * pc] = src[off + 32:off + 32 + 72 * pc]
            off += 32 + 72 * pc
        return out

    def wait_results(self):
        self._check(self.lib.b3g_wait_results(self.ctx))

    def fixture_contacts(self):
        """Island-graph edges: (offsets (nFixtures + 1,), contact indices) with
        fixture f's contacts in its edge-list order at offsets[f]:offsets[f + 1]."""
        n = self.counts()["contacts"]
        offsets = np.zeros(self.scene.n_fixtures + 1, np.uint32)
        out = np.zeros(max(2 * n, 1), np.uint32)
        m = self._check(self.lib.b3g_fetch_fixture_contacts(self.ctx, N.ptr(offsets, u32), N.ptr(out, u32), len(out)))
        return offsets, out[:m]

    def shape_cast(self, casts):
        """b3World::ShapeCast keeping every hit, per cast (SHAPE_CAST_DTYPE):
        (index (k, 3): cast, fixture, triangle; hits (k, 7): point, normal, fraction)."""
        c = np.ascontiguousarray(casts, N.SHAPE_CAST_DTYPE)
        cap = 64 * len(c) + 1024
        while True:
            idx = np.zeros((cap, 3), np.uint32)
            hits = np.zeros((cap, 7), np.float32)
            m = self._check(self.lib.b3g_shape_cast(self.ctx, len(c), ctypes.c_void_p(c.ctypes.data),
                                                    N.ptr(idx, u32), N.ptr(hits, ctypes.c_float), cap))
            if m <= cap:
                return idx[:m], hits[:m]
            cap = m

    def shape_cast_single(self, casts):
        """b3World::ShapeCastSingle per cast: (fixture and triangle (n, 2),
        0xFFFFFFFF when none; hit (n, 7): point, normal, fraction)."""
        c = np.ascontiguousarray(casts, N.SHAPE_CAST_DTYPE)
        fix = np.zeros((max(len(c), 1), 2), np.uint32)
        hit = np.zeros((max(len(c), 1), 7), np.float32)
        self._check(self.lib.b3g_shape_cast_single(self.ctx, len(c), ctypes.c_void_p(c.ctypes.data),
                                                   N.ptr(fix, u32), N.ptr(hit, ctypes.c_float)))
        return fix[:len(c)], hit[:len(c)]

    def time_of_impact(self, queries):
        """b3TimeOfImpact(b3TOIInput) per TOI_INPUT_DTYPE query: (n, 4) u32
        state, t bits, iterations, 0."""
        q = np.ascontiguousarray(queries, N.TOI_INPUT_DTYPE)
        out = np.zeros((max(len(q), 1), 4), np.uint32)
        self._check(self.lib.b3g_time_of_impact(self.ctx, len(q), ctypes.c_void_p(q.ctypes.data), N.ptr(out, u32)))
        return out[:len(q)]

    def time_of_impact_aabb(self, queries):
        """b3TimeOfImpact(aabb1, d1, aabb2, d2) per (18,) float query: (n, 4) u32."""
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, 18)
        out = np.zeros((max(len(q), 1), 4), np.uint32)
        self._check(self.lib.b3g_time_of_impact_aabb(self.ctx, len(q), N.ptr(q, ctypes.c_float), N.ptr(out, u32)))
        return out[:len(q)]

    def gjk_shape_cast(self, queries):
        """b3ShapeCast per GJK_CAST_DTYPE query: (n, 9) float32 words hit,
        t, point, normal, iterations."""
        q = np.ascontiguousarray(queries, N.GJK_CAST_DTYPE)
        out = np.zeros((max(len(q), 1), 9), np.float32)
        self._check(self.lib.b3g_gjk_shape_cast(self.ctx, len(q), ctypes.c_void_p(q.ctypes.data),
                                                N.ptr(out, ctypes.c_float)))
        return out[:len(q)]

    def set_materials(self, friction, restitution):
        """Friction and restitution per fixture (b3Fixture::m_friction, m_restitution)."""
        fr = np.ascontiguousarray(friction, np.float32)
        re = np.ascontiguousarray(restitution, np.float32)
        assert len(fr) == len(re) == self.scene.n_fixtures
        self._check(self.lib.b3g_set_materials(self.ctx, N.ptr(fr, ctypes.c_float), N.ptr(re, ctypes.c_float)))

    def contact_constraints(self, bodies, dt_ratio=1.0, warm=True, contacts=None):
        """b3ContactSolver's constructor + InitializeVelocityConstraints on the
        last pass: bodies is a SOLVER_BODY_DTYPE array (one per body);
        contacts the contact-list positions to solve, in order (None: every
        touching non-sensor contact in list order). Returns (constraints,
        manifolds) as CONTACT_CONSTRAINT_DTYPE / MANIFOLD_CONSTRAINT_DTYPE arrays."""
        b = np.ascontiguousarray(bodies, N.SOLVER_BODY_DTYPE)
        assert len(b) == self.n_bodies
        lst = None if contacts is None else np.ascontiguousarray(contacts, np.uint32)
        k = self.counts()["contacts"] if lst is None else len(lst)
        con = np.zeros(max(k, 1), N.CONTACT_CONSTRAINT_DTYPE)
        man = np.zeros(max(3 * k, 1), N.MANIFOLD_CONSTRAINT_DTYPE)
        counts = np.zeros(2, np.uint32)
        m = self._check(self.lib.b3g_contact_constraints(
            self.ctx, 0 if lst is None else len(lst), None if lst is None else N.ptr(lst, u32),
            ctypes.c_void_p(b.ctypes.data), float(dt_ratio), 1 if warm else 0, ctypes.c_void_p(con.ctypes.data),
            len(con), ctypes.c_void_p(man.ctypes.data), len(man), N.ptr(counts, u32)))
        return con[:m], man[:counts[1]]

    def ended(self):
        c = self.counts()
        out = np.zeros((max(c["ended"], 1), 3), np.uint32)
        m = self._check(self.lib.b3g_fetch_ended(self.ctx, N.ptr(out, u32), c["ended"]))
        return out[:m]

    def awake(self):
        """Awake flag per body after the last pass (its wake-ups applied)."""
        out = np.zeros(max(self.n_bodies, 1), np.uint8)
        self._check(self.lib.b3g_fetch_awake(self.ctx, N.ptr(out, ctypes.c_uint8), self.n_bodies))
        return out[: self.n_bodies]

    def caches(self):
        n = self.counts()["contacts"]
        out = np.zeros((max(n, 1), 4), np.uint32)
        m = self._check(self.lib.b3g_fetch_caches(self.ctx, N.ptr(out, u32), n))
        return out[:m]

    def fat_aabbs(self):
        nf = self.scene.n_fixtures
        out = np.zeros((nf, 6), np.float32)
        self._check(self.lib.b3g_fetch_fat_aabbs(self.ctx, N.ptr(out, f32), nf))
        return out

    def load_impulses(self, normal, tangent, motor):
        n = np.ascontiguousarray(normal, np.float32)
        t = np.ascontiguousarray(tangent, np.float32)
        m = np.ascontiguousarray(motor, np.float32)
        self._check(self.lib.b3g_load_impulses(self.ctx, N.ptr(n, f32), N.ptr(t, f32), N.ptr(m, f32)))

    # -- world queries (after a pass) --------------------------------------

    def query_aabb(self, boxes, worlds=None, capacity=None):
        """b3World::QueryAABB for each box (6 floats): (k, 2) u32 (query, fixture)."""
        b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
        w = None if worlds is None else np.ascontiguousarray(worlds, np.uint32)
        cap = capacity or max(1024, 64 * len(b))
        while True:
            out = np.zeros((cap, 2), np.uint32)
            k = self._check(self.lib.b3g_query_aabb(self.ctx, len(b), N.ptr(b, f32), N.ptr(w, u32), N.ptr(out, u32), cap))
            if k <= cap:
                return out[:k]
            cap = k

    def ray_cast(self, rays, worlds=None, capacity=None):
        """b3World::RayCast keeping every hit, for each ray (p1, p2):
        (k, 2) u32 (ray, fixture) and (k, 7) f32 (point, normal, fraction)."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        w = None if worlds is None else np.ascontiguousarray(worlds, np.uint32)
        cap = capacity or max(1024, 16 * len(r))
        while True:
            idx = np.zeros((cap, 2), np.uint32)
            hit = np.zeros((cap, 7), np.float32)
            k = self._check(self.lib.b3g_ray_cast(self.ctx, len(r), N.ptr(r, f32), N.ptr(w, u32), N.ptr(idx, u32),
                                                  N.ptr(hit, f32), cap))
            if k <= cap:
                return idx[:k], hit[:k]
            cap = k

    def ray_cast_single(self, rays, worlds=None):
        """b3World::RayCastSingle for each ray: fixture (0xFFFFFFFF: no hit)
        and (n, 7) f32 (point, normal, fraction)."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        w = None if worlds is None else np.ascontiguousarray(worlds, np.uint32)
        fix = np.zeros(max(len(r), 1), np.uint32)
        hit = np.zeros((max(len(r), 1), 7), np.float32)
        self._check(self.lib.b3g_ray_cast_single(self.ctx, len(r), N.ptr(r, f32), N.ptr(w, u32), N.ptr(fix, u32),
                                                 N.ptr(hit, f32)))
        return fix[:len(r)], hit[:len(r)]

    def load_mesh_impulses(self, normal, tangent, motor):
        """Impulses of manifolds 1 and 2 per contact: normal (n, 2, 4),
        tangent (n, 2, 2), motor (n, 2)."""
        n = np.ascontiguousarray(normal, np.float32)
        t = np.ascontiguousarray(tangent, np.float32)
        m = np.ascontiguousarray(motor, np.float32)
        self._check(self.lib.b3g_load_mesh_impulses(self.ctx, N.ptr(n, f32), N.ptr(t, f32), N.ptr(m, f32)))

    def totals(self, reset=False):
        """Cumulative device counters: passes, contacts, manifolds, points, begun, ended."""
        out = np.zeros(8, np.uint64)
        self._check(self.lib.b3g_get_totals(self.ctx, N.ptr(out, ctypes.c_uint64), 1 if reset else 0))
        names = ("passes", "contacts", "manifolds", "points", "begun", "ended", "launches", "graph_passes")
        return dict(zip(names, (int(x) for x in out)))

    def mesh_wings(self, m, n_triangles):
        out = np.zeros(3 * max(n_triangles, 1), np.uint32)
        k = self._check(self.lib.b3g_mesh_wings(self.ctx, m, N.ptr(out, u32), n_triangles))
        return out[: 3 * k].reshape(-1, 3)

    def autotune(self, reps=10, stream=None):
        """Times the tunable kernels on the last pass's data and keeps the
        fastest launch shapes; returns the tuning table."""
        out = np.zeros(N.TUNE_COUNT, np.uint32)
        s = ctypes.c_void_p(int(stream)) if stream else None
        self._check(self.lib.b3g_autotune(self.ctx, int(reps), s, N.ptr(out, u32)))
        return out

    def tuning(self):
        out = np.zeros(N.TUNE_COUNT, np.uint32)
        self._check(self.lib.b3g_get_tuning(self.ctx, N.ptr(out, u32)))
        return out

    def set_tuning(self, table):
        t = np.ascontiguousarray(table, np.uint32)
        assert t.size == N.TUNE_COUNT
        self._check(self.lib.b3g_set_tuning(self.ctx, N.ptr(t, u32)))

    def set_profiling(self, on=True):
        self._check(self.lib.b3g_set_profiling(self.ctx, 1 if on else 0))

    def profile(self):
        """Per-stage summed milliseconds and pass counts (CUDA events on the pass stream)."""
        ms = np.zeros(16, np.float64)
        cnt = np.zeros(16, np.uint32)
        n = self._check(self.lib.b3g_get_profile(self.ctx, N.ptr(ms, ctypes.c_double), N.ptr(cnt, u32), 16))
        return {self.lib.b3g_stage_name(k).decode(): (float(ms[k]), int(cnt[k])) for k in range(n)}

    def device_results(self):
        a, b = ctypes.c_void_p(), ctypes.c_void_p()
        self._check(self.lib.b3g_device_results(self.ctx, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def collide_pairs(self, fixA, fixB, xfA, xfB, xf0A=None, xf0B=None, cache=None):
        """Stand-alone narrowphase on explicit pairs and transforms (7 floats each)."""
        n = len(fixA)
        fa = np.ascontiguousarray(fixA, np.uint32)
        fb = np.ascontiguousarray(fixB, np.uint32)
        xa = np.ascontiguousarray(xfA, np.float32).reshape(-1)
        xb = np.ascontiguousarray(xfB, np.float32).reshape(-1)
        x0a = None if xf0A is None else np.ascontiguousarray(xf0A, np.float32).reshape(-1)
        x0b = None if xf0B is None else np.ascontiguousarray(xf0B, np.float32).reshape(-1)
        cc = None if cache is None else np.ascontiguousarray(cache, np.uint32).reshape(-1)
        out = np.zeros(max(n, 1), N.MANIFOLD_DTYPE)
        self._check(
            self.lib.b3g_collide_pairs(
                self.ctx, n, N.ptr(fa, u32), N.ptr(fb, u32), N.ptr(xa, f32), N.ptr(xb, f32), N.ptr(x0a, f32),
                N.ptr(x0b, f32), N.ptr(cc, u32), ctypes.c_void_p(out.ctypes.data),
            )
        )
        if cache is not None:
            cache[...] = cc.reshape(cache.shape)
        return out[:n]

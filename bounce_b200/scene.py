"""Seeded synthetic scenes for the collision pipeline and the kinematic driver
that moves their bodies between passes.

Scenes follow the workloads the pipeline is measured on:

* ``plain_scene``   1,000 unit boxes (half extent 0.5 m) + 1,000 spheres
  (r = 0.5 m), positions uniform in a 20 m cube above a static 100 x 1 x 100 m
  ground box, uniform random orientations.
* ``mixed_scene``   N mixed bodies: 40 % spheres r ~ U[0.2, 1], 30 % capsules
  r ~ U[0.1, 0.5], half-height ~ U[0.2, 1] (segment along local y), 30 % convex
  hulls of 8-32 points on ellipsoids with semi-axes ~ U[0.3, 1.2]; positions
  uniform in a cube of side L, linear velocities N(0, 1) m/s, angular N(0, 1) rad/s.
* ``batched_scene`` many independent worlds whose body counts are log-uniform
  in [16, 4096], each with the plain-scene shape mix.

All arithmetic that feeds the pipeline's inputs is float32 with the same
operation order as the reference's inline math (include/bounce/common/math/
quat.h:270-274, transform.h:66-69, body.h SynchronizeTransform), so transforms
computed here equal the ones b3Body would hold, bit for bit.
"""
import os

import numpy as np

from . import _native as N
from . import hull as H

F = np.float32

# Hull construction for scene input: the native builder in the CUDA library
# (fast) or its pure-Python restatement in hull.py (the same arrays bit for
# bit), for processes that must not map the CUDA library.
NATIVE_HULLS = True

# ---------------------------------------------------------------------------
# float32 vector helpers with the reference's operation order.


def _cross(a, b):
    return np.stack(
        [
            a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
            a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
            a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0],
        ],
        axis=-1,
    ).astype(F)


def quat_rotate(q, v):
    """b3Mul(quat, vec): v + s * t + qv x t with t = 2 (qv x v)."""
    qv = q[..., :3]
    s = q[..., 3:4]
    t = F(2) * _cross(qv, v)
    return ((v + s * t) + _cross(qv, t)).astype(F)


def xf_apply(p, q, v):
    """b3Mul(transform, vec)."""
    return (quat_rotate(q, v) + p).astype(F)


def quat_normalize(q):
    """b3Quat::Normalize: v scaled by 1/len, s divided by len."""
    v = q[..., :3]
    s = q[..., 3]
    l = np.sqrt(((v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1]) + v[..., 2] * v[..., 2]) + s * s).astype(F)
    ok = l > F(1.1920928955078125e-07)
    inv = np.where(ok, F(1) / np.where(ok, l, F(1)), F(1)).astype(F)
    out = q.copy()
    out[..., 0] = np.where(ok, v[..., 0] * inv, v[..., 0])
    out[..., 1] = np.where(ok, v[..., 1] * inv, v[..., 1])
    out[..., 2] = np.where(ok, v[..., 2] * inv, v[..., 2])
    out[..., 3] = np.where(ok, s / np.where(ok, l, F(1)), s)
    return out.astype(F)


def random_quats(rng, n):
    """Uniform random unit quaternions (Shoemake), x y z w."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    q = np.stack(
        [a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2), b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)],
        axis=-1,
    )
    return q.astype(F)


# ---------------------------------------------------------------------------
# Hull pool.


class HullPool:
    """Packed b3Hull arrays (include/b3g.h b3g_set_hulls layout)."""

    def __init__(self):
        self.desc, self.verts, self.edges, self.faces, self.planes, self.centroids = [], [], [], [], [], []
        self._nv = self._ne = self._nf = 0

    def _add(self, v, e, f, p, c, counts):
        nv, ne, nf = (int(x) for x in counts)
        self.desc.append([self._nv, nv, self._ne, ne, self._nf, nf])
        self.verts.append(v[: 3 * nv])
        self.edges.append(e[: 5 * ne])
        self.faces.append(f[:nf])
        self.planes.append(p[: 4 * nf])
        self.centroids.append(c)
        self._nv += nv
        self._ne += ne
        self._nf += nf
        return len(self.desc) - 1

    def add_points(self, pts):
        if not NATIVE_HULLS:
            try:
                v, e, f, p, c, counts = H.hull_from_points(pts)
            except ValueError:
                raise ValueError("degenerate hull point set") from None
            return self._add(v, e, f, p, c, counts)
        lib = N.load()
        pts = np.ascontiguousarray(pts, dtype=F)
        n = len(pts)
        v = np.zeros(3 * n, F)
        e = np.zeros(5 * (6 * n), np.uint32)
        f = np.zeros(2 * n, np.uint32)
        p = np.zeros(4 * 2 * n, F)
        c = np.zeros(3, F)
        counts = np.zeros(3, np.uint32)
        rc = lib.b3g_hull_from_points(
            N.ptr(pts, N.ctypes.c_float), n, N.ptr(v, N.ctypes.c_float), N.ptr(e, N.ctypes.c_uint32),
            N.ptr(f, N.ctypes.c_uint32), N.ptr(p, N.ctypes.c_float), N.ptr(c, N.ctypes.c_float),
            N.ptr(counts, N.ctypes.c_uint32),
        )
        if rc != 0:
            raise ValueError("degenerate hull point set")
        return self._add(v, e, f, p, c, counts)

    def add_box(self, ex, ey, ez):
        if not NATIVE_HULLS:
            return self._add(*H.hull_box(ex, ey, ez))
        lib = N.load()
        v = np.zeros(24, F)
        e = np.zeros(5 * 24, np.uint32)
        f = np.zeros(6, np.uint32)
        p = np.zeros(24, F)
        c = np.zeros(3, F)
        counts = np.zeros(3, np.uint32)
        lib.b3g_hull_box(
            F(ex), F(ey), F(ez), N.ptr(v, N.ctypes.c_float), N.ptr(e, N.ctypes.c_uint32), N.ptr(f, N.ctypes.c_uint32),
            N.ptr(p, N.ctypes.c_float), N.ptr(c, N.ctypes.c_float), N.ptr(counts, N.ctypes.c_uint32),
        )
        return self._add(v, e, f, p, c, counts)

    def extend(self, arrays):
        """Append packed hulls (the arrays() layout of another pool); returns
        the index of the first."""
        first = len(self.desc)
        d = np.asarray(arrays["desc"], np.int64).reshape(-1, 6)
        for k in range(len(d)):
            v0, nv, e0, ne, f0, nf = (int(x) for x in d[k])
            self._add(arrays["verts"][3 * v0:3 * (v0 + nv)], arrays["edges"][5 * e0:5 * (e0 + ne)],
                      arrays["faces"][f0:f0 + nf], arrays["planes"][4 * f0:4 * (f0 + nf)],
                      arrays["centroids"][3 * k:3 * k + 3], (nv, ne, nf))
        return first

    def arrays(self):
        cat = lambda xs, dt: np.ascontiguousarray(np.concatenate(xs) if xs else np.zeros(0, dt), dtype=dt)
        return dict(
            desc=np.ascontiguousarray(np.array(self.desc, np.uint32).reshape(-1)),
            verts=cat(self.verts, F),
            edges=cat(self.edges, np.uint32),
            faces=cat(self.faces, np.uint32),
            planes=cat(self.planes, F),
            centroids=np.ascontiguousarray(np.array(self.centroids, F).reshape(-1)),
        )

    def __len__(self):
        return len(self.desc)


# ---------------------------------------------------------------------------
# Scenes.


class Scene:
    """Bodies (one fixture each here, the API allows several), fixtures and hulls."""

    def __init__(self):
        self.hulls = HullPool()
        self.body_world, self.body_type, self.body_pos, self.body_quat = [], [], [], []
        self.body_lin, self.body_ang = [], []
        self.fix_body, self.fix_type, self.fix_hull, self.fix_params, self.fix_flags = [], [], [], [], []
        self.hull_centroid_of = {}

    def add_body(self, world, btype, pos, quat, lin=(0, 0, 0), ang=(0, 0, 0)):
        self.body_world.append(world)
        self.body_type.append(btype)
        self.body_pos.append(pos)
        self.body_quat.append(quat)
        self.body_lin.append(lin)
        self.body_ang.append(ang)
        return len(self.body_world) - 1

    def add_fixture(self, body, stype, params, hull=0, flags=0):
        p = np.zeros(12, F)
        p[: len(params)] = params
        self.fix_body.append(body)
        self.fix_type.append(stype)
        self.fix_hull.append(hull)
        self.fix_params.append(p)
        self.fix_flags.append(flags)
        return len(self.fix_body) - 1

    def finalize(self, hull_arrays=None):
        """Pack the lists into arrays. hull_arrays: prebuilt b3g_set_hulls
        arrays to use instead of this scene's HullPool."""
        self.hull_arrays = hull_arrays if hull_arrays is not None else self.hulls.arrays()
        self.body_world = np.ascontiguousarray(self.body_world, np.uint32)
        self.body_type = np.ascontiguousarray(self.body_type, np.uint32)
        self.body_pos = np.ascontiguousarray(np.array(self.body_pos, F).reshape(-1, 3))
        self.body_quat = np.ascontiguousarray(np.array(self.body_quat, F).reshape(-1, 4))
        self.body_lin = np.ascontiguousarray(np.array(self.body_lin, F).reshape(-1, 3))
        self.body_ang = np.ascontiguousarray(np.array(self.body_ang, F).reshape(-1, 3))
        self.fix_body = np.ascontiguousarray(self.fix_body, np.uint32)
        self.fix_type = np.ascontiguousarray(self.fix_type, np.uint32)
        self.fix_hull = np.ascontiguousarray(self.fix_hull, np.uint32)
        self.fix_params = np.ascontiguousarray(np.array(self.fix_params, F).reshape(-1))
        self.fix_flags = np.ascontiguousarray(self.fix_flags, np.uint32)
        self.body_pose = np.ascontiguousarray(np.concatenate([self.body_pos, self.body_quat], axis=1))
        self.local_center = self._local_centers()
        return self

    @property
    def n_bodies(self):
        return len(self.body_world)

    @property
    def n_fixtures(self):
        return len(self.fix_body)

    @property
    def n_worlds(self):
        return int(self.body_world.max()) + 1 if self.n_bodies else 0

    def _local_centers(self):
        """Body centre of mass in body frame for single-fixture dynamic bodies:
        the shape's centroid (sphere centre, capsule midpoint, hull volume
        centroid); zero for static and kinematic bodies (body.cpp:265-281)."""
        lc = np.zeros((self.n_bodies, 3), F)
        params = self.fix_params.reshape(-1, 12)
        cents = self.hull_arrays["centroids"].reshape(-1, 3)
        for f in range(self.n_fixtures):
            b = self.fix_body[f]
            if self.body_type[b] != N.BODY_DYNAMIC:
                continue
            t = self.fix_type[f]
            if t == N.SHAPE_SPHERE:
                lc[b] = params[f, 0:3]
            elif t == N.SHAPE_CAPSULE:
                lc[b] = F(0.5) * (params[f, 0:3] + params[f, 3:6])
            elif t == N.SHAPE_HULL:
                lc[b] = cents[self.fix_hull[f]]
        return lc

    def set_local_centers(self, lc):
        self.local_center = np.ascontiguousarray(lc, F).reshape(-1, 3)

    def world_subset(self, w):
        """The bodies and fixtures of world w as a one-world scene (world 0,
        same hull arrays), with the indices they had here: returns
        (scene, body indices, fixture indices)."""
        bodies = np.nonzero(self.body_world == w)[0]
        fixtures = np.nonzero(self.body_world[self.fix_body] == w)[0]
        remap = np.full(self.n_bodies, -1, np.int64)
        remap[bodies] = np.arange(len(bodies))
        s = Scene()
        s.hull_arrays = self.hull_arrays
        s.body_world = np.zeros(len(bodies), np.uint32)
        s.body_type = np.ascontiguousarray(self.body_type[bodies])
        s.body_pos = np.ascontiguousarray(self.body_pos[bodies])
        s.body_quat = np.ascontiguousarray(self.body_quat[bodies])
        s.body_lin = np.ascontiguousarray(self.body_lin[bodies])
        s.body_ang = np.ascontiguousarray(self.body_ang[bodies])
        s.body_pose = np.ascontiguousarray(self.body_pose[bodies])
        s.fix_body = np.ascontiguousarray(remap[self.fix_body[fixtures]].astype(np.uint32))
        s.fix_type = np.ascontiguousarray(self.fix_type[fixtures])
        s.fix_hull = np.ascontiguousarray(self.fix_hull[fixtures])
        s.fix_params = np.ascontiguousarray(self.fix_params.reshape(-1, 12)[fixtures].reshape(-1))
        s.fix_flags = np.ascontiguousarray(self.fix_flags[fixtures])
        s.local_center = np.ascontiguousarray(self.local_center[bodies])
        return s, bodies, fixtures


def plain_scene(seed=1, n_boxes=1000, n_spheres=1000, cube=20.0, world=0, scene=None, box_hull=None,
                ground_hull=None):
    """Boxes and spheres above a static ground box."""
    rng = np.random.default_rng(seed)
    s = scene if scene is not None else Scene()
    if box_hull is None:
        box_hull = s.hulls.add_box(0.5, 0.5, 0.5)
    if ground_hull is None:
        ground_hull = s.hulls.add_box(50.0, 0.5, 50.0)
    g = s.add_body(world, N.BODY_STATIC, (0, -0.5, 0), (0, 0, 0, 1))
    s.add_fixture(g, N.SHAPE_HULL, [0.0], hull=ground_hull)
    n = n_boxes + n_spheres
    half = cube / 2
    pos = np.stack(
        [rng.uniform(-half, half, n), rng.uniform(0.5, 0.5 + cube, n), rng.uniform(-half, half, n)], axis=-1
    ).astype(F)
    quat = random_quats(rng, n)
    lin = rng.normal(0, 1, (n, 3)).astype(F)
    ang = rng.normal(0, 1, (n, 3)).astype(F)
    for i in range(n):
        b = s.add_body(world, N.BODY_DYNAMIC, pos[i], quat[i], lin[i], ang[i])
        if i < n_boxes:
            s.add_fixture(b, N.SHAPE_HULL, [0.0], hull=box_hull)
        else:
            s.add_fixture(b, N.SHAPE_SPHERE, [0, 0, 0, 0.5])
    return s


def ellipsoid_points(rng, n, axes):
    d = rng.normal(0, 1, (n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return (d * axes).astype(F)


def mixed_scene(seed=2, n=65536, side=49.0, hull_pts=(8, 32), hull_axes=(0.3, 1.2), world=0, scene=None,
                static_frac=0.0, sensor_frac=0.0):
    """Mixed spheres / capsules / hulls in a cube, all dynamic unless
    static_frac / sensor_frac turn that fraction of the bodies static / of the
    fixtures into sensors (drawn from a second generator, so the other draws
    do not change)."""
    rng = np.random.default_rng(seed)
    s = scene if scene is not None else Scene()
    b0, f0 = len(s.body_type), len(s.fix_type)
    kind = rng.random(n)
    pos = rng.uniform(-side / 2, side / 2, (n, 3)).astype(F)
    quat = random_quats(rng, n)
    lin = rng.normal(0, 1, (n, 3)).astype(F)
    ang = rng.normal(0, 1, (n, 3)).astype(F)
    for i in range(n):
        b = s.add_body(world, N.BODY_DYNAMIC, pos[i], quat[i], lin[i], ang[i])
        k = kind[i]
        if k < 0.4:
            s.add_fixture(b, N.SHAPE_SPHERE, [0, 0, 0, rng.uniform(0.2, 1.0)])
        elif k < 0.7:
            r = rng.uniform(0.1, 0.5)
            h = rng.uniform(0.2, 1.0)
            s.add_fixture(b, N.SHAPE_CAPSULE, [0, -h, 0, 0, h, 0, r])
        else:
            while True:
                m = int(rng.integers(hull_pts[0], hull_pts[1] + 1))
                axes = rng.uniform(hull_axes[0], hull_axes[1], 3)
                try:
                    h = s.hulls.add_points(ellipsoid_points(rng, m, axes))
                    break
                except ValueError:
                    continue
            s.add_fixture(b, N.SHAPE_HULL, [0.0], hull=h)
    if static_frac > 0 or sensor_frac > 0:
        rng2 = np.random.default_rng(seed + 0x5EED)
        for i in np.nonzero(rng2.random(n) < static_frac)[0]:
            s.body_type[b0 + i] = N.BODY_STATIC
            s.body_lin[b0 + i] = np.zeros(3, F)
            s.body_ang[b0 + i] = np.zeros(3, F)
        for i in np.nonzero(rng2.random(n) < sensor_frac)[0]:
            s.fix_flags[f0 + i] = N.FIXTURE_SENSOR
    return s


def batched_scene(seed=3, n_worlds=1024, lo=16, hi=4096, cube=20.0):
    """Independent worlds, body counts log-uniform in [lo, hi], plain-scene mix
    (boxes and spheres in equal numbers above a ground box per world)."""
    rng = np.random.default_rng(seed)
    s = Scene()
    box = s.hulls.add_box(0.5, 0.5, 0.5)
    counts = np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), n_worlds))).astype(int)
    for w in range(n_worlds):
        nb = int(counts[w])
        # Keep the body density of the plain scene: cube volume scales with nb.
        side = cube * (nb / 2000.0) ** (1.0 / 3.0)
        plain_scene(seed=int(rng.integers(1 << 31)), n_boxes=nb // 2, n_spheres=nb - nb // 2, cube=max(side, 4.0),
                    world=w, scene=s, box_hull=box)
    return s, counts


# ---------------------------------------------------------------------------
# Kinematic driver.


class KinematicDriver:
    """Moves bodies with constant velocities between passes and produces the
    per-pass body state (include/b3g.h b3g_collide layout, 17 floats per body)
    and the sweep input of the reference driver (14 floats per body).

    Per pass k the sweep start is the previous pose and the sweep end the new
    one: c_k = c_{k-1} + dt v, q_k = normalize(q_{k-1} + dt/2 (w, 0) q_{k-1})."""

    def __init__(self, scene, dt=1.0 / 60.0, walls=None):
        """walls: half-size of an axis-aligned box whose faces reflect the
        centre-of-mass velocity, keeping the body density constant over long
        runs (None: free motion)."""
        self.s = scene
        self.dt = F(dt)
        self.walls = None if walls is None else F(walls)
        self.lin = scene.body_lin.copy()
        self.lc = scene.local_center
        p, q = scene.body_pos, scene.body_quat
        # b3Body::ResetMass: worldCenter = xf * localCenter (body.cpp).
        self.c = xf_apply(p, q, self.lc)
        self.q = q.copy()
        self.c0 = self.c.copy()
        self.q0 = self.q.copy()
        self.p = p.copy()
        self.moving = scene.body_type != N.BODY_STATIC
        self.step_index = 0

    def advance(self, mask=None):
        """Move one step (static bodies stay; with a mask, only the bodies it
        flags move, the others keep their sweep as a sleeping body does)."""
        dt = self.dt
        m = self.moving if mask is None else (self.moving & (np.asarray(mask) != 0))
        if self.walls is not None:
            out_hi = (self.c > self.walls) & (self.lin > 0)
            out_lo = (self.c < -self.walls) & (self.lin < 0)
            self.lin = np.where(out_hi | out_lo, -self.lin, self.lin).astype(F)
        c1 = (self.c + dt * self.lin).astype(F)
        w = self.s.body_ang
        q = self.q
        # qdot = 0.5 * (w, 0) * q  (quat.h b3Derivative / b3Integrate)
        wv = w
        qv, qs = q[:, :3], q[:, 3:4]
        dv = (_cross(wv, qv) + qs * wv).astype(F)  # w x qv + qs w (0 * qv term vanishes)
        ds = (-(wv * qv).sum(axis=1, keepdims=True)).astype(F)
        qd = np.concatenate([F(0.5) * dv, F(0.5) * ds], axis=1).astype(F)
        q1 = quat_normalize((q + dt * qd).astype(F))
        self.c0 = np.where(m[:, None], self.c, self.c0).astype(F)
        self.q0 = np.where(m[:, None], self.q, self.q0).astype(F)
        self.c = np.where(m[:, None], c1, self.c).astype(F)
        self.q = np.where(m[:, None], q1, self.q).astype(F)
        # b3Body::SynchronizeTransform: xf.p = worldCenter - R(q) localCenter.
        self.p = np.where(m[:, None], (self.c - quat_rotate(self.q, self.lc)).astype(F), self.p).astype(F)
        self.step_index += 1

    def state17(self):
        """Per-body pipeline input: xf (p, q), sweep worldCenter0, orientation0, localCenter."""
        out = np.empty((self.s.n_bodies, 17), F)
        out[:, 0:3] = self.p
        out[:, 3:7] = self.q
        out[:, 7:10] = self.c0
        out[:, 10:14] = self.q0
        out[:, 14:17] = self.lc
        return np.ascontiguousarray(out.reshape(-1))

    def sweeps14(self):
        """Reference driver input: worldCenter0, orientation0, worldCenter, orientation."""
        out = np.empty((self.s.n_bodies, 14), F)
        out[:, 0:3] = self.c0
        out[:, 3:7] = self.q0
        out[:, 7:10] = self.c
        out[:, 10:14] = self.q
        return np.ascontiguousarray(out.reshape(-1))


def grid_mesh(nx, nz, spacing, seed, amplitude=0.5):
    """Vertices (nx * nz, 3) and triangles (2 per cell, counter-clockwise seen
    from +y) of a height field: heights are a seeded sum of sines."""
    rng = np.random.default_rng(seed)
    xs = (np.arange(nx) - (nx - 1) / 2.0) * spacing
    zs = (np.arange(nz) - (nz - 1) / 2.0) * spacing
    ph = rng.uniform(0, 2 * np.pi, 4)
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    Y = amplitude * (np.sin(0.7 * X + ph[0]) * np.sin(0.5 * Z + ph[1]) + 0.5 * np.sin(1.3 * X + ph[2]) * np.sin(0.9 * Z + ph[3]))
    V = np.stack([X, Y, Z], axis=-1).astype(F).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(nz - 1), indexing="ij")
    a, b, c, d = i * nz + j, (i + 1) * nz + j, (i + 1) * nz + j + 1, i * nz + j + 1
    tris = np.stack([np.stack([a, d, c], -1), np.stack([a, c, b], -1)], axis=2).reshape(-1, 3)
    return V, tris.astype(np.int64)


def terrain_triangles(nx, nz, spacing, seed, amplitude=0.5):
    """Triangles of a height-field grid of nx x nz vertices (two per cell) and
    the edge wings of each (the third vertex of the triangle across each
    edge, as b3Mesh adjacency gives them): returns (params (n, 12), wings (n, 12))."""
    V, tris = grid_mesh(nx, nz, spacing, seed, amplitude)
    edge_owner = {}
    for t, (a, b, c) in enumerate(tris):
        for k, (u, v) in enumerate(((a, b), (b, c), (c, a))):
            edge_owner.setdefault((min(u, v), max(u, v)), []).append((t, k))
    params = np.zeros((len(tris), 12), F)
    wings = np.zeros((len(tris), 12), F)
    for t, (a, b, c) in enumerate(tris):
        params[t, 0:3], params[t, 3:6], params[t, 6:9] = V[a], V[b], V[c]
        for k, (u, v) in enumerate(((a, b), (b, c), (c, a))):
            for (t2, _) in edge_owner[(min(u, v), max(u, v))]:
                if t2 != t:
                    third = [x for x in tris[t2] if x != u and x != v][0]
                    wings[t, 3 * k:3 * k + 3] = V[third]
                    wings[t, 9 + k] = 1.0
    return params, wings


def terrain_scene(seed=3, n=800, grid=12, spacing=1.5, height=4.0, static_frac=0.0):
    """Mixed moving bodies (spheres, capsules, hulls) above a static terrain of
    triangle fixtures with edge wings (scene.tri_wings: fixture -> 12 floats)."""
    rng = np.random.default_rng(seed)
    s = Scene()
    g = s.add_body(0, N.BODY_STATIC, (0, 0, 0), (0, 0, 0, 1))
    params, wings = terrain_triangles(grid, grid, spacing, seed)
    first = len(s.fix_type)
    for p in params:
        s.add_fixture(g, N.SHAPE_TRIANGLE, list(p[:9]) + [0.0])
    half = 0.5 * spacing * (grid - 1)
    pos = np.stack([rng.uniform(-half, half, n), rng.uniform(-0.5, height, n), rng.uniform(-half, half, n)],
                   axis=-1).astype(F)
    quat = random_quats(rng, n)
    lin = rng.normal(0, 1, (n, 3)).astype(F)
    lin[:, 1] -= 1.0
    ang = rng.normal(0, 1, (n, 3)).astype(F)
    for i in range(n):
        b = s.add_body(0, N.BODY_DYNAMIC, pos[i], quat[i], lin[i], ang[i])
        k = rng.random()
        if k < 0.35:
            s.add_fixture(b, N.SHAPE_SPHERE, [0, 0, 0, rng.uniform(0.2, 0.6)])
        elif k < 0.65:
            r = rng.uniform(0.1, 0.4)
            h = rng.uniform(0.2, 0.7)
            s.add_fixture(b, N.SHAPE_CAPSULE, [0, -h, 0, 0, h, 0, r])
        else:
            while True:
                m = int(rng.integers(8, 20))
                axes = rng.uniform(0.3, 0.8, 3)
                try:
                    hh = s.hulls.add_points(ellipsoid_points(rng, m, axes))
                    break
                except ValueError:
                    continue
            s.add_fixture(b, N.SHAPE_HULL, [0.0], hull=hh)
    s.tri_fixtures = np.arange(first, first + len(params), dtype=np.uint32)
    s.tri_wings = wings
    return s


def mesh_terrain_scene(seed=5, n=800, grid=14, spacing=1.5, height=4.0, scale=(1.0, 1.0, 1.0)):
    """Mixed moving bodies above a static triangle-mesh terrain (one mesh
    fixture; scene.mesh_arrays holds the mesh)."""
    rng = np.random.default_rng(seed)
    s = Scene()
    V, tris = grid_mesh(grid, grid, spacing, seed)
    s.mesh_arrays = dict(desc=np.array([0, len(V), 0, len(tris)], np.uint32),
                         verts=np.ascontiguousarray(V.reshape(-1), F),
                         tris=np.ascontiguousarray(tris.reshape(-1), np.uint32))
    g = s.add_body(0, N.BODY_STATIC, (0, 0, 0), (0, 0, 0, 1))
    s.add_fixture(g, N.SHAPE_MESH, [scale[0], scale[1], scale[2], 0.0], hull=0)
    half = 0.5 * spacing * (grid - 1) * min(scale[0], scale[2])
    pos = np.stack([rng.uniform(-half, half, n), rng.uniform(-0.5, height, n), rng.uniform(-half, half, n)],
                   axis=-1).astype(F)
    quat = random_quats(rng, n)
    lin = rng.normal(0, 1, (n, 3)).astype(F)
    lin[:, 1] -= 1.0
    ang = rng.normal(0, 1, (n, 3)).astype(F)
    for i in range(n):
        b = s.add_body(0, N.BODY_DYNAMIC, pos[i], quat[i], lin[i], ang[i])
        k = rng.random()
        if k < 0.35:
            s.add_fixture(b, N.SHAPE_SPHERE, [0, 0, 0, rng.uniform(0.2, 0.6)])
        elif k < 0.65:
            r = rng.uniform(0.1, 0.4)
            h = rng.uniform(0.2, 0.7)
            s.add_fixture(b, N.SHAPE_CAPSULE, [0, -h, 0, 0, h, 0, r])
        else:
            while True:
                m = int(rng.integers(8, 20))
                axes = rng.uniform(0.3, 0.8, 3)
                try:
                    hh = s.hulls.add_points(ellipsoid_points(rng, m, axes))
                    break
                except ValueError:
                    continue
            s.add_fixture(b, N.SHAPE_HULL, [0.0], hull=hh)
    return s


# ---------------------------------------------------------------------------
# Hull-heavy pile over a mesh ground.


def sines_heights(X, Z, seed, amplitude=2.0):
    """Heights sum_k a_k sin(f_k x + p_k) sin(g_k z + q_k) over 4 seeded
    terms whose amplitudes a_k add up to `amplitude` (wavelengths 12-60 m)."""
    rng = np.random.default_rng(seed)
    h = np.zeros(np.broadcast(X, Z).shape, dtype=np.float64)
    for _ in range(4):
        f, g = 2 * np.pi / rng.uniform(12.0, 60.0, 2)
        p, q = rng.uniform(0, 2 * np.pi, 2)
        h += (amplitude / 4.0) * np.sin(f * X + p) * np.sin(g * Z + q)
    return h


def sines_mesh(n, spacing, seed, amplitude=2.0):
    """An n x n vertex grid mesh (2 triangles per cell, counter-clockwise from
    +y) with sines_heights: returns (vertices (n*n, 3), triangles)."""
    xs = (np.arange(n) - (n - 1) / 2.0) * spacing
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    V = np.stack([X, sines_heights(X, Z, seed, amplitude), Z], axis=-1).astype(F).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    a, b, c, d = i * n + j, (i + 1) * n + j, (i + 1) * n + j + 1, i * n + j + 1
    tris = np.stack([np.stack([a, d, c], -1), np.stack([a, c, b], -1)], axis=2).reshape(-1, 3)
    return V, tris.astype(np.int64)


def _pile_hull_chunk(job):
    """Worker: quickhulls of m ~ U{lo..hi} points on ellipsoids with
    semi-axes ~ U[alo, ahi] (seeded per chunk); returns packed arrays."""
    seed, count, pts, axes = job
    rng = np.random.default_rng(seed)
    pool = HullPool()
    while len(pool) < count:
        m = int(rng.integers(pts[0], pts[1] + 1))
        ax = rng.uniform(axes[0], axes[1], 3)
        try:
            pool.add_points(ellipsoid_points(rng, m, ax))
        except ValueError:
            continue
    return pool.arrays()


def _padded_hulls(desc, verts, planes, idx, quats, vmax, fmax):
    """Rotated vertices (m, vmax, 3) and planes (m, fmax, 4) of hulls idx
    (float64), padding masked out: padded vertices repeat vertex 0 and padded
    planes are (0, 0, 0, +inf), which never bind."""
    m = len(idx)
    W = np.empty((m, vmax, 3))
    P = np.zeros((m, fmax, 4))
    P[:, :, 3] = np.inf
    for r, k in enumerate(idx):
        v0, nv, f0, nf = int(desc[k, 0]), int(desc[k, 1]), int(desc[k, 4]), int(desc[k, 5])
        W[r, :nv] = verts[v0:v0 + nv]
        W[r, nv:] = verts[v0]
        P[r, :nf] = planes[f0:f0 + nf]
    q = quats[idx][:, None, :]
    W = quat_rotate(np.broadcast_to(q, (m, vmax, 4)).astype(F), W.astype(F)).astype(np.float64)
    P[:, :, :3] = quat_rotate(np.broadcast_to(q, (m, fmax, 4)).astype(F), P[:, :, :3].astype(F))
    return W, P


def _profile(P, dy, X, Z):
    """Vertical lines at (X, Z) (m, k) through hulls with planes P (m, f, 4)
    lifted by dy (m): bottom, top (m, k) and whether each line hits."""
    n = P[:, None, :, :3]
    off = (P[:, None, :, 3] + P[:, None, :, 1] * dy[:, None, None]) - (X[:, :, None] * n[..., 0] + Z[:, :, None] * n[..., 2])
    ny = np.broadcast_to(n[..., 1], off.shape)
    up, down = ny > 1e-6, ny < -1e-6
    side = ~(up | down)
    with np.errstate(invalid="ignore", divide="ignore"):
        ratio = off / np.where(up | down, ny, 1.0)
    top = np.min(np.where(up, ratio, np.inf), axis=2)
    bot = np.max(np.where(down, ratio, -np.inf), axis=2)
    hit = (bot <= top) & np.all(~side | (off >= -1e-9), axis=2)
    return bot, top, hit


def _clearances(Wl, Pl, yl, Wu, Pu, yu):
    """Vertical clearance between lower hulls (Wl, Pl at heights yl) and the
    upper hulls above them (Wu, Pu at yu), from each hull's vertices against
    the other's surface; +inf where no vertex lies over the other hull."""
    _, top, hit = _profile(Pl, yl, Wu[..., 0], Wu[..., 2])
    c1 = np.min(np.where(hit, (Wu[..., 1] + yu[:, None]) - top, np.inf), axis=1)
    bot, _, hit = _profile(Pu, yu, Wl[..., 0], Wl[..., 2])
    c2 = np.min(np.where(hit, bot - (Wl[..., 1] + yl[:, None]), np.inf), axis=1)
    return np.minimum(c1, c2)


def _pile_columns(job):
    """Worker: builds the hulls of a chunk of columns (seeded per chunk) and
    stacks them level by level; returns (packed hull arrays, heights
    (columns, per_column))."""
    global NATIVE_HULLS
    hull_seed, per_column, cx, cz, quats, gap, seed, amplitude, pts, axes, native = job
    NATIVE_HULLS = native
    m = len(cx)
    arrays = _pile_hull_chunk((hull_seed, m * per_column, pts, axes))
    desc = arrays["desc"].reshape(-1, 6)
    verts = arrays["verts"].reshape(-1, 3)
    planes = arrays["planes"].reshape(-1, 4).astype(np.float64)
    vmax, fmax = int(desc[:, 1].max()), int(desc[:, 5].max())
    ys = np.empty((m, per_column))
    below = None
    for lv in range(per_column):
        idx = np.arange(m) * per_column + lv
        W, P = _padded_hulls(desc, verts, planes, idx, quats, vmax, fmax)
        if below is None:
            # the lowest vertex clears the terrain below it by `gap`
            gh = sines_heights(cx[:, None] + W[..., 0], cz[:, None] + W[..., 2], seed, amplitude)
            y = np.max(gh - W[..., 1], axis=1) + gap
        else:
            # first above the lower hull's highest vertex, then lowered until
            # the hulls are `gap` apart along the vertical
            Wl, Pl, yl = below
            y = yl + Wl[..., 1].max(axis=1) + gap - W[..., 1].min(axis=1)
            cl = _clearances(Wl, Pl, yl, W, P, y)
            y = np.where(np.isfinite(cl) & (cl > gap), y - (cl - gap), y)
        ys[:, lv] = y
        below = (W, P, y)
    return arrays, ys


def pile_scene(seed=9, columns=512, per_column=512, grid=512, spacing=0.5, amplitude=2.0, gap=1e-3,
               column_pitch=7.5, settle=0.03, jitter=0.01, spin=0.05, pts=(12, 64), axes=(0.3, 1.0),
               chunk_columns=8, workers=None):
    """Hull-heavy dense pile: columns x per_column distinct convex hulls
    (quickhulls of 12-64 points on ellipsoids, semi-axes U[0.3, 1.0] m,
    random orientation) stacked in vertical columns with `gap` m of vertical
    clearance between neighbours, over a static mesh ground (a grid x grid
    vertex sines terrain at `spacing` m). Hull building and stacking run in
    spawned workers, chunk_columns columns each; the scene depends on the
    chunk size, not on the worker count.

    Motion: the pile settles. The hull at level i of its column moves down at
    settle * i m/s (neighbours close at `settle` m/s, so the gaps close within
    the first passes and the stack then stays in contact), plus N(0, jitter)
    m/s and N(0, spin) rad/s."""
    import multiprocessing as mp

    rng = np.random.default_rng(seed)
    n = columns * per_column
    s = Scene()
    V, T = sines_mesh(grid, spacing, seed, amplitude)
    s.mesh_arrays = dict(desc=np.array([0, len(V), 0, len(T)], np.uint32),
                         verts=np.ascontiguousarray(V.reshape(-1), F),
                         tris=np.ascontiguousarray(T.reshape(-1), np.uint32))
    g = s.add_body(0, N.BODY_STATIC, (0, 0, 0), (0, 0, 0, 1))
    s.add_fixture(g, N.SHAPE_MESH, [1.0, 1.0, 1.0, 0.0], hull=0)
    cols = int(np.ceil(np.sqrt(columns / 2.0)))
    rows = (columns + cols - 1) // cols
    quats = random_quats(rng, n)
    lin = rng.normal(0, jitter, (n, 3))
    lin[:, 1] -= settle * np.tile(np.arange(per_column), columns)
    lin = lin.astype(F)
    ang = rng.normal(0, spin, (n, 3)).astype(F)
    ci = np.arange(columns)
    cx = (ci % cols - (cols - 1) / 2.0) * column_pitch
    cz = (ci // cols - (rows - 1) / 2.0) * column_pitch
    jobs = []
    for j, c0 in enumerate(range(0, columns, chunk_columns)):
        c1 = min(columns, c0 + chunk_columns)
        jobs.append((seed * 100003 + j, per_column, cx[c0:c1], cz[c0:c1],
                     quats[c0 * per_column:c1 * per_column], gap, seed, amplitude, pts, axes, NATIVE_HULLS))
    workers = workers or min(len(jobs), os.cpu_count() or 1)
    if workers <= 1:
        parts = [_pile_columns(jb) for jb in jobs]
    else:
        with mp.get_context("spawn").Pool(workers) as p:
            parts = p.map(_pile_columns, jobs)
    ys = np.concatenate([y for _, y in parts])
    for arrays, _ in parts:
        s.hulls.extend(arrays)
    for c in range(columns):
        for lv in range(per_column):
            k = c * per_column + lv
            b = s.add_body(0, N.BODY_DYNAMIC, (cx[c], ys[c, lv], cz[c]), quats[k], lin[k], ang[k])
            s.add_fixture(b, N.SHAPE_HULL, [0.0], hull=k)
    return s


# ---------------------------------------------------------------------------
# Queries of the time-of-impact entry points.


def unit_quats(rng, n):
    """n uniform random unit quaternions (xyzw)."""
    q = rng.normal(size=(n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def qmul(a, b):
    """Quaternion products of (n, 4) xyzw arrays."""
    av, aw = a[:, :3], a[:, 3:]
    bv, bw = b[:, :3], b[:, 3:]
    v = np.cross(av, bv) + aw * bv + bw * av
    w = aw * bw - np.sum(av * bv, axis=1, keepdims=True)
    return np.concatenate([v, w], axis=1)


def random_convex_shapes(rng, n, n_hulls):
    """Types and params of random convex shapes (hull indices into the pool)."""
    types = rng.choice([N.SHAPE_SPHERE, N.SHAPE_CAPSULE, N.SHAPE_TRIANGLE, N.SHAPE_HULL], n, p=[0.25, 0.25, 0.15, 0.35])
    params = np.zeros((n, 12), np.float32)
    hulls = np.zeros(n, np.uint32)
    for i, t in enumerate(types):
        if t == N.SHAPE_SPHERE:
            params[i, :4] = [*rng.uniform(-0.1, 0.1, 3), rng.uniform(0.2, 0.8)]
        elif t == N.SHAPE_CAPSULE:
            h = rng.uniform(0.2, 0.8)
            params[i, :7] = [0, -h, 0, 0, h, 0, rng.uniform(0.1, 0.4)]
        elif t == N.SHAPE_TRIANGLE:
            params[i, :9] = rng.uniform(-0.8, 0.8, 9)
            params[i, 9] = 0.0
        else:
            hulls[i] = rng.integers(0, n_hulls)
    return types.astype(np.uint32), params, hulls


def toi_queries(rng, n, n_hulls):
    """Seeded b3TOIInput queries (TOI_INPUT_DTYPE): shape A sweeps from a
    random point toward the middle while rotating a little, shape B drifts
    near the middle; quaternion pairs of both signs; tMax = 1."""
    q = np.zeros(n, N.TOI_INPUT_DTYPE)
    q["type_a"], q["params_a"], q["hull_a"] = random_convex_shapes(rng, n, n_hulls)
    q["type_b"], q["params_b"], q["hull_b"] = random_convex_shapes(rng, n, n_hulls)
    for side, move in (("sweep_a", 1.0), ("sweep_b", 0.3)):
        sw = np.zeros((n, 18), np.float32)
        sw[:, 0:3] = rng.uniform(-0.1, 0.1, (n, 3))
        q0 = unit_quats(rng, n)
        small = np.concatenate([rng.normal(0, 0.3, (n, 3)), np.ones((n, 1))], axis=1)
        small /= np.linalg.norm(small, axis=1, keepdims=True)
        q1 = qmul(q0, small)
        flip = rng.random(n) < 0.3
        q1[flip] = -q1[flip]
        sw[:, 3:7] = q0
        sw[:, 11:15] = q1
        if side == "sweep_a":
            c0 = rng.uniform(-3, 3, (n, 3))
            target = rng.uniform(-1, 1, (n, 3))
            d = target - c0
            sw[:, 7:10] = c0
            sw[:, 15:18] = c0 + d * rng.uniform(0.5, 2.5, (n, 1)) * move
        else:
            c0 = rng.uniform(-0.5, 0.5, (n, 3))
            sw[:, 7:10] = c0
            sw[:, 15:18] = c0 + rng.normal(0, move, (n, 3))
        q[side] = sw
    q["t_max"] = 1.0
    return q

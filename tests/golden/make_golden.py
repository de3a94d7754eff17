"""Generates the golden fixtures in this directory by running the reference
(Bounce, built from its own sources into oracle/_ref by oracle/Makefile) on
small seeded scenes. Run from the repository root after `make -C oracle`:

    python tests/golden/make_golden.py

Each scene file holds the scene arrays (hulls, bodies, fixtures), and per
collision pass the body state fed to the pipeline (17 floats per body, read
back from the reference's bodies), the reference's fat AABBs, its contact
list (fixture A, fixture B, flags) sorted by pair, the hull feature caches
and every manifold point of touching contacts, from the FP32 build and the
FP64 rerun (-DB3_USE_DOUBLE) of the same routines (FP64 points stored as
float32).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from bounce_b200 import scene as S  # noqa: E402
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

SCENES = {
    "plain_small": lambda: S.plain_scene(seed=31, n_boxes=120, n_spheres=120, cube=6.0),
    "mixed_small": lambda: S.mixed_scene(seed=32, n=400, side=9.0),
}
PASSES = 3


def pack_pass(rw):
    rc = rw.contacts()
    key = (rc["fixtureA"].astype(np.uint64) << 32) | rc["fixtureB"]
    order = np.argsort(key)
    rc = rc[order]
    m = rc["manifolds"][:, 0]
    pc = np.where(rc["manifoldCount"] > 0, m["pointCount"], 0).astype(np.uint32)
    touch = np.nonzero(pc > 0)[0]
    pts = m["points"][touch]
    return dict(
        pairs=np.stack([rc["fixtureA"], rc["fixtureB"], rc["flags"], rc["manifoldCount"]], axis=1).astype(np.uint32),
        cache=rc["cache"].astype(np.uint32),
        point_count=pc,
        touch_index=touch.astype(np.uint32),
        # FP32 results are float32 values stored exactly; FP64 results are
        # stored rounded to float32 (1e-7 relative, far below the 1e-4 m tolerance).
        n=pts["n"].astype(np.float32), p1=pts["p1"].astype(np.float32), p2=pts["p2"].astype(np.float32),
        key=pts["key"].astype(np.uint32),
        tri=pts["triangleKey"].astype(np.uint32), edge=pts["edgeContact"].astype(np.uint8),
        fat=rw.fat_aabbs(),
    )


def make(name, build):
    sc = build().finalize()
    r32 = O.RefWorld(sc, 32)
    r64 = O.RefWorld(sc, 64)
    sc.set_local_centers(r32.local_centers())
    drv = S.KinematicDriver(sc)
    out = {}
    ha = sc.hull_arrays
    for k in ("desc", "verts", "edges", "faces", "planes", "centroids"):
        out[f"hull_{k}"] = ha[k]
    for k in ("body_world", "body_type", "body_pose", "body_lin", "body_ang", "fix_body", "fix_type", "fix_hull",
              "fix_params", "fix_flags", "local_center"):
        out[k] = getattr(sc, k)
    for p in range(PASSES):
        if p == 0:
            r32.first_pass()
            r64.first_pass()
        else:
            drv.advance()
            r32.set_sweeps(drv.sweeps14())
            r64.set_sweeps(drv.sweeps14())
            r32.step_pass()
            r64.step_pass()
        out[f"p{p}_state"] = r32.bodies17()
        for prec, rw in ((32, r32), (64, r64)):
            for k, v in pack_pass(rw).items():
                out[f"p{p}_r{prec}_{k}"] = v
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


def collide_poses():
    """Direct b3Collide* calls on the testbed's fixed poses (box_edge_contact.h,
    box_face_contact.h, capsule_collision.h, deep_capsule.h) plus seeded random
    poses of every convex pair type."""
    sc = S.Scene()
    box = sc.hulls.add_box(1.0, 1.0, 1.0)
    rng = np.random.default_rng(33)
    ell = sc.hulls.add_points(S.ellipsoid_points(rng, 20, np.array([0.8, 0.5, 0.6])))
    tall = sc.hulls.add_box(1.0, 2.0, 1.0)      # box_edge_contact.h:27
    tall_up = sc.hulls.add_box(1.0, 2.0, 1.0)   # box_face_contact.h:27-29, translated by (0, 2, 0)
    slab = sc.hulls.add_box(4.0, 1.0, 4.0)      # deep_capsule.h:27
    ha = sc.hulls.arrays()
    d = ha["desc"].reshape(-1, 6)[tall_up]
    t = np.array([0.0, 2.0, 0.0], np.float32)
    v = ha["verts"].reshape(-1, 3)
    v[d[0]:d[0] + d[1]] += t
    pl = ha["planes"].reshape(-1, 4)
    pl[d[4]:d[4] + d[5], 3] += pl[d[4]:d[4] + d[5], :3] @ t
    ha["centroids"].reshape(-1, 3)[tall_up] += t
    hulls = O.RefHulls(ha, 32)
    shapes = {
        "sphere": (0, [0, 0, 0, 1.0], 0),
        "capsule": (1, [0, -1, 0, 0, 1, 0, 0.5], 0),
        "box": (3, [0.0], box),
        "ellipsoid": (3, [0.0], ell),
        "tall": (3, [0.0], tall),
        "tall_up": (3, [0.0], tall_up),
        "slab": (3, [0.0], slab),
        "deep_capsule": (1, [1, -1, 0, 0, 1, 0, 2.0], 0),      # deep_capsule.h:31-33
        "long_capsule": (1, [0, -5, 0, 0, 5, 0, 1.0], 0),      # capsule_collision.h:27-29
        "short_capsule": (1, [0, -1, 0, 0, 1, 0, 1.0], 0),     # capsule_collision.h:33-35
    }
    kinds = [("sphere", "sphere"), ("capsule", "sphere"), ("capsule", "capsule"), ("box", "sphere"),
             ("box", "capsule"), ("box", "box"), ("ellipsoid", "box"), ("ellipsoid", "ellipsoid"),
             ("ellipsoid", "capsule"), ("ellipsoid", "sphere")]
    recs = []
    for a, b in kinds:
        for i in range(60):
            qa, qb = S.random_quats(rng, 2)
            pa = rng.uniform(-0.3, 0.3, 3).astype(np.float32)
            pb = (pa + rng.normal(0, 1, 3) * rng.uniform(0.5, 2.5)).astype(np.float32)
            recs.append((a, b, np.concatenate([pa, qa]), np.concatenate([pb, qb])))
    # The testbed scenes' fixed poses, and the same poses after the scenes'
    # keyboard steps (B moved by multiples of 0.05 m along x and y).
    ident = np.array([0, 0, 0, 0, 0, 0, 1], np.float32)
    f32 = lambda *a: np.array(a, np.float32)
    half = np.float32(0.5) * (np.float32(0.55) * np.float32(np.pi))  # b3QuatRotationZ(0.55 pi)
    qz = f32(0, 0, np.sin(half), np.cos(half))
    fixed = [
        # box_edge_contact.h:30-35
        ("tall", "tall", np.concatenate([f32(1.5, 1.0, 0.0), f32(0, 0, 0, 1)]),
         np.concatenate([f32(-1.29999995, 1.34999979, 0.0), f32(0.810514629, 0.342624813, 0.334119707, 0.337692767)])),
        # box_face_contact.h:27-36
        ("tall_up", "box", ident, ident),
        # deep_capsule.h:27-35
        ("slab", "deep_capsule", ident, np.concatenate([f32(0, 0, 0), qz])),
        # capsule_collision.h:27-37
        ("long_capsule", "short_capsule", ident, ident),
    ]
    for a, b, xfa, xfb in fixed:
        for dx in (0, -2, 3):
            for dy in (0, 2, -4):
                moved = xfb.copy()
                moved[0] += np.float32(0.05) * dx
                moved[1] += np.float32(0.05) * dy
                recs.append((a, b, xfa, moved))
    out = {f"hull_{k}": v for k, v in ha.items()}
    ta, tb, xa, xb, caches, dumps = [], [], [], [], [], []
    for a, b, xfa, xfb in recs:
        A, B = shapes[a], shapes[b]
        cache = np.array([0, 1, 0, 0], np.uint32)
        m = O.collide(hulls, A[0], A[1], A[2], B[0], B[1], B[2], xfa, xfb, xfa, xfb, cache, 32)
        ta.append([A[0], A[2]])
        tb.append([B[0], B[2]])
        xa.append(xfa)
        xb.append(xfb)
        caches.append(cache.copy())
        dumps.append(m)
    out["shape_a"] = np.array([shapes[r[0]][1] + [0] * (12 - len(shapes[r[0]][1])) for r in recs], np.float32)
    out["shape_b"] = np.array([shapes[r[1]][1] + [0] * (12 - len(shapes[r[1]][1])) for r in recs], np.float32)
    out["type_a"] = np.array(ta, np.uint32)
    out["type_b"] = np.array(tb, np.uint32)
    out["xf_a"] = np.array(xa, np.float32)
    out["xf_b"] = np.array(xb, np.float32)
    out["cache_out"] = np.array(caches, np.uint32)
    d = np.array(dumps)
    out["point_count"] = d["pointCount"].astype(np.uint32)
    out["n"] = d["points"]["n"]
    out["p1"] = d["points"]["p1"]
    out["p2"] = d["points"]["p2"]
    out["key"] = d["points"]["key"].astype(np.uint32)
    path = os.path.join(HERE, "collide_poses.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


def triangle_poses():
    """Direct b3Collide* calls of the triangle pairs (triangle-sphere,
    triangle-capsule, hull-triangle) on seeded poses around one triangle,
    without wings, with coplanar wings on every edge, and with one coplanar,
    one bent and one missing wing."""
    sc = S.Scene()
    rng = np.random.default_rng(41)
    small = sc.hulls.add_box(0.4, 0.4, 0.4)
    ell = sc.hulls.add_points(S.ellipsoid_points(rng, 16, np.array([0.6, 0.35, 0.45])))
    ha = sc.hulls.arrays()
    hulls = O.RefHulls(ha, 32)
    tri = [-1.5, 0, 1, 1.5, 0, 1, 0, 0, -1.6, 0.0]
    shapes = {
        "triangle": (2, tri, 0),
        "sphere": (0, [0, 0, 0, 0.5], 0),
        "capsule": (1, [0, -0.6, 0, 0, 0.6, 0, 0.3], 0),
        "box": (3, [0.0], small),
        "ellipsoid": (3, [0.0], ell),
    }
    z = [0.0] * 3
    wing_sets = [
        np.zeros(12, np.float32),
        np.array([0, 0, 3.5, 2.5, 0, -1.5, -2.5, 0, -1.5, 1, 1, 1], np.float32),
        np.array([0, 0, 3.5, 2.5, -0.7, -1.5] + z + [1, 1, 0], np.float32),
    ]
    kinds = [("triangle", "sphere"), ("triangle", "capsule"), ("box", "triangle"), ("ellipsoid", "triangle")]
    recs = []
    for a, b in kinds:
        for w, wings in enumerate(wing_sets):
            verts = np.array(tri[:9], np.float32).reshape(3, 3)
            for i in range(60):
                qa, qb = S.random_quats(rng, 2)
                pa = rng.uniform(-0.3, 0.3, 3).astype(np.float32)
                if i % 2:
                    # near an edge: a point on it pushed out a little
                    e = int(rng.integers(3))
                    t = rng.uniform(0.1, 0.9)
                    on = verts[e] + t * (verts[(e + 1) % 3] - verts[e])
                    out = on - verts.mean(axis=0)
                    local = on + rng.uniform(0.0, 0.5) * out / np.linalg.norm(out)
                    local[1] = rng.uniform(-0.3, 0.55)
                else:
                    local = np.array([rng.uniform(-1.8, 1.8), rng.uniform(-0.4, 0.6), rng.uniform(-1.8, 1.4)])
                local = local.astype(np.float32)
                pb = (pa + S.quat_rotate(qa[None], local[None])[0]).astype(np.float32)
                recs.append((a, b, np.concatenate([pa, qa]), np.concatenate([pb, qb]), wings))
    out = {f"hull_{k}": v for k, v in ha.items()}
    ta, tb, xa, xb, wa, wb, dumps = [], [], [], [], [], [], []
    for a, b, xfa, xfb, wings in recs:
        A, B = shapes[a], shapes[b]
        m = O.collide(hulls, A[0], A[1], A[2], B[0], B[1], B[2], xfa, xfb, xfa, xfb, None, 32,
                      wingsA=wings if A[0] == 2 else None, wingsB=wings if B[0] == 2 else None)
        ta.append([A[0], A[2]])
        tb.append([B[0], B[2]])
        xa.append(xfa)
        xb.append(xfb)
        wa.append(wings if A[0] == 2 else np.zeros(12, np.float32))
        wb.append(wings if B[0] == 2 else np.zeros(12, np.float32))
        dumps.append(m)
    pad = lambda v: v + [0] * (12 - len(v))
    out["shape_a"] = np.array([pad(shapes[r[0]][1]) for r in recs], np.float32)
    out["shape_b"] = np.array([pad(shapes[r[1]][1]) for r in recs], np.float32)
    out["type_a"] = np.array(ta, np.uint32)
    out["type_b"] = np.array(tb, np.uint32)
    out["xf_a"] = np.array(xa, np.float32)
    out["xf_b"] = np.array(xb, np.float32)
    out["wings_a"] = np.array(wa, np.float32)
    out["wings_b"] = np.array(wb, np.float32)
    d = np.array(dumps)
    out["point_count"] = d["pointCount"].astype(np.uint32)
    out["n"] = d["points"]["n"]
    out["p1"] = d["points"]["p1"]
    out["p2"] = d["points"]["p2"]
    out["key"] = d["points"]["key"].astype(np.uint32)
    path = os.path.join(HERE, "triangle_poses.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "points", int(out["point_count"].sum()))


if __name__ == "__main__":
    assert O.available(32) and O.available(64), "build the oracle first: make -C oracle"
    only = sys.argv[1:]
    if not only:
        for name, build in SCENES.items():
            make(name, build)
        collide_poses()
    if not only or "triangle_poses" in only:
        triangle_poses()

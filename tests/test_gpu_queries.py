"""World queries on the device against the reference's own b3World entry
points, after collision passes:

* QueryAABB: the fixtures reported for each box (as sets; the reference
  reports them in its dynamic tree's order),
* RayCast with a listener that keeps every hit: per ray the set of
  (fixture, point, normal, fraction), bit for bit,
* RayCastSingle: the closest fixture, point, normal and fraction, bit for bit,

on spheres, capsules and hulls, on a triangle terrain and on a mesh terrain;
and in a batched context, that a query only meets its own world.
"""
import numpy as np
import pytest

from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline

pytestmark = pytest.mark.gpu


def run_passes(O, sc, passes):
    rw = O.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    for k in range(passes):
        if k:
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
    assert pipe.counts()["status"] == 0
    return rw, pipe


def random_boxes(rng, lo, hi, n, size):
    c = rng.uniform(lo, hi, (n, 3))
    e = rng.uniform(0.05, size, (n, 3))
    return np.concatenate([c - e, c + e], axis=1).astype(np.float32)


def random_rays(rng, lo, hi, n):
    p1 = rng.uniform(lo, hi, (n, 3))
    p2 = rng.uniform(lo, hi, (n, 3))
    return np.concatenate([p1, p2], axis=1).astype(np.float32)


def check_queries(rw, pipe, rng, lo, hi, label, n=150, size=2.0):
    boxes = random_boxes(rng, lo, hi, n, size)
    got = pipe.query_aabb(boxes)
    found = 0
    for i, b in enumerate(boxes):
        want = np.sort(rw.query_aabb(b))
        mine = np.sort(got[got[:, 0] == i, 1])
        assert np.array_equal(mine, want), f"{label}: QueryAABB {i}: {mine[:8]} vs {want[:8]}"
        found += len(want)
    assert found > 0

    rays = random_rays(rng, lo, hi, n)
    idx, hits = pipe.ray_cast(rays)
    fix1, hit1 = pipe.ray_cast_single(rays)
    nhit = 0
    for i, r in enumerate(rays):
        wf, wh = rw.ray_cast(r)
        o = np.argsort(wf, kind="stable")
        wf, wh = wf[o], wh[o].astype(np.float32)
        sel = idx[:, 0] == i
        mf, mh = idx[sel, 1], hits[sel]
        o = np.argsort(mf, kind="stable")
        mf, mh = mf[o], mh[o]
        assert np.array_equal(mf, wf), f"{label}: RayCast {i}: fixtures {mf} vs {wf}"
        bad = np.nonzero(~np.all(mh == wh, axis=1))[0]
        assert len(bad) == 0, f"{label}: RayCast {i}: hits differ {mh[bad[:2]]} vs {wh[bad[:2]]}"
        sf, sh = rw.ray_cast_single(r)
        if sf is None:
            assert fix1[i] == 0xFFFFFFFF, f"{label}: RayCastSingle {i}: gpu hit {fix1[i]}, reference none"
        else:
            nhit += 1
            assert fix1[i] == sf, f"{label}: RayCastSingle {i}: fixture {fix1[i]} vs {sf}"
            assert np.array_equal(hit1[i], sh.astype(np.float32)), f"{label}: RayCastSingle {i}: {hit1[i]} vs {sh}"
    assert nhit > 0
    return nhit


def test_queries_mixed_shapes(oracle_mod):
    sc = S.mixed_scene(seed=31, n=2000, side=16.0, static_frac=0.05, sensor_frac=0.03).finalize()
    rw, pipe = run_passes(oracle_mod, sc, 4)
    check_queries(rw, pipe, np.random.default_rng(3), -8.0, 8.0, "mixed")
    # the device-buffer entry point gives the host one's results
    import ctypes

    import torch

    rays = random_rays(np.random.default_rng(8), -8.0, 8.0, 500)
    fix, hit = pipe.ray_cast_single(rays)
    d_rays = torch.from_numpy(rays).cuda()
    d_fix = torch.empty(len(rays), dtype=torch.int32, device="cuda")
    d_hit = torch.empty((len(rays), 7), dtype=torch.float32, device="cuda")
    pipe._check(pipe.lib.b3g_ray_cast_single_device(pipe.ctx, len(rays), ctypes.c_void_p(d_rays.data_ptr()), None,
                                                    ctypes.c_void_p(d_fix.data_ptr()),
                                                    ctypes.c_void_p(d_hit.data_ptr()), None))
    torch.cuda.synchronize()
    assert np.array_equal(d_fix.cpu().numpy().view(np.uint32), fix)
    assert np.array_equal(d_hit.cpu().numpy(), hit)
    pipe.close()


def test_queries_triangle_terrain(oracle_mod):
    sc = S.terrain_scene(seed=3, n=600).finalize()
    rw, pipe = run_passes(oracle_mod, sc, 3)
    check_queries(rw, pipe, np.random.default_rng(4), -8.0, 6.0, "triangles")
    pipe.close()


def test_queries_mesh_terrain(oracle_mod):
    sc = S.mesh_terrain_scene(seed=5, n=500, scale=(1.2, 0.9, 1.1)).finalize()
    rw, pipe = run_passes(oracle_mod, sc, 3)
    rng = np.random.default_rng(5)
    check_queries(rw, pipe, rng, -9.0, 5.0, "mesh")
    # rays from above straight down onto the terrain all hit the mesh or a body
    p1 = np.concatenate([rng.uniform(-8, 8, (100, 1)), np.full((100, 1), 30.0), rng.uniform(-8, 8, (100, 1))], 1)
    p2 = p1 * [1.0, 0.0, 1.0] + [0.0, -10.0, 0.0]
    fix, _ = pipe.ray_cast_single(np.concatenate([p1, p2], 1))
    assert np.all(fix != 0xFFFFFFFF)
    pipe.close()


def test_queries_stay_in_their_world():
    sc, _ = S.batched_scene(seed=12, n_worlds=6, lo=40, hi=300)
    sc.finalize()
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    pipe.collide(drv.state17())
    fat = pipe.fat_aabbs()
    fworld = sc.body_world[sc.fix_body]
    rng = np.random.default_rng(9)
    boxes = random_boxes(rng, -10.0, 10.0, 120, 3.0)
    worlds = rng.integers(0, sc.n_worlds, 120).astype(np.uint32)
    got = pipe.query_aabb(boxes, worlds)
    for i, (b, w) in enumerate(zip(boxes, worlds)):
        over = np.all(fat[:, 0:3] <= b[3:6], axis=1) & np.all(fat[:, 3:6] >= b[0:3], axis=1) & (fworld == w)
        assert np.array_equal(np.sort(got[got[:, 0] == i, 1]), np.nonzero(over)[0]), f"box {i}"
    rays = random_rays(rng, -10.0, 10.0, 120)
    idx, _ = pipe.ray_cast(rays, worlds)
    assert np.all(fworld[idx[:, 1]] == worlds[idx[:, 0]])
    pipe.close()

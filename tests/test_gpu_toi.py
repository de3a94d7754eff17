"""Time of impact and the GJK shape cast on the device against the
reference's own free functions, bit for bit (state, time, iterations; hit,
time, point, normal, iterations):

* b3TimeOfImpact(const b3TOIInput&) (time_of_impact.cpp:465-660) on sweeps of
  spheres, capsules, triangles and hulls that translate and rotate (quaternion
  pairs of both signs),
* b3TimeOfImpact(aabb1, d1, aabb2, d2) (time_of_impact.cpp:782-902),
* b3ShapeCast (gjk.cpp:938-1102),

with the states and hit flags spread over their cases.
"""
import numpy as np
import pytest

from bounce_b200 import _native as N
from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline
from bounce_b200.scene import random_convex_shapes as random_shapes
from bounce_b200.scene import toi_queries, unit_quats

pytestmark = pytest.mark.gpu


def test_time_of_impact_sweeps(oracle_mod):
    sc = S.mixed_scene(seed=7, n=200, side=8.0).finalize()
    hulls = oracle_mod.RefHulls(sc.hull_arrays)
    pipe = CollisionPipeline(sc)
    q = toi_queries(np.random.default_rng(1), 4000, len(sc.hull_arrays["desc"]) // 6)
    mine = pipe.time_of_impact(q)
    want = hulls.time_of_impact(q.view(np.float32).reshape(-1, 68))
    bad = np.nonzero(~np.all(mine == want, axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} differ, first {bad[:5]}: {mine[bad[:3]]} vs {want[bad[:3]]}"
    states = np.bincount(want[:, 0], minlength=5)
    assert states[2] > 20 and states[3] > 500 and states[4] > 500, states
    assert np.max(want[:, 2]) > 2
    pipe.close()


def test_time_of_impact_aabbs(oracle_mod):
    sc = S.mixed_scene(seed=7, n=50, side=6.0).finalize()
    pipe = CollisionPipeline(sc)
    rng = np.random.default_rng(2)
    n = 5000
    q = np.zeros((n, 18), np.float32)
    for off in (0, 9):
        c = rng.uniform(-3, 3, (n, 3))
        e = rng.uniform(0.1, 1.0, (n, 3))
        q[:, off:off + 3] = c - e
        q[:, off + 3:off + 6] = c + e
        q[:, off + 6:off + 9] = rng.normal(0, 3, (n, 3))
    q[::7, 6:9] = q[::7, 15:18]  # equal displacements: d = 0
    q[::11, 7] = q[::11, 16]      # one axis with d = 0
    mine = pipe.time_of_impact_aabb(q)
    want = oracle_mod.time_of_impact_aabb(q)
    bad = np.nonzero(~np.all(mine == want, axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} differ: {mine[bad[:3]]} vs {want[bad[:3]]}"
    states = np.bincount(want[:, 0], minlength=5)
    assert states[2] > 50 and states[3] > 50 and states[4] > 50, states
    pipe.close()


def test_gjk_shape_cast(oracle_mod):
    sc = S.mixed_scene(seed=7, n=200, side=8.0).finalize()
    hulls = oracle_mod.RefHulls(sc.hull_arrays)
    pipe = CollisionPipeline(sc)
    rng = np.random.default_rng(3)
    n = 4000
    nh = len(sc.hull_arrays["desc"]) // 6
    q = np.zeros(n, N.GJK_CAST_DTYPE)
    q["type_a"], q["params_a"], q["hull_a"] = random_shapes(rng, n, nh)
    q["type_b"], q["params_b"], q["hull_b"] = random_shapes(rng, n, nh)
    pa = rng.uniform(-1, 1, (n, 3))
    q["xf_a"] = np.concatenate([pa, unit_quats(rng, n)], axis=1)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    pb = pa + u * rng.uniform(2.0, 5.0, (n, 1))
    q["xf_b"] = np.concatenate([pb, unit_quats(rng, n)], axis=1)
    aim = pa + rng.normal(0, 0.6, (n, 3)) - pb
    q["translation_b"] = aim * rng.uniform(0.3, 1.6, (n, 1))
    mine = pipe.gjk_shape_cast(q)
    want = hulls.gjk_shape_cast(q.view(np.float32).reshape(-1, 48))
    mw, ww = mine.view(np.uint32), want.view(np.uint32)
    bad = np.nonzero(~np.all(mw == ww, axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} differ: {mine[bad[:3]]} vs {want[bad[:3]]}"
    hits = int(np.sum(ww[:, 0] == 1))
    assert 200 < hits < n - 200, hits
    pipe.close()

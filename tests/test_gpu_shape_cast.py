"""Shape casts on the device (b3g_shape_cast, b3g_shape_cast_single) against
the reference's own b3World::ShapeCast and ShapeCastSingle (world.cpp:568-851,
the translational b3TimeOfImpact of time_of_impact.cpp:666-776 on each
candidate), after collision passes, bit for bit:

* ShapeCast with a listener that keeps every hit: per cast the multiset of
  (fixture, point, normal, fraction) (the reference reports a mesh fixture
  once per touching triangle),
* ShapeCastSingle: the fraction, and fixture, point and normal unless two
  hits share the smallest fraction exactly (the reference keeps the first its
  tree meets, the device the smaller fixture and triangle),

casting spheres, capsules and hulls through mixed shapes, a triangle terrain
and a mesh terrain.
"""
import numpy as np
import pytest

from bounce_b200 import _native as N
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


def inward_casts(sc, rng, n, radius, length):
    """Casts from points on a sphere around the scene toward its middle (with
    some spread), so that most first contacts come at a fraction above 0."""
    c = random_casts(sc, rng, n, 0.0, 0.0)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    c["position"] = radius * u
    aim = rng.uniform(-0.3 * radius, 0.3 * radius, (n, 3)) - c["position"]
    aim /= np.linalg.norm(aim, axis=1, keepdims=True)
    c["displacement"] = aim * rng.uniform(length[0], length[1], (n, 1))
    return c


def random_casts(sc, rng, n, lo, hi, length=(1.0, 6.0)):
    """Casts of the scene's own sphere, capsule and hull shapes from random
    poses along random displacements."""
    params = sc.fix_params.reshape(-1, 12)
    pool = np.nonzero(np.isin(sc.fix_type, [N.SHAPE_SPHERE, N.SHAPE_CAPSULE, N.SHAPE_HULL]))[0]
    pick = rng.choice(pool, n)
    c = np.zeros(n, N.SHAPE_CAST_DTYPE)
    c["type"] = sc.fix_type[pick]
    c["hull"] = np.where(sc.fix_type[pick] == N.SHAPE_HULL, sc.fix_hull[pick], 0)
    c["params"] = params[pick]
    c["position"] = rng.uniform(lo, hi, (n, 3))
    q = rng.normal(size=(n, 4))
    c["rotation"] = q / np.linalg.norm(q, axis=1, keepdims=True)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    c["displacement"] = d * rng.uniform(length[0], length[1], (n, 1))
    return c


def rows(fix, hits):
    """Hits as sortable rows: fixture, then the float32 bit patterns."""
    h = np.ascontiguousarray(np.asarray(hits, np.float32)).view(np.uint32)
    r = np.concatenate([np.asarray(fix, np.uint64)[:, None], h.astype(np.uint64)], axis=1)
    return r[np.lexsort(r.T[::-1])] if len(r) else r


def check_casts(rw, pipe, casts, label):
    idx, hits = pipe.shape_cast(casts)
    fix1, hit1 = pipe.shape_cast_single(casts)
    raw = casts.view(np.float32).reshape(-1, 28)
    total = single = ties = 0
    for i in range(len(casts)):
        wf, wh = rw.shape_cast(raw[i])
        sel = idx[:, 0] == i
        mine, want = rows(idx[sel, 1], hits[sel]), rows(wf, wh)
        assert mine.shape == want.shape and np.array_equal(mine, want), \
            f"{label}: ShapeCast {i}: {len(mine)} hits vs {len(want)}\n{mine[:4]}\n{want[:4]}"
        total += len(want)
        sf, sh = rw.shape_cast_single(raw[i])
        if sf is None:
            assert fix1[i, 0] == 0xFFFFFFFF, f"{label}: ShapeCastSingle {i}: gpu hit {fix1[i]}, reference none"
            continue
        single += 1
        sh = sh.astype(np.float32)
        assert hit1[i, 6] == sh[6], f"{label}: ShapeCastSingle {i}: fraction {hit1[i, 6]} vs {sh[6]}"
        if fix1[i, 0] == sf and np.array_equal(hit1[i], sh):
            continue
        # an exact tie: the reference's pick is among the hits at this fraction
        at = hits[sel][:, 6] == sh[6]
        assert np.sum(at) > 1 and sf in idx[sel][at, 1], \
            f"{label}: ShapeCastSingle {i}: {fix1[i]} {hit1[i]} vs {sf} {sh}"
        ties += 1
    return total, single, ties


def test_shape_cast_mixed_shapes(oracle_mod):
    sc = S.mixed_scene(seed=37, n=1500, side=14.0, static_frac=0.05, sensor_frac=0.03).finalize()
    rw, pipe = run_passes(oracle_mod, sc, 3)
    rng = np.random.default_rng(1)
    # from outside the body cube inward (first contacts at fractions above 0),
    # and from inside it (many casts start touching: fraction 0, exact ties)
    total, single, ties = check_casts(rw, pipe, inward_casts(sc, rng, 200, 12.0, (6.0, 14.0)), "mixed inward")
    assert total > 200 and single > 100 and ties <= single // 5, (total, single, ties)
    total, single, _ = check_casts(rw, pipe, random_casts(sc, rng, 100, -7.0, 7.0), "mixed inside")
    assert total > 200 and single > 50, (total, single)
    pipe.close()


def test_shape_cast_triangle_terrain(oracle_mod):
    sc = S.terrain_scene(seed=3, n=500).finalize()
    rw, pipe = run_passes(oracle_mod, sc, 2)
    total, single, _ = check_casts(rw, pipe, random_casts(sc, np.random.default_rng(2), 150, -8.0, 5.0),
                                   "triangles")
    assert total > 50 and single > 20, (total, single)
    pipe.close()


def test_shape_cast_mesh_terrain(oracle_mod):
    sc = S.mesh_terrain_scene(seed=5, n=400, scale=(1.2, 0.9, 1.1)).finalize()
    rw, pipe = run_passes(oracle_mod, sc, 2)
    rng = np.random.default_rng(3)
    casts = random_casts(sc, rng, 150, -8.0, 5.0)
    # half of them straight down onto the terrain
    casts["displacement"][::2] = np.array([0.0, -12.0, 0.0], np.float32)
    casts["position"][::2, 1] = 6.0
    total, single, _ = check_casts(rw, pipe, casts, "mesh")
    idx, _ = pipe.shape_cast(casts)
    assert np.any(sc.fix_type[idx[:, 1]] == N.SHAPE_MESH) and total > 50 and single > 40, (total, single)
    pipe.close()

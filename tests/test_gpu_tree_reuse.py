"""LBVH reuse: a pass rebuilds the broadphase tree only every few passes (and
when the proxy set changes) and refits it in between. None of it may change
a result: the tree rebuilt every pass, every third pass and every eighth pass
(the default) gives the same contact list (order included), manifolds,
caches and fat AABBs, pass after pass, on one world and on many worlds in one
context, with bodies fast enough that the refit tree's boxes grow far from
the shape it was built for."""
import numpy as np
import pytest

from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline

from tests.test_gpu_batched import assert_same, results

pytestmark = pytest.mark.gpu


def fast(sc, factor):
    """The scene with its velocities scaled (bodies cross several of their
    own sizes between rebuilds)."""
    sc.body_lin = (np.float32(factor) * sc.body_lin).astype(np.float32)
    sc.body_ang = (np.float32(factor) * sc.body_ang).astype(np.float32)
    return sc


def run(sc, interval, passes, graph=False):
    drv = S.KinematicDriver(sc, walls=float(np.abs(sc.body_pos).max()))
    pipe = CollisionPipeline(sc, graph=graph)
    if interval is not None:
        pipe.set_tree_rebuild_interval(interval)
    out = []
    for _ in range(passes):
        pipe.collide(drv.state17())
        out.append(results(pipe))
        drv.advance()
    pipe.close()
    return out


@pytest.mark.parametrize("interval", [3, None])
def test_tree_reuse_matches_rebuild_every_pass(interval):
    sc = fast(S.mixed_scene(seed=71, n=3000, side=18.0).finalize(), 6.0)
    ref = run(sc, 1, 20)
    got = run(sc, interval, 20)
    for k, (a, b) in enumerate(zip(ref, got)):
        assert_same(a, b, f"interval {interval}, pass {k}")
    assert ref[-1]["counts"]["contacts"] > 1000


def test_tree_reuse_many_worlds_and_graphs():
    """Several worlds share the tree (each walk stops at its world's end): the
    refit passes must keep every world's leaves where the walks look."""
    sc, _ = S.batched_scene(seed=72, n_worlds=24, lo=16, hi=600)
    sc = fast(sc.finalize(), 6.0)
    ref = run(sc, 1, 18)
    got = run(sc, None, 18, graph=True)
    for k, (a, b) in enumerate(zip(ref, got)):
        assert_same(a, b, f"batched, pass {k}")


def test_tree_rebuild_interval_rejects_zero():
    sc = S.mixed_scene(seed=73, n=200, side=8.0).finalize()
    pipe = CollisionPipeline(sc)
    with pytest.raises(Exception):
        pipe.set_tree_rebuild_interval(0)
    pipe.close()

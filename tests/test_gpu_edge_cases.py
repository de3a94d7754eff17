"""Edge cases of the collision pass against the reference:

* a contact capacity too small for the pass is reported (B3G_E_CAPACITY),
  never silently truncated;
* worlds with one body, with only static bodies, and with bodies that never
  come near each other produce no contacts;
* coincident shapes (sphere centres on top of each other, a sphere centre on
  a capsule segment, a capsule of zero length, a hull and a sphere at the
  hull's centroid) give the reference's manifolds bit for bit.
"""
import numpy as np
import pytest

from bounce_b200 import _native as N
from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline
from tests.parity import compare_contacts, compare_fat_aabbs

pytestmark = pytest.mark.gpu

ID = (0.0, 0.0, 0.0, 1.0)


def run(O, sc, passes=3):
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
        compare_fat_aabbs(pipe, rw, f"pass {k}")
        compare_contacts(pipe, rw, f"pass {k}")
    return pipe


def test_capacity_overflow_is_reported():
    sc = S.mixed_scene(seed=3, n=3000, side=14.0).finalize()
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc, max_contacts=1000)
    pipe.collide(drv.state17())
    with pytest.raises(N.B3GError) as e:
        pipe.counts()
    assert e.value.code == N.B3G_E_CAPACITY
    pipe.close()


def test_scenes_without_contacts(oracle_mod):
    one = S.Scene()
    b = one.add_body(0, N.BODY_DYNAMIC, (0, 0, 0), ID, (1, 0, 0), (0, 1, 0))
    one.add_fixture(b, N.SHAPE_SPHERE, [0, 0, 0, 0.5])
    one.finalize()
    static = S.Scene()
    for i in range(4):
        b = static.add_body(0, N.BODY_STATIC, (0.3 * i, 0, 0), ID)
        static.add_fixture(b, N.SHAPE_SPHERE, [0, 0, 0, 0.5])
    static.finalize()
    far = S.Scene()
    for i in range(50):
        b = far.add_body(0, N.BODY_DYNAMIC, (10.0 * i, 0, 0), ID, (0, 0.5, 0))
        far.add_fixture(b, N.SHAPE_CAPSULE, [0, -0.5, 0, 0, 0.5, 0, 0.3])
    far.finalize()
    for sc in (one, static, far):
        pipe = run(oracle_mod, sc)
        assert pipe.counts()["contacts"] == 0
        pipe.close()


def test_coincident_shapes(oracle_mod):
    sc = S.Scene()
    box = sc.hulls.add_box(0.5, 0.4, 0.3)
    specs = [
        # two spheres with the same centre
        ((S.N.SHAPE_SPHERE, [0, 0, 0, 0.5], 0), (S.N.SHAPE_SPHERE, [0, 0, 0, 0.3], 0), (0, 0, 0)),
        # a sphere centred on a capsule's segment
        ((S.N.SHAPE_CAPSULE, [0, -0.5, 0, 0, 0.5, 0, 0.2], 0), (S.N.SHAPE_SPHERE, [0, 0, 0, 0.3], 0), (0, 0.2, 0)),
        # a capsule of zero length against a sphere
        ((S.N.SHAPE_CAPSULE, [0, 0, 0, 0, 0, 0, 0.4], 0), (S.N.SHAPE_SPHERE, [0, 0, 0, 0.3], 0), (0.1, 0, 0)),
        # two capsules on the same segment
        ((S.N.SHAPE_CAPSULE, [0, -0.5, 0, 0, 0.5, 0, 0.2], 0), (S.N.SHAPE_CAPSULE, [0, -0.5, 0, 0, 0.5, 0, 0.2], 0),
         (0, 0, 0)),
        # a sphere at a box's centre, and a box on a box
        ((S.N.SHAPE_HULL, [0.0], box), (S.N.SHAPE_SPHERE, [0, 0, 0, 0.2], 0), (0, 0, 0)),
        ((S.N.SHAPE_HULL, [0.0], box), (S.N.SHAPE_HULL, [0.0], box), (0, 0.7, 0)),
        # a capsule through a box's centre
        ((S.N.SHAPE_HULL, [0.0], box), (S.N.SHAPE_CAPSULE, [0, -0.5, 0, 0, 0.5, 0, 0.1], 0), (0, 0, 0)),
    ]
    for i, (a, b, off) in enumerate(specs):
        x = 10.0 * i
        ba = sc.add_body(0, N.BODY_DYNAMIC, (x, 0, 0), ID)
        sc.add_fixture(ba, a[0], a[1], hull=a[2])
        bb = sc.add_body(0, N.BODY_DYNAMIC, (x + off[0], off[1], off[2]), ID)
        sc.add_fixture(bb, b[0], b[1], hull=b[2])
    sc.finalize()
    pipe = run(oracle_mod, sc, passes=1)
    # every pair has a contact; which of them touch is the reference's call
    # (compared above), most do
    assert pipe.counts()["contacts"] == len(specs)
    assert pipe.counts()["touching"] >= len(specs) - 2
    pipe.close()


def test_walk_limit_reports_timeout_and_recovers(oracle_mod):
    """A device wait that runs out is reported, not hidden, and leaves the
    context usable: with the broadphase walks capped at 3 node visits the pass
    reports B3G_E_TIMEOUT (b3g_get_counts) and finds fewer pairs; with the
    bound restored the next passes match the reference again."""
    sc = S.mixed_scene(seed=61, n=1500, side=14.0).finalize()
    rw = oracle_mod.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    rw.first_pass()
    pipe.collide(drv.state17())
    full = pipe.counts()["contacts"]
    compare_contacts(pipe, rw, "before the limit")
    pipe.set_walk_limit(3)
    drv.advance()
    pipe.collide(drv.state17())
    with pytest.raises(N.B3GError) as err:
        pipe.counts()
    assert err.value.code == N.B3G_E_TIMEOUT
    assert pipe.pass_stats()["raw_pairs"] < full
    pipe.set_walk_limit(0)
    # The next pass starts clean; its new contacts (all pairs again) then
    # match a reference world driven through the same motion.
    rw2 = oracle_mod.RefWorld(sc)
    rw2.set_local_centers(sc.local_center)
    rw2.first_pass()
    drv2 = S.KinematicDriver(sc)
    for _ in range(2):
        drv2.advance()
        rw2.set_sweeps(drv2.sweeps14())
        rw2.step_pass()
    drv.advance()
    pipe.collide(drv.state17())
    assert pipe.counts()["status"] == 0
    g = pipe.contacts()
    r = rw2.pairs()
    key = lambda a: np.sort((a[:, 0].astype(np.uint64) << np.uint64(32)) | a[:, 1])
    assert np.array_equal(key(g), key(r))
    pipe.close()

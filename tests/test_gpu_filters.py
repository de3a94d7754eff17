"""Collision filters against the reference, bit for bit: joints that keep
their bodies from colliding (b3Body::ShouldCollide, body.cpp:240-263) and a
contact filter (b3ContactFilter, asked by AddPair, contact_manager.cpp:86-92,
and for every contact by UpdateContacts, :189-199).

The reference world gets real b3SphereJoints with collideConnected = false and
a seeded contact filter (oracle/ref_harness.cpp filter_rejects); the device
gets the same joints as body pairs (b3g_set_joint_pairs) and the same
filter's answers: for the last pass's contacts before a pass
(b3g_set_contact_veto) and for the new pairs the pass stops to ask about
(b3g_fetch_new_pairs / b3g_finish_pass). Joints come and go and the filter
changes its answers between passes, so pairs a filter once refused must wait
for a proxy to move before they can become contacts, as in the reference.
"""
import numpy as np
import pytest

from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline
from tests.parity import compare_contacts, compare_ended, compare_fat_aabbs, compare_order

pytestmark = pytest.mark.gpu


def _check_pass(pipe, rw, prev, label):
    c = pipe.counts()
    assert c["status"] == 0, c
    compare_fat_aabbs(pipe, rw, label)
    st = compare_contacts(pipe, rw, label)
    compare_order(pipe, rw, label)
    cur = rw.pairs()
    if prev is not None:
        compare_ended(pipe, prev, cur, label)
    return cur, st


def _touching_body_pairs(pipe, sc, rng, frac):
    c = pipe.contacts()
    t = c[(c[:, 2] & 1) != 0]
    pairs = np.stack([sc.fix_body[t[:, 0]], sc.fix_body[t[:, 1]]], axis=1)
    pick = rng.random(len(pairs)) < frac
    return pairs[pick].astype(np.uint32)


def test_joint_pairs_match_reference(oracle_mod):
    sc = S.mixed_scene(seed=31, n=3000, side=18.0, static_frac=0.05).finalize()
    rw = oracle_mod.RefWorld(sc)
    rw.set_local_centers(sc.local_center)
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    rng = np.random.default_rng(5)
    prev = None
    joints = np.zeros((0, 2), np.uint32)
    destroyed = 0
    for k in range(12):
        if k == 2:
            # Joints between half the touching bodies and some random pairs:
            # their contacts go at the next pass, touching or not.
            joints = np.concatenate([_touching_body_pairs(pipe, sc, rng, 0.5),
                                     rng.integers(0, sc.n_bodies, (200, 2)).astype(np.uint32)])
            joints = joints[joints[:, 0] != joints[:, 1]]
            rw.add_joints(joints)
            pipe.set_joint_pairs(joints)
        if k == 7:
            # Half the joints go: their pairs come back only once a proxy moves.
            joints = joints[: len(joints) // 2]
            rw.clear_joints()
            rw.add_joints(joints)
            pipe.set_joint_pairs(joints)
        if k:
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
        prev, st = _check_pass(pipe, rw, prev, f"joints pass {k}")
        if k == 2:
            destroyed = pipe.counts()["ended"]  # the new joints' contacts go in this pass
    assert destroyed > 100, destroyed
    pipe.close()
    rw.close()


def _filter_run(oracle_mod, sc, passes, modulus, label, sleep_frac=0.0, joints_at=None, seed=3):
    """Both worlds under the seeded contact filter, whose salt changes every
    third pass; optionally bodies falling asleep and joints added."""
    rw = oracle_mod.RefWorld(sc)
    rw.set_local_centers(sc.local_center)
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc, contact_filter=True)
    rng = np.random.default_rng(seed)
    prev = None
    moved = np.ones(sc.n_bodies, np.uint8)
    asked = vetoed = 0
    for k in range(passes):
        salt = k // 3
        rw.set_filter(modulus, salt)
        if joints_at is not None and k == joints_at:
            joints = _touching_body_pairs(pipe, sc, rng, 0.3)
            rw.add_joints(joints)
            pipe.set_joint_pairs(joints)
        if k:
            # UpdateContacts asks the filter about every contact of the list.
            c = pipe.contacts()
            veto = oracle_mod.filter_rejects(c[:, 0], c[:, 1], modulus, salt).astype(np.uint8)
            pipe.set_contact_veto(veto)
            if sleep_frac > 0:
                drv.advance(moved)
                awake = moved & (rng.random(sc.n_bodies) > sleep_frac).astype(np.uint8)
                rw.set_sweeps(drv.sweeps14())
                rw.step_pass_sleep(moved, awake)
                pipe.set_awake(awake)
            else:
                drv.advance()
                rw.set_sweeps(drv.sweeps14())
                rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
        cand = pipe.new_pairs()
        # The pairs AddPair asks the filter about, in the same order.
        calls = rw.filter_calls()
        assert np.array_equal(cand, calls), (
            f"{label} pass {k}: {len(cand)} new pairs vs {len(calls)} filter calls in AddPair")
        keep = ~oracle_mod.filter_rejects(cand[:, 0], cand[:, 1], modulus, salt)
        pipe.finish_pass(keep.astype(np.uint8))
        asked += len(cand)
        vetoed += int(np.count_nonzero(~keep))
        prev, _ = _check_pass(pipe, rw, prev, f"{label} pass {k}")
        if sleep_frac > 0:
            ga, ra = pipe.awake(), rw.awake()
            assert np.array_equal(ga, ra), f"{label} pass {k}: awake flags differ"
            moved = ga.copy()
    pipe.close()
    rw.close()
    return asked, vetoed


def test_contact_filter_matches_reference(oracle_mod):
    sc = S.mixed_scene(seed=33, n=3000, side=18.0, sensor_frac=0.05).finalize()
    asked, vetoed = _filter_run(oracle_mod, sc, 10, 4, "filter", joints_at=5)
    assert asked > 1000 and vetoed > 200, (asked, vetoed)


def test_contact_filter_with_sleeping_bodies(oracle_mod):
    """Contacts of sleeping bodies are filtered too (UpdateContacts asks the
    filter before it skips inactive contacts)."""
    sc = S.mixed_scene(seed=35, n=1500, side=14.0, static_frac=0.1).finalize()
    _filter_run(oracle_mod, sc, 8, 3, "filter-sleep", sleep_frac=0.4)


def test_filter_calls_outside_a_pass_fail():
    sc = S.mixed_scene(seed=37, n=200, side=6.0).finalize()
    pipe = CollisionPipeline(sc, contact_filter=True)
    drv = S.KinematicDriver(sc)
    pipe.collide(drv.state17())
    with pytest.raises(Exception):
        pipe.collide(drv.state17())  # the open pass waits for finish_pass
    with pytest.raises(Exception):
        pipe.counts()
    pipe.new_pairs()
    with pytest.raises(Exception):
        pipe.finish_pass(np.ones(1_000_000, np.uint8))  # wrong count
    pipe.finish_pass(None)
    assert pipe.counts()["status"] == 0
    with pytest.raises(Exception):
        pipe.set_contact_veto(np.zeros(pipe.counts()["contacts"] + 1, np.uint8))
    with pytest.raises(Exception):
        pipe.set_joint_pairs(np.array([[0, sc.n_bodies]], np.uint32))
    pipe.close()

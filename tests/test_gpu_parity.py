"""GPU parity against the reference's own FP32 collision pipeline (oracle/_ref):
contact sets, fat AABBs, manifolds, feature ids and hull feature caches must
be identical, pass after pass."""
import numpy as np
import pytest

from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline
from tests.parity import compare_contacts, compare_fat_aabbs, compare_order

pytestmark = pytest.mark.gpu


def run_parity(O, sc, passes, label, awake_fn=None):
    rw = O.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    stats = []
    for k in range(passes):
        if k:
            drv.advance()
            if awake_fn is not None:
                aw = awake_fn(k, sc.n_bodies)
                rw.set_awake(aw)
                pipe.set_awake(aw)
            rw.set_sweeps(drv.sweeps14())
            # The reference derives m_xf from the sweep; the driver's float32
            # transform must be the same bits.
            ref_state = rw.bodies17().reshape(-1, 17)
            assert np.array_equal(ref_state[:, 0:7], drv.state17().reshape(-1, 17)[:, 0:7])
            rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
        c = pipe.counts()
        assert c["status"] == 0, c
        compare_fat_aabbs(pipe, rw, f"{label} pass {k}")
        stats.append(compare_contacts(pipe, rw, f"{label} pass {k}"))
    pipe.close()
    return stats


def test_plain_first_pass(oracle_mod):
    sc = S.plain_scene(seed=1).finalize()
    st = run_parity(oracle_mod, sc, 1, "plain")
    assert st[0]["touching"] > 1000


def test_plain_many_passes(oracle_mod):
    sc = S.plain_scene(seed=5, n_boxes=400, n_spheres=400, cube=10.0).finalize()
    run_parity(oracle_mod, sc, 12, "plain-12")


def test_mixed_passes(oracle_mod):
    sc = S.mixed_scene(seed=7, n=3000, side=18.0).finalize()
    st = run_parity(oracle_mod, sc, 8, "mixed")
    assert st[-1]["touching"] > 100


def test_list_order(oracle_mod):
    """New contacts first in descending proxy-pair order, then the older ones
    in their previous order (broad_phase.h:181-206, contact_manager.cpp:105-111),
    and the destroyed ones listed in list order."""
    sc = S.mixed_scene(seed=11, n=2000, side=16.0).finalize()
    rw = oracle_mod.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    prev = None
    for k in range(6):
        if k:
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
        assert pipe.counts()["status"] == 0
        compare_order(pipe, rw, f"order pass {k}")
        cur = rw.pairs()
        if prev is not None:
            ck = set(map(tuple, cur[:, :2].tolist()))
            want = np.array([r for r in prev.tolist() if (r[0], r[1]) not in ck], np.uint32).reshape(-1, 3)
            got = pipe.ended()
            assert np.array_equal(got[:, :2], want[:, :2]), f"pass {k}: ended list"
            assert np.array_equal(got[:, 2] & 1, want[:, 2] & 1), f"pass {k}: ended touching flags"
        prev = cur
    pipe.close()


def run_sleeping(O, sc, passes, label, seed, sleep_frac, impulses=False):
    """Sleep as the reference's solver produces it: the bodies awake after a
    pass (wake-ups included) move in the next one, a random part of them falls
    asleep right after moving (synchronised, then asleep for UpdateContacts),
    and a sleeping body keeps its sweep."""
    rw = O.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    rng = np.random.default_rng(seed)
    dynamic = sc.body_type != 0
    moved = np.ones(sc.n_bodies, np.uint8)
    woken_total = 0
    for k in range(passes):
        if k:
            if impulses:
                # the solver's impulses handed back for every contact
                n = pipe.counts()["contacts"]
                normal = rng.uniform(0, 5, (n, 3, 4)).astype(np.float32)
                tangent = rng.uniform(-1, 1, (n, 3, 2)).astype(np.float32)
                motor = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
                rw.load_impulses(normal, tangent, motor)
                pipe.load_impulses(normal[:, 0], tangent[:, 0], motor[:, 0])
            drv.advance(moved)
            awake = moved & (rng.random(sc.n_bodies) > sleep_frac).astype(np.uint8)
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass_sleep(moved, awake)
            pipe.set_awake(awake)
        else:
            awake = moved
            rw.first_pass()
        pipe.collide(drv.state17())
        c = pipe.counts()
        assert c["status"] == 0, c
        compare_fat_aabbs(pipe, rw, f"{label} pass {k}")
        compare_contacts(pipe, rw, f"{label} pass {k}")
        compare_order(pipe, rw, f"{label} pass {k}")
        ga, ra = pipe.awake(), rw.awake()
        bad = np.nonzero(ga != ra)[0]
        assert len(bad) == 0, f"{label} pass {k}: awake flags differ at {len(bad)} bodies, first {bad[:5]}"
        woken_total += int(np.count_nonzero(dynamic & (ga != 0) & (awake == 0)))
        moved = ga.copy()
    pipe.close()
    return woken_total


def test_mixed_sleeping(oracle_mod):
    """Asleep bodies are neither synchronised nor collided (world.cpp:427-442,
    contact_manager.cpp:253-259); contacts that start or stop touching, and
    destroyed contacts with points, wake bodies for the contacts after them in
    the list (contact.cpp:249-254, contact.cpp:108-126)."""
    sc = S.mixed_scene(seed=9, n=1500, side=14.0, static_frac=0.1, sensor_frac=0.05).finalize()
    woken = run_sleeping(oracle_mod, sc, 8, "sleep", seed=100, sleep_frac=0.3)
    assert woken > 0


def test_sleeping_with_solver_impulses(oracle_mod):
    """Impulses handed back by the host solver warm-start the contacts that
    run and stay in the manifolds of the contacts UpdateContacts skips."""
    sc = S.mixed_scene(seed=21, n=1500, side=14.0, static_frac=0.1, sensor_frac=0.05).finalize()
    run_sleeping(oracle_mod, sc, 6, "sleep-impulses", seed=5, sleep_frac=0.5, impulses=True)


def test_mostly_sleeping(oracle_mod):
    """Most bodies asleep: long wake-up chains through the list."""
    sc = S.mixed_scene(seed=13, n=2500, side=15.0, static_frac=0.05, sensor_frac=0.03).finalize()
    woken = run_sleeping(oracle_mod, sc, 8, "mostly-asleep", seed=7, sleep_frac=0.8)
    assert woken > 0


def test_packed_results_match_touching():
    """The packed touching output unpacks to b3g_fetch_touching's records
    (point slots past pointCount aside)."""
    sc = S.mixed_scene(seed=19, n=3000, side=18.0).finalize()
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    for k in range(4):
        pipe.collide(drv.state17())
        drv.advance()
        idx, man = pipe.touching()
        contacts = np.zeros((200000, 3), np.uint32)
        index = np.zeros(200000, np.uint32)
        packed = np.zeros(200000 * 320, np.uint8)
        cnt = pipe.fetch_results_packed_async(contacts, index, packed)
        pipe.wait_results()
        assert cnt["manifolds"] == len(idx)
        assert np.array_equal(index[:len(idx)], idx)
        assert np.array_equal(contacts[:cnt["contacts"]], pipe.contacts())
        got = pipe.unpack_manifolds(packed, len(idx))
        assert np.array_equal(got["pointCount"], man["pointCount"])
        for f in ("tangentImpulse", "motorImpulse", "motorSpeed", "tangentSpeed1", "tangentSpeed2"):
            assert np.array_equal(got[f], man[f]), f
        mask = np.arange(4)[None, :] < man["pointCount"][:, None]
        assert np.array_equal(got["points"][mask].view(np.uint8), man["points"][mask].view(np.uint8))
    pipe.close()


def test_async_results_match_sync():
    """b3g_fetch_results_async, with the next pass running while the copies
    travel, returns what the synchronous fetches return for the same pass;
    the asynchronous context replays its passes from CUDA graphs fed with
    pinned host state."""
    import torch

    sc = S.mixed_scene(seed=17, n=3000, side=18.0).finalize()
    drv = S.KinematicDriver(sc)
    sync_pipe = CollisionPipeline(sc)
    async_pipe = CollisionPipeline(sc, graph=True)
    pinned = [torch.empty(17 * sc.n_bodies, dtype=torch.float32).pin_memory() for _ in range(2)]
    cap = 200000
    bufs = [(np.zeros((cap, 3), np.uint32), np.zeros(cap, np.uint32), np.zeros(cap, S.N.MANIFOLD_DTYPE))
            for _ in range(2)]
    pending = None
    expected = []
    for k in range(6):
        state = drv.state17()
        sync_pipe.collide(state)
        expected.append((sync_pipe.contacts().copy(), *[x.copy() for x in sync_pipe.touching()]))
        host = pinned[k % 2].numpy()
        host[:] = state
        async_pipe.collide(host)  # runs while the previous pass's copies travel
        if pending is not None:
            async_pipe.wait_results()
            j, cnt = pending
            c, i, m = bufs[j]
            want_c, want_i, want_m = expected[k - 1]
            assert np.array_equal(c[:cnt["contacts"]], want_c)
            assert np.array_equal(i[:cnt["manifolds"]], want_i)
            assert np.array_equal(m[:cnt["manifolds"]].view(np.uint8), want_m.view(np.uint8))
        j = k % 2
        pending = (j, async_pipe.fetch_results_async(*bufs[j]))
        drv.advance()
    async_pipe.wait_results()
    assert async_pipe.totals()["graph_passes"] >= 3
    sync_pipe.close()
    async_pipe.close()


def test_fixture_edge_lists(oracle_mod):
    """The island graph's edges: every fixture's contacts in the order of its
    b3Fixture::m_contactList, pass after pass (contacts created, kept and
    destroyed), against the reference's own edge lists."""
    sc = S.mixed_scene(seed=23, n=2000, side=15.0, static_frac=0.05).finalize()
    rw = oracle_mod.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    for k in range(6):
        if k:
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
        assert pipe.counts()["status"] == 0
        offsets, edges = pipe.fixture_contacts()
        want_off, want_pairs = rw.fixture_edges()
        assert np.array_equal(offsets, want_off), f"pass {k}: edge counts differ"
        got_pairs = pipe.contacts()[edges, :2]
        assert np.array_equal(got_pairs, want_pairs), f"pass {k}: edge order differs"
    pipe.close()

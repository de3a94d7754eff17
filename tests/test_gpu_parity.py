"""GPU parity against the reference's own FP32 collision pipeline (oracle/_ref):
contact sets, fat AABBs, manifolds, feature ids and hull feature caches must
be identical, pass after pass."""
import numpy as np
import pytest

from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline
from tests.parity import compare_contacts, compare_fat_aabbs

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


@pytest.mark.xfail(strict=True, reason="wake-ups inside UpdateContacts follow the reference's contact-list "
                   "order (contact.cpp:455-460, contact.cpp:227-237); the pass does not propagate them yet")
def test_mixed_sleeping(oracle_mod):
    """Asleep bodies are neither synchronised nor collided (world.cpp:427-442,
    contact_manager.cpp:262-268)."""
    sc = S.mixed_scene(seed=9, n=1500, side=14.0).finalize()

    def awake(k, n):
        rng = np.random.default_rng(100 + k)
        return (rng.random(n) > 0.3).astype(np.uint8)

    run_parity(oracle_mod, sc, 5, "sleep", awake_fn=awake)

"""Batched worlds, captured passes and launch shapes: none of them may change
a result.

* many worlds in one context give, world by world, the contact list (order
  included), manifolds, caches and fat AABBs of one context per world;
* passes replayed from a captured CUDA graph give the results of passes
  launched kernel by kernel;
* every launch shape of the tuning table, and the autotuner's choice, give
  the results of the default shapes.
"""
import numpy as np
import pytest

from bounce_b200 import _native as N
from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline

pytestmark = pytest.mark.gpu


def results(p):
    """Everything a pass produces, with manifold points past pointCount
    (unspecified, as in the reference) left out."""
    c = p.contacts()
    man = p.manifolds()
    pc = np.where((c[:, 2] >> 8) & 0xFF, man["pointCount"], 0)
    mask = np.arange(4)[None, :] < pc[:, None]
    pts = {f: man["points"][f][mask] for f in ("n", "p1", "p2", "normalImpulse", "key", "persisting")}
    return dict(contacts=c, pc=pc, pts=pts, tangent=man["tangentImpulse"][pc > 0], caches=p.caches(),
                fat=p.fat_aabbs(), ended=p.ended(), counts=p.counts(), awake=p.awake())


def assert_same(a, b, label):
    for k in ("contacts", "pc", "caches", "fat", "ended", "tangent", "awake"):
        assert np.array_equal(a[k], b[k]), f"{label}: {k} differ"
    for f in a["pts"]:
        assert np.array_equal(a["pts"][f], b["pts"][f]), f"{label}: manifold {f} differ"
    assert a["counts"] == b["counts"], f"{label}: counts differ"


def test_graph_replay_matches_direct():
    torch = pytest.importorskip("torch")
    sc = S.mixed_scene(seed=17, n=3000, side=18.0).finalize()
    drv = S.KinematicDriver(sc)
    direct = CollisionPipeline(sc)
    graphed = CollisionPipeline(sc, graph=True)
    # Three state buffers in turn: a parity's graph sees its state move to
    # another address every time and re-points its copy node.
    dev = [torch.empty(sc.n_bodies * 17, dtype=torch.float32, device="cuda") for _ in range(3)]
    for k in range(10):
        if k:
            drv.advance()
        st = drv.state17()
        direct.collide(st)
        dev[k % 3].copy_(torch.from_numpy(st))
        torch.cuda.synchronize()
        graphed.collide(dev[k % 3].data_ptr(), on_device=True)
        assert_same(results(direct), results(graphed), f"pass {k}")
    t = graphed.totals()
    assert t["graph_passes"] == 9, t
    assert t["launches"] == direct.totals()["launches"]
    direct.close()
    graphed.close()


def test_launch_shapes_do_not_change_results():
    sc = S.mixed_scene(seed=19, n=3000, side=18.0).finalize()
    drv = S.KinematicDriver(sc)
    base = CollisionPipeline(sc)
    low = CollisionPipeline(sc)
    high = CollisionPipeline(sc)
    tuned = CollisionPipeline(sc)
    t = base.tuning()
    assert list(t) == [4] * 5 + [8] + [4] * 3 + [4, 4, 2, 128]
    lo = np.array([1] * 9 + [1, 2, 1, 64], np.uint32)
    hi = np.array([16] * 9 + [16, 8, 8, 256], np.uint32)
    low.set_tuning(lo)
    high.set_tuning(hi)
    assert np.array_equal(high.tuning(), hi)
    with pytest.raises(N.B3GError):
        low.set_tuning(np.array([3] * 13, np.uint32))
    chosen = None
    for k in range(6):
        if k:
            drv.advance()
        st = drv.state17()
        for p in (base, low, high, tuned):
            p.collide(st)
        if k == 1:
            before = results(tuned)
            chosen = tuned.autotune(reps=3)
            # Re-running the tuned kernels on the pass's data changes nothing.
            assert_same(before, results(tuned), "after autotune")
        r = results(base)
        for name, p in (("low", low), ("high", high), ("tuned", tuned)):
            assert_same(r, results(p), f"pass {k} {name}")
    print("autotuned launch shapes:", chosen.tolist())
    for p in (base, low, high, tuned):
        p.close()


def test_batched_worlds_match_world_by_world():
    sc, counts = S.batched_scene(seed=5, n_worlds=24, lo=16, hi=600, cube=20.0)
    sc.finalize()
    drv = S.KinematicDriver(sc)
    batched = CollisionPipeline(sc)
    worlds = []
    for w in range(len(counts)):
        sub, bodies, fixtures = sc.world_subset(w)
        worlds.append((CollisionPipeline(sub), bodies, fixtures))
    fix_world = sc.body_world[sc.fix_body]
    for k in range(5):
        if k:
            drv.advance()
        st = drv.state17().reshape(-1, 17)
        batched.collide(np.ascontiguousarray(st.reshape(-1)))
        g = results(batched)
        local = np.full(sc.n_fixtures, -1, np.int64)
        for w, (p, bodies, fixtures) in enumerate(worlds):
            p.collide(np.ascontiguousarray(st[bodies].reshape(-1)))
            r = results(p)
            local[fixtures] = np.arange(len(fixtures))
            sel = fix_world[g["contacts"][:, 0]] == w
            mine = g["contacts"][sel].astype(np.int64)
            mine[:, 0] = local[mine[:, 0]]
            mine[:, 1] = local[mine[:, 1]]
            assert np.array_equal(mine, r["contacts"].astype(np.int64)), f"pass {k} world {w}: contact list"
            assert np.array_equal(g["pc"][sel], r["pc"]), f"pass {k} world {w}: point counts"
            assert np.array_equal(g["caches"][sel], r["caches"]), f"pass {k} world {w}: caches"
            assert np.array_equal(g["fat"][fixtures], r["fat"]), f"pass {k} world {w}: fat AABBs"
            gm = batched.manifolds()[sel]
            rm = p.manifolds()
            mask = np.arange(4)[None, :] < r["pc"][:, None]
            for f in ("n", "p1", "p2", "key", "normalImpulse", "persisting"):
                assert np.array_equal(gm["points"][f][mask], rm["points"][f][mask]), f"pass {k} world {w}: {f}"
            ge = g["ended"]
            esel = fix_world[ge[:, 0]] == w if len(ge) else np.zeros(0, bool)
            e = ge[esel].astype(np.int64)
            if len(e):
                e[:, 0] = local[e[:, 0]]
                e[:, 1] = local[e[:, 1]]
            assert np.array_equal(e, r["ended"].astype(np.int64)), f"pass {k} world {w}: ended"
    batched.close()
    for p, _, _ in worlds:
        p.close()

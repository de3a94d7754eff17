"""Triangle shapes on the GPU against the reference, bit for bit:

* b3CollideTriangleAndSphere / TriangleAndCapsule / HullAndTriangle through
  b3g_collide_pairs on the committed pose fixture (no wings, coplanar wings,
  a bent and a missing wing), and
* collision passes over a terrain of static triangle fixtures whose edges
  carry the wings of the grid's adjacency, under moving spheres, capsules and
  hulls: contact list (order included), fat AABBs, manifolds, ids.
"""
import numpy as np
import pytest

from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline
from tests import golden_util as G
from tests.parity import compare_contacts, compare_fat_aabbs
from tests.parity import compare_order

pytestmark = pytest.mark.gpu


def test_triangle_pairs_match_reference_poses():
    d = G.load("triangle_poses")
    sc = S.Scene()
    hull_arrays = {k: np.ascontiguousarray(d[f"hull_{k}"]) for k in
                   ("desc", "verts", "edges", "faces", "planes", "centroids")}
    # One fixture (on its own dynamic body) per distinct shape and wing set.
    shapes = {}
    wings = []
    fa, fb = [], []
    for i in range(len(d["point_count"])):
        for side in (0, 1):
            t = d["type_a"][i] if side == 0 else d["type_b"][i]
            sp = d["shape_a"][i] if side == 0 else d["shape_b"][i]
            w = d["wings_a"][i] if side == 0 else d["wings_b"][i]
            key = (int(t[0]), int(t[1]), sp.tobytes(), w.tobytes() if t[0] == 2 else b"")
            if key not in shapes:
                b = sc.add_body(0, S.N.BODY_DYNAMIC, (0, 0, 0), (0, 0, 0, 1))
                shapes[key] = sc.add_fixture(b, int(t[0]), sp, hull=int(t[1]))
                if t[0] == 2:
                    wings.append((shapes[key], w))
            (fa if side == 0 else fb).append(shapes[key])
    sc.finalize(hull_arrays)
    sc.tri_fixtures = np.array([f for f, _ in wings], np.uint32)
    sc.tri_wings = np.array([w for _, w in wings], np.float32)
    pipe = CollisionPipeline(sc)
    cache = np.tile(np.array([0, 1, 0, 0], np.uint32), (len(fa), 1))
    man = pipe.collide_pairs(fa, fb, d["xf_a"], d["xf_b"], d["xf_a"], d["xf_b"], cache)
    pc = d["point_count"]
    assert np.array_equal(man["pointCount"], pc)
    mask = np.arange(4)[None, :] < pc[:, None]
    for f in ("n", "p1", "p2"):
        bad = np.nonzero(~np.all(man["points"][f] == d[f].astype(np.float32), axis=-1) & mask)
        assert len(bad[0]) == 0, (f, bad[0][:5])
    assert np.array_equal(man["points"]["key"][mask], d["key"][mask])
    pipe.close()


def test_terrain_passes_match_reference(oracle_mod):
    sc = S.terrain_scene(seed=3, n=800).finalize()
    rw = oracle_mod.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    kinds = set()
    for k in range(8):
        if k:
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
        assert pipe.counts()["status"] == 0
        compare_fat_aabbs(pipe, rw, f"terrain pass {k}")
        compare_contacts(pipe, rw, f"terrain pass {k}")
        compare_order(pipe, rw, f"terrain pass {k}")
        c = pipe.contacts()
        touching = c[(c[:, 2] & 1) == 1]
        kinds |= set(zip(sc.fix_type[touching[:, 0]].tolist(), sc.fix_type[touching[:, 1]].tolist()))
    assert {(2, 0), (2, 1), (3, 2)} <= kinds, kinds
    pipe.close()

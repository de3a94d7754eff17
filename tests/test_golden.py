"""CPU checks that pin the oracle: the scene generator and hull builder
reproduce the golden inputs, the reference build reproduces the golden
outputs it was used to make, and the C restatement of the broadphase front
end (oracle/restate.c) reproduces the reference's fat AABBs and contact sets."""
import numpy as np
import pytest

from bounce_b200 import scene as S
from tests import golden_util as G


@pytest.mark.parametrize("name", G.SCENES)
def test_generator_reproduces_golden_inputs(name):
    d = G.load(name)
    builders = {
        "plain_small": lambda: S.plain_scene(seed=31, n_boxes=120, n_spheres=120, cube=6.0),
        "mixed_small": lambda: S.mixed_scene(seed=32, n=400, side=9.0),
    }
    sc = builders[name]().finalize()
    for k in ("desc", "verts", "edges", "faces", "planes"):
        assert np.array_equal(sc.hull_arrays[k], d[f"hull_{k}"]), k
    for k in ("body_type", "body_pose", "fix_body", "fix_type", "fix_hull", "fix_params"):
        assert np.array_equal(getattr(sc, k), d[k]), k


@pytest.mark.parametrize("name", G.SCENES)
def test_reference_reproduces_golden_outputs(name, oracle_mod):
    O = oracle_mod
    d = G.load(name)
    sc = G.scene_from(d)
    rw = O.RefWorld(sc, 32)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    for p in range(G.PASSES):
        if p == 0:
            rw.first_pass()
        else:
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass()
        assert np.array_equal(rw.bodies17(), d[f"p{p}_state"])
        pairs = rw.pairs()
        order = np.argsort(G.contact_keys(pairs))
        assert np.array_equal(pairs[order][:, :2], d[f"p{p}_r32_pairs"][:, :2])
        assert np.array_equal(rw.fat_aabbs(), d[f"p{p}_r32_fat"])


@pytest.mark.parametrize("name", G.SCENES)
def test_restatement_matches_reference_golden(name, oracle_mod):
    """restate.c: fat AABBs bit-exact and contact sets identical to the
    reference's, pass after pass (creation pass, then MoveProxy passes)."""
    O = oracle_mod
    d = G.load(name)
    sc = G.scene_from(d)
    fat = np.zeros((sc.n_fixtures, 6), np.float32)
    for p in range(G.PASSES):
        O.restate_sync(sc, d[f"p{p}_state"], fat, creation=(p == 0))
        assert np.array_equal(fat, d[f"p{p}_r32_fat"]), f"pass {p}: fat AABBs differ"
        pairs = O.restate_pairs(sc, fat)
        assert np.array_equal(pairs, d[f"p{p}_r32_pairs"][:, :2]), f"pass {p}: contact sets differ"


def test_fp64_rerun_agrees_with_fp32_within_tolerance():
    """The FP32 reference stated against its FP64 rerun: same contact sets on
    these scenes, and manifold points within the pipeline's tolerance
    (1e-4 m) wherever both produce the same point count (SAT ties are counted)."""
    for name in G.SCENES:
        d = G.load(name)
        for p in range(G.PASSES):
            a, b = d[f"p{p}_r32_pairs"], d[f"p{p}_r64_pairs"]
            assert np.array_equal(a[:, :2], b[:, :2])
            pa, pb = d[f"p{p}_r32_point_count"], d[f"p{p}_r64_point_count"]
            same = np.nonzero(pa == pb)[0]
            assert len(same) >= 0.97 * len(pa)
            ta = {int(i): k for k, i in enumerate(d[f"p{p}_r32_touch_index"])}
            tb = {int(i): k for k, i in enumerate(d[f"p{p}_r64_touch_index"])}
            worst = 0.0
            for i in same:
                if pa[i] == 0:
                    continue
                ka, kb = ta[int(i)], tb[int(i)]
                for j in range(pa[i]):
                    if not np.array_equal(d[f"p{p}_r32_key"][ka, j], d[f"p{p}_r64_key"][kb, j]):
                        continue  # feature choice differs: a tie, counted by the GPU tests
                    e = np.abs(d[f"p{p}_r32_p1"][ka, j] - d[f"p{p}_r64_p1"][kb, j]).max()
                    worst = max(worst, float(e))
            assert worst <= 1e-4, (name, p, worst)


def test_reference_reproduces_triangle_poses(oracle_mod):
    """The committed triangle-pair fixture (tests/golden/make_golden.py
    triangle_poses) is what the reference computes: the pin for the GPU
    triangle tests."""
    O = oracle_mod
    d = G.load("triangle_poses")
    ha = {k: np.ascontiguousarray(d[f"hull_{k}"]) for k in ("desc", "verts", "edges", "faces", "planes", "centroids")}
    hulls = O.RefHulls(ha, 32)
    for i in range(len(d["point_count"])):
        ta, tb = d["type_a"][i], d["type_b"][i]
        m = O.collide(hulls, int(ta[0]), d["shape_a"][i], int(ta[1]), int(tb[0]), d["shape_b"][i], int(tb[1]),
                      d["xf_a"][i], d["xf_b"][i], None, None, None, 32,
                      wingsA=d["wings_a"][i] if ta[0] == 2 else None, wingsB=d["wings_b"][i] if tb[0] == 2 else None)
        pc = int(m["pointCount"])
        assert pc == d["point_count"][i], i
        for f in ("n", "p1", "p2"):
            assert np.array_equal(m["points"][f][:pc].astype(np.float32), d[f][i][:pc]), (i, f)
        assert np.array_equal(m["points"]["key"][:pc], d["key"][i][:pc]), i


def test_fp64_error_statement_triangles_and_meshes(oracle_mod):
    """The reference's FP32 results (which the GPU reproduces bit for bit)
    against its FP64 rerun on a triangle terrain and a mesh terrain: the same
    contacts; where both pick the same features, points within 1e-4 m and
    normals within 1e-3 rad (near-degenerate sphere and capsule contacts turn
    FP32 rounding into a few 1e-4 rad of normal); feature choices that differ
    (ties) stay rare."""
    O = oracle_mod
    from bounce_b200 import scene as S

    def keys(a, b):
        return (np.asarray(a, np.uint64) << np.uint64(32)) | np.asarray(b, np.uint64)

    for name, sc in (("mesh", S.mesh_terrain_scene(seed=5, n=400).finalize()),
                     ("triangles", S.terrain_scene(seed=3, n=400).finalize())):
        r32 = O.RefWorld(sc, precision=32)
        sc.set_local_centers(r32.local_centers())
        r64 = O.RefWorld(sc, precision=64)
        drv = S.KinematicDriver(sc)
        for k in range(3):
            if k:
                drv.advance()
                sw = drv.sweeps14()
                for rw in (r32, r64):
                    rw.set_sweeps(sw)
                    rw.step_pass()
            else:
                r32.first_pass()
                r64.first_pass()
            a, b = r32.contacts(), r64.contacts()
            ka, kb = keys(a["fixtureA"], a["fixtureB"]), keys(b["fixtureA"], b["fixtureB"])
            assert np.array_equal(np.sort(ka), np.sort(kb)), (name, k)
            _, ia, ib = np.intersect1d(ka, kb, return_indices=True)
            worst_p = worst_n = 0.0
            ties = points = 0
            for i, j in zip(ia, ib):
                for m in range(min(a["manifoldCount"][i], b["manifoldCount"][j])):
                    ma, mb = a["manifolds"][i, m], b["manifolds"][j, m]
                    if ma["pointCount"] != mb["pointCount"]:
                        ties += 1
                        continue
                    for q in range(ma["pointCount"]):
                        pa, pb = ma["points"][q], mb["points"][q]
                        if not (np.array_equal(pa["key"], pb["key"]) and pa["triangleKey"] == pb["triangleKey"]):
                            ties += 1
                            continue
                        points += 1
                        worst_p = max(worst_p, float(np.abs(pa["p1"] - pb["p1"]).max()),
                                      float(np.abs(pa["p2"] - pb["p2"]).max()))
                        c = np.dot(pa["n"], pb["n"]) / (np.linalg.norm(pa["n"]) * np.linalg.norm(pb["n"]))
                        worst_n = max(worst_n, float(np.arccos(np.clip(c, -1.0, 1.0))))
            assert points > 100
            assert worst_p <= 1e-4, (name, k, worst_p)
            assert worst_n <= 1e-3, (name, k, worst_n)
            assert ties <= 0.05 * points, (name, k, ties)

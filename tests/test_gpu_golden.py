"""GPU pipeline against the committed golden fixtures (made by running the
reference; see tests/golden/make_golden.py). Needs no reference build on the
GPU box.

* FP32: contact sets, fat AABBs, touching flags, point counts, feature ids,
  hull feature caches and manifold points identical to the reference's FP32
  results (bit for bit).
* FP64: the errors of the GPU manifolds and of the reference's FP32
  manifolds are both stated against the reference's FP64 rerun (point,
  normal angle, separation) and printed; the GPU's error may not exceed the
  reference's. Contacts whose point count or feature ids differ from the
  FP64 run (SAT axis ties) are counted and reported. The pipeline's own
  tolerance (|dpoint| <= 1e-4 m, normal angle <= 1e-4 rad, |dseparation| <=
  1e-5 m against the FP32 reference) is met with zero error: results are
  bit-identical.
"""
import numpy as np
import pytest

from bounce_b200 import _native as N
from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline
from tests import golden_util as G

pytestmark = pytest.mark.gpu

TOL_POINT = 1e-4
TOL_ANGLE = 1e-4
TOL_SEP = 1e-5


def quat_rot(q, v):
    qv, s = q[..., :3], q[..., 3:4]
    t = 2.0 * np.cross(qv, v)
    return v + s * t + np.cross(qv, t)


@pytest.mark.parametrize("name", G.SCENES)
def test_pipeline_matches_golden(name):
    d = G.load(name)
    sc = G.scene_from(d)
    pipe = CollisionPipeline(sc)
    report = []
    for p in range(G.PASSES):
        pipe.collide(np.ascontiguousarray(d[f"p{p}_state"]))
        assert pipe.counts()["status"] == 0
        assert np.array_equal(pipe.fat_aabbs(), d[f"p{p}_r32_fat"]), f"pass {p}: fat AABBs"
        g = pipe.contacts()
        order = np.argsort(G.contact_keys(g))
        g = g[order]
        ref = d[f"p{p}_r32_pairs"]
        assert np.array_equal(g[:, :2], ref[:, :2]), f"pass {p}: contact sets"
        assert np.array_equal(g[:, 2] & 1, ref[:, 2] & 1), f"pass {p}: touching flags"
        man = pipe.manifolds()[order]
        pc = np.where((g[:, 2] >> 8) & 0xFF, man["pointCount"], 0)
        assert np.array_equal(pc, d[f"p{p}_r32_point_count"]), f"pass {p}: point counts"
        rcache = d[f"p{p}_r32_cache"]
        hh = rcache[:, 0] != 0xFFFFFFFF  # hull-hull contacts
        assert np.array_equal(pipe.caches()[order][hh], rcache[hh]), f"pass {p}: feature caches"
        ti = d[f"p{p}_r32_touch_index"]
        pts = man["points"][ti]
        mask = np.arange(4)[None, :] < pc[ti][:, None]
        for f in ("n", "p1", "p2"):
            assert np.array_equal(pts[f][mask], d[f"p{p}_r32_{f}"][mask]), f"pass {p}: {f}"
        assert np.array_equal(pts["key"][mask], d[f"p{p}_r32_key"][mask]), f"pass {p}: feature ids"

        # Error statement against the FP64 rerun.
        pc64 = d[f"p{p}_r64_point_count"]
        ti64 = {int(i): k for k, i in enumerate(d[f"p{p}_r64_touch_index"])}
        state = d[f"p{p}_state"].reshape(-1, 17)
        ties = 0
        worst_gpu = np.zeros(3)
        worst_ref = np.zeros(3)
        for k, i in enumerate(ti):
            if pc64[i] != pc[i] or int(i) not in ti64:
                ties += 1
                continue
            k64 = ti64[int(i)]
            if not np.array_equal(pts["key"][k, : pc[i]], d[f"p{p}_r64_key"][k64, : pc[i]]):
                ties += 1
                continue
            A, B = g[i, 0], g[i, 1]
            xa, xb = state[sc.fix_body[A]].astype(np.float64), state[sc.fix_body[B]].astype(np.float64)

            def sep(nl, p1, p2):
                nw = quat_rot(xa[3:7], nl)
                ca = quat_rot(xa[3:7], p1) + xa[0:3]
                cb = quat_rot(xb[3:7], p2) + xb[0:3]
                return np.dot(cb - ca, nw)

            def err(n, p1, p2, j):
                n, p1, p2 = (np.asarray(x, np.float64) for x in (n, p1, p2))
                n64 = d[f"p{p}_r64_n"][k64, j].astype(np.float64)
                q1 = d[f"p{p}_r64_p1"][k64, j].astype(np.float64)
                q2 = d[f"p{p}_r64_p2"][k64, j].astype(np.float64)
                ang = np.arccos(np.clip(np.dot(n, n64) / (np.linalg.norm(n) * np.linalg.norm(n64)), -1, 1))
                dp = max(np.abs(p1 - q1).max(), np.abs(p2 - q2).max())
                ds = abs(sep(n, p1, p2) - sep(n64, q1, q2))
                return np.array([dp, ang, ds])

            for j in range(pc[i]):
                worst_gpu = np.maximum(worst_gpu, err(pts["n"][k, j], pts["p1"][k, j], pts["p2"][k, j], j))
                worst_ref = np.maximum(worst_ref, err(d[f"p{p}_r32_n"][k, j], d[f"p{p}_r32_p1"][k, j],
                                                      d[f"p{p}_r32_p2"][k, j], j))
        report.append((p, len(ti), ties, worst_gpu, worst_ref))
        assert np.all(worst_gpu <= worst_ref), (p, worst_gpu, worst_ref)
        assert ties <= max(2, 0.02 * len(ti)), (p, ties)
    pipe.close()
    for p, n, t, wg, wr in report:
        print(f"{name} pass {p}: {n} touching, {t} SAT ties vs FP64; worst vs FP64 (point m, normal rad, "
              f"separation m): GPU {wg.tolist()} reference FP32 {wr.tolist()}")


def test_collide_pairs_matches_reference_poses():
    """b3g_collide_pairs on the testbed poses and seeded random poses of every
    convex pair type, against the reference's b3Collide* results."""
    d = G.load("collide_poses")
    sc = S.Scene()
    hull_arrays = {k: np.ascontiguousarray(d[f"hull_{k}"]) for k in
                   ("desc", "verts", "edges", "faces", "planes", "centroids")}
    # One fixture (on its own dynamic body) per distinct shape.
    shapes = {}
    fa, fb = [], []
    for i in range(len(d["point_count"])):
        for side, (t, sp) in enumerate(((d["type_a"][i], d["shape_a"][i]), (d["type_b"][i], d["shape_b"][i]))):
            key = (int(t[0]), int(t[1]), sp.tobytes())
            if key not in shapes:
                b = sc.add_body(0, N.BODY_DYNAMIC, (0, 0, 0), (0, 0, 0, 1))
                shapes[key] = sc.add_fixture(b, int(t[0]), sp, hull=int(t[1]))
            (fa if side == 0 else fb).append(shapes[key])
    sc.finalize(hull_arrays)
    pipe = CollisionPipeline(sc)
    cache = np.tile(np.array([0, 1, 0, 0], np.uint32), (len(fa), 1))
    man = pipe.collide_pairs(fa, fb, d["xf_a"], d["xf_b"], d["xf_a"], d["xf_b"], cache)
    assert np.array_equal(man["pointCount"], d["point_count"])
    mask = np.arange(4)[None, :] < d["point_count"][:, None]
    for f in ("n", "p1", "p2"):
        assert np.array_equal(man["points"][f][mask], d[f].astype(np.float32)[mask]), f
    assert np.array_equal(man["points"]["key"][mask], d["key"][mask])
    hh = (d["type_a"][:, 0] == 3) & (d["type_b"][:, 0] == 3)
    assert np.array_equal(cache[hh], d["cache_out"][hh])
    pipe.close()

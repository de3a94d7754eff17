"""CPU check of the solver-input oracle: the records the reference's own
b3ContactSolver constructor and InitializeVelocityConstraints produce
(oracle/ref_harness.cpp refw_contact_solver, which the GPU tests compare
against word for word) agree with an independent float64 restatement of
contact_solver.cpp:28-305 and collision.cpp:63-101 computed here from the
reference's manifolds, within float32 rounding. This pins the record layout
(include/b3g.h) and the reading of the algorithm the device kernel follows.
"""
import numpy as np

from bounce_b200 import _native as N
from bounce_b200 import scene as S


def rotate(q, v):
    """Rotate v by the unit quaternion q (xyzw), float64."""
    u, s = q[..., :3], q[..., 3:4]
    t = 2.0 * np.cross(u, v)
    return v + s * t + np.cross(u, t)


def perp(n):
    """b3Perp (vec3.h:243-259)."""
    out = np.where(np.abs(n[..., :1]) >= np.sqrt(1.0 / 3.0),
                   np.stack([n[..., 1], -n[..., 0], np.zeros_like(n[..., 0])], -1),
                   np.stack([np.zeros_like(n[..., 0]), n[..., 2], -n[..., 1]], -1))
    return out / np.linalg.norm(out, axis=-1, keepdims=True)


def test_reference_solver_records_match_restatement(oracle_mod):
    O = oracle_mod
    sc = S.mixed_scene(seed=41, n=1200, side=11.0, static_frac=0.05, sensor_frac=0.03).finalize()
    rw = O.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    rw.first_pass()
    rng = np.random.default_rng(3)
    n = sc.n_bodies
    sweeps = drv.sweeps14().reshape(-1, 14)
    inv_mass, _, world_inv_i = rw.mass_data()
    b = np.zeros(n, N.SOLVER_BODY_DTYPE)
    b["x"], b["q"] = sweeps[:, 7:10], sweeps[:, 10:14]
    b["v"] = rng.normal(0.0, 3.0, (n, 3))
    b["w"] = rng.normal(0.0, 2.0, (n, 3))
    b["invMass"], b["invI"] = inv_mass, world_inv_i
    b["localCenter"] = np.asarray(rw.local_centers(), np.float32).reshape(-1, 3)
    fr = rng.uniform(0, 1, sc.n_fixtures).astype(np.float32)
    re = rng.uniform(0, 1, sc.n_fixtures).astype(np.float32)
    dt_ratio = 0.8
    rcon, rman = rw.contact_solver(b.view(np.float32).reshape(-1, 28), fr, re, dt_ratio=dt_ratio)
    con = rcon.view(N.CONTACT_CONSTRAINT_DTYPE).reshape(-1)
    man = rman.view(N.MANIFOLD_CONSTRAINT_DTYPE).reshape(-1)

    cl = rw.contacts()
    touching = (cl["flags"] & 1) == 1
    sensor = ((sc.fix_flags[cl["fixtureA"]] | sc.fix_flags[cl["fixtureB"]]) & 1) == 1
    sel = np.nonzero(touching & ~sensor)[0]
    assert np.array_equal(con["contact"], sel) and len(sel) > 300
    assert np.array_equal(con["manifoldStart"], np.concatenate([[0], np.cumsum(con["manifoldCount"])[:-1]]))

    f64 = lambda a: np.asarray(a, np.float64)
    bodies = {k: f64(b[k]) for k in ("x", "q", "v", "w", "invMass", "localCenter")}
    inv_i = f64(b["invI"]).reshape(-1, 3, 3).transpose(0, 2, 1)  # rows from the stored columns
    close = lambda a, e, tol=2e-4: np.allclose(a, e, rtol=tol, atol=tol * (1.0 + np.abs(e).max()))
    for k, c in enumerate(con):
        rec = cl[c["contact"]]
        fa, fb = rec["fixtureA"], rec["fixtureB"]
        A, B = sc.fix_body[fa], sc.fix_body[fb]
        assert (c["indexA"], c["indexB"]) == (A, B)
        assert c["friction"] == np.float32(np.sqrt(np.float32(fr[fa] * fr[fb])))
        assert c["restitution"] == max(re[fa], re[fb])
        assert c["invMassA"] == b["invMass"][A] and np.array_equal(c["invIA"], b["invI"][A])
        xA, xB = bodies["x"][A], bodies["x"][B]
        qA, qB = bodies["q"][A], bodies["q"][B]
        pA0 = xA - rotate(qA, bodies["localCenter"][A])
        pB0 = xB - rotate(qB, bodies["localCenter"][B])
        mA, mB = bodies["invMass"][A], bodies["invMass"][B]
        iA, iB = inv_i[A], inv_i[B]
        for j in range(c["manifoldCount"]):
            mc = man[c["manifoldStart"] + j]
            dm = rec["manifolds"][j]
            pc = int(dm["pointCount"])
            assert mc["pointCount"] == pc and mc["constraint"] == k
            assert np.allclose(mc["tangentImpulse"], dt_ratio * dm["tangentImpulse"], rtol=1e-6)
            if pc == 0:
                continue
            pts = dm["points"][:pc]
            nA = rotate(qA, pts["n"])
            cA = rotate(qA, pts["p1"]) + pA0
            cB = rotate(qB, pts["p2"]) + pB0
            point = 0.5 * ((cA + c["radiusA"] * nA) + (cB - c["radiusB"] * nA))
            center = point.mean(0)
            normal = nA.sum(0)
            normal /= np.linalg.norm(normal)
            assert close(mc["normal"], normal)
            assert close(mc["rA"], center - xA) and close(mc["rB"], center - xB)
            if abs(abs(normal[0]) - np.sqrt(1.0 / 3.0)) > 1e-4:
                t1 = perp(normal)
                assert close(mc["tangent1"], t1) and close(mc["tangent2"], np.cross(t1, normal))
            for q in range(pc):
                vp = mc["points"][q]
                rA, rB = point[q] - xA, point[q] - xB
                assert close(vp["rA"], rA) and close(vp["rB"], rB)
                rnA, rnB = np.cross(rA, nA[q]), np.cross(rB, nA[q])
                K = mA + mB + rnA @ iA @ rnA + rnB @ iB @ rnB
                assert close(vp["normalMass"], 1.0 / K if K > 0 else 0.0)
                dv = bodies["v"][B] + np.cross(bodies["w"][B], rB) - bodies["v"][A] - np.cross(bodies["w"][A], rA)
                vn = nA[q] @ dv
                if abs(vn + 1.0) > 1e-3:
                    bias = -c["restitution"] * vn if vn < -1.0 else 0.0
                    assert close(vp["velocityBias"], bias, 1e-3)
                assert np.isclose(vp["normalImpulse"], dt_ratio * pts["normalImpulse"][q], rtol=1e-6)
                pp = mc["positionPoints"][q]
                assert np.array_equal(pp["localNormalA"], pts["n"][q].astype(np.float32))
            twist = mc["normal"].astype(np.float64) @ (iA + iB) @ mc["normal"].astype(np.float64)
            if twist > 1e-6:
                assert close(mc["motorMass"], 1.0 / twist, 1e-3)

"""Solver input on the GPU (b3g_contact_constraints) against the reference's
own b3ContactSolver constructor and InitializeVelocityConstraints
(contact_solver.cpp:28-149, :177-305) run on the reference world after the
same collision passes, bit for bit: every word of every contact constraint
(bodies, masses, inertias, mixed friction and restitution, radii) and of
every manifold constraint (world-manifold centre, normal and tangents,
tangent and twist masses, warm-start impulses; per point the anchors,
normal mass, impulse and restitution bias; the position-constraint points).

Scenes: spheres, capsules and hulls with static bodies and sensors (the
default selection skips sensor contacts), and a mesh terrain (up to three
manifolds per contact), with the solver's impulses handed back between
passes so the warm-start terms are not zero; the default contact selection
and a caller's list (a shuffled subset, as an island would order it), with
and without warm starting.
"""
import numpy as np
import pytest

from bounce_b200 import _native as N
from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline

pytestmark = pytest.mark.gpu


def solver_bodies(rw, drv, rng, random_mass=False):
    """One b3g_solver_body per body: the pass's centre of mass and
    orientation, random velocities (large enough that some approach speeds
    pass B3_VELOCITY_THRESHOLD), and the reference's mass data (or random
    positive masses and inertias)."""
    sweeps = drv.sweeps14().reshape(-1, 14)
    n = len(sweeps)
    inv_mass, _, world_inv_i = rw.mass_data()
    b = np.zeros(n, N.SOLVER_BODY_DTYPE)
    b["x"] = sweeps[:, 7:10]
    b["q"] = sweeps[:, 10:14]
    b["v"] = rng.normal(0.0, 3.0, (n, 3))
    b["w"] = rng.normal(0.0, 2.0, (n, 3))
    b["localCenter"] = np.asarray(rw.local_centers(), np.float32).reshape(-1, 3)
    if random_mass:
        dyn = inv_mass > 0
        b["invMass"] = np.where(dyn, rng.uniform(0.1, 2.0, n), 0.0)
        a = rng.normal(0.0, 1.0, (n, 3, 3)).astype(np.float32)
        spd = np.einsum("nij,nkj->nik", a, a) + np.eye(3, dtype=np.float32)
        b["invI"] = np.where(dyn[:, None], spd.reshape(n, 9), 0.0)
    else:
        b["invMass"] = inv_mass
        b["invI"] = world_inv_i
    return b


def compare(pipe, rw, bodies, fr, re, label, contacts=None, dt_ratio=1.0, warm=True):
    con, man = pipe.contact_constraints(bodies, dt_ratio=dt_ratio, warm=warm, contacts=contacts)
    rcon, rman = rw.contact_solver(bodies.view(np.float32).reshape(-1, 28), fr, re, dt_ratio=dt_ratio, warm=warm,
                                   contacts=contacts)
    assert len(con) == len(rcon), f"{label}: {len(con)} constraints vs {len(rcon)}"
    assert len(man) == len(rman), f"{label}: {len(man)} manifolds vs {len(rman)}"
    gc = con.view(np.uint32).reshape(-1, 32)
    bad = np.nonzero(~np.all(gc == rcon, axis=1))[0]
    assert len(bad) == 0, (f"{label}: contact constraint {bad[0]} differs:\n{con[bad[0]]}\n"
                           f"{rcon[bad[0]].view(N.CONTACT_CONSTRAINT_DTYPE)}")
    gm = man.view(np.uint32).reshape(-1, 116)
    bad = np.nonzero(~np.all(gm == rman, axis=1))[0]
    if len(bad):
        i = bad[0]
        words = np.nonzero(gm[i] != rman[i])[0]
        raise AssertionError(f"{label}: manifold constraint {i} differs in words {words[:12]}:\n{man[i]}\n"
                             f"{rman[i].view(N.MANIFOLD_CONSTRAINT_DTYPE)}")
    return con, man


def run(O, sc, passes, check, impulses=False, seed=0):
    rw = O.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    rng = np.random.default_rng(seed)
    for k in range(passes):
        if k:
            if impulses:
                n = pipe.counts()["contacts"]
                normal = rng.uniform(0, 5, (n, 3, 4)).astype(np.float32)
                tangent = rng.uniform(-1, 1, (n, 3, 2)).astype(np.float32)
                motor = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
                rw.load_impulses(normal, tangent, motor)
                pipe.load_impulses(normal[:, 0], tangent[:, 0], motor[:, 0])
                pipe.load_mesh_impulses(normal[:, 1:], tangent[:, 1:], motor[:, 1:])
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
        assert pipe.counts()["status"] == 0
        check(k, rw, pipe, drv, rng)
    pipe.close()


def test_solver_input_mixed_shapes(oracle_mod):
    sc = S.mixed_scene(seed=41, n=2500, side=15.0, static_frac=0.05, sensor_frac=0.03).finalize()
    nf = sc.n_fixtures
    seen = {"constraints": 0, "bias": 0, "sensor_skipped": 0}

    def check(k, rw, pipe, drv, rng):
        fr = rng.uniform(0.0, 1.0, nf).astype(np.float32)
        re = rng.uniform(0.0, 1.0, nf).astype(np.float32)
        pipe.set_materials(fr, re)
        bodies = solver_bodies(rw, drv, rng, random_mass=(k % 2 == 1))
        con, man = compare(pipe, rw, bodies, fr, re, f"pass {k}")
        seen["constraints"] += len(con)
        seen["bias"] += int(np.sum(man["points"]["velocityBias"] != 0))
        c = pipe.contacts()
        touching = (c[:, 2] & 1) == 1
        sensor = ((sc.fix_flags[c[:, 0]] | sc.fix_flags[c[:, 1]]) & 1) == 1
        seen["sensor_skipped"] += int(np.sum(touching & sensor))
        assert len(con) == int(np.sum(touching & ~sensor))
        # a caller's order: a shuffled subset of the touching contacts
        sel = np.nonzero(touching & ~sensor)[0]
        sub = rng.permutation(sel)[: max(1, len(sel) // 2)]
        compare(pipe, rw, bodies, fr, re, f"pass {k} list", contacts=sub, dt_ratio=0.75, warm=(k % 2 == 0))

    run(oracle_mod, sc, 4, check, impulses=True, seed=5)
    assert seen["constraints"] > 1000 and seen["bias"] > 100 and seen["sensor_skipped"] > 0, seen


def test_solver_input_mesh_terrain(oracle_mod):
    sc = S.mesh_terrain_scene(seed=6, n=500, scale=(1.1, 0.9, 1.2)).finalize()
    nf = sc.n_fixtures
    seen = {"multi": 0, "manifolds": 0}

    def check(k, rw, pipe, drv, rng):
        fr = rng.uniform(0.0, 1.0, nf).astype(np.float32)
        re = rng.uniform(0.0, 1.0, nf).astype(np.float32)
        pipe.set_materials(fr, re)
        bodies = solver_bodies(rw, drv, rng)
        con, man = compare(pipe, rw, bodies, fr, re, f"mesh pass {k}")
        seen["multi"] += int(np.sum(con["manifoldCount"] > 1))
        seen["manifolds"] += len(man)
        assert np.array_equal(np.repeat(np.arange(len(con)), con["manifoldCount"]), man["constraint"])
        compare(pipe, rw, bodies, fr, re, f"mesh pass {k} cold", warm=False)

    run(oracle_mod, sc, 6, check, impulses=True, seed=9)
    assert seen["multi"] > 0 and seen["manifolds"] > 200, seen


def test_solver_input_device_entry_point(oracle_mod):
    """b3g_contact_constraints_device on device buffers gives the host entry
    point's records, with capacities smaller than the totals honoured and the
    totals still reported."""
    import ctypes

    import torch

    sc = S.mixed_scene(seed=43, n=1500, side=12.0).finalize()
    rw = oracle_mod.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    rw.first_pass()
    pipe.collide(drv.state17())
    rng = np.random.default_rng(2)
    bodies = solver_bodies(rw, drv, rng)
    con, man = pipe.contact_constraints(bodies)
    assert len(con) > 100
    d_bodies = torch.from_numpy(bodies.view(np.uint8).copy()).cuda()
    cap_c, cap_m = len(con) // 2, len(man) // 3
    d_con = torch.zeros(cap_c * 128, dtype=torch.uint8, device="cuda")
    d_man = torch.zeros(cap_m * 464, dtype=torch.uint8, device="cuda")
    d_counts = torch.zeros(2, dtype=torch.int32, device="cuda")
    pipe._check(pipe.lib.b3g_contact_constraints_device(
        pipe.ctx, 0, None, ctypes.c_void_p(d_bodies.data_ptr()), 1.0, 1, ctypes.c_void_p(d_con.data_ptr()), cap_c,
        ctypes.c_void_p(d_man.data_ptr()), cap_m, ctypes.c_void_p(d_counts.data_ptr()), None))
    torch.cuda.synchronize()
    assert d_counts.cpu().numpy().tolist() == [len(con), len(man)]
    assert np.array_equal(d_con.cpu().numpy().view(N.CONTACT_CONSTRAINT_DTYPE).view(np.uint32),
                          con[:cap_c].view(np.uint32))
    assert np.array_equal(d_man.cpu().numpy().view(N.MANIFOLD_CONSTRAINT_DTYPE).view(np.uint32),
                          man[:cap_m].view(np.uint32))
    with pytest.raises(N.B3GError):
        pipe.contact_constraints(bodies, contacts=np.array([pipe.counts()["contacts"]], np.uint32))
    pipe.close()

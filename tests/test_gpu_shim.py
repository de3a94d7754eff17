"""The reference-side shim, compiled and run: Bounce with its contact manager
replaced by bounce_b200/shim/b3g_contact_manager.cpp (the collision pass on
the device through the C ABI) steps b3World::Step with the reference's own
solver, islands and sleep, and must stay bit-identical to the stock Bounce
build: body transforms and sweeps, awake flags, the contact list in list
order, and every manifold with the solver's impulses, after every step.

Both builds come from the unmodified reference sources (oracle/Makefile:
libb3ref32.so and libb3shim.so, the latter without contact_manager.cpp).
"""
import numpy as np
import pytest

from bounce_b200 import scene as S

pytestmark = pytest.mark.gpu

F = np.float32


def falling_scene(seed=41):
    """Boxes and spheres over a ground box, with capsules and hulls dropped
    from above: they fall, collide, pile up and some fall asleep."""
    s = S.plain_scene(seed=seed, n_boxes=200, n_spheres=200, cube=8.0)
    b0 = len(s.body_type)
    S.mixed_scene(seed=seed + 2, n=200, side=6.0, scene=s)
    for i in range(b0, len(s.body_type)):
        p = np.asarray(s.body_pos[i], F)
        s.body_pos[i] = (p + np.array([0.0, 12.0, 0.0], F)).astype(F)
    for i in range(len(s.body_type)):
        s.body_lin[i] = (F(0.1) * np.asarray(s.body_lin[i], F)).astype(F)
        s.body_ang[i] = (F(0.1) * np.asarray(s.body_ang[i], F)).astype(F)
    return s.finalize()


def compare_worlds(ref, shim, label):
    rb, sb = ref.bodies17(), shim.bodies17()
    bad = np.nonzero(np.any(rb.reshape(-1, 17) != sb.reshape(-1, 17), axis=1))[0]
    assert len(bad) == 0, f"{label}: {len(bad)} bodies differ, first {bad[:5]}"
    assert np.array_equal(ref.awake(), shim.awake()), f"{label}: awake flags differ"
    rp, sp = ref.pairs(), shim.pairs()
    # The reference's Solve ends with FindNewContacts (world.cpp:424-449): the
    # contacts it creates wait, without manifolds, for the next step's
    # UpdateContacts. The shim creates them in that step's device pass, at
    # the same places of the list. Between steps they are the only difference.
    rk = (rp[:, 0].astype(np.uint64) << np.uint64(32)) | rp[:, 1]
    sk = (sp[:, 0].astype(np.uint64) << np.uint64(32)) | sp[:, 1]
    kept = np.isin(rk, sk)
    fresh = rp[~kept]
    assert np.all((fresh[:, 2] & 0xFF01) == 0), f"{label}: contacts missing from the shim's list were updated"
    rp = rp[kept]
    assert len(rp) == len(sp), f"{label}: {len(sp)} contacts vs {len(rp)}"
    assert np.array_equal(rp[:, :2], sp[:, :2]), f"{label}: contact list order differs"
    assert np.array_equal(rp[:, 2] & 0xFF01, sp[:, 2] & 0xFF01), f"{label}: contact flags differ"
    rc, sc = ref.contacts()[kept], shim.contacts()
    assert np.array_equal(rc["manifoldCount"], sc["manifoldCount"]), f"{label}: manifold counts differ"
    rm, sm = rc["manifolds"][:, 0], sc["manifolds"][:, 0]
    pc = np.where(rc["manifoldCount"] > 0, rm["pointCount"], 0)
    assert np.array_equal(pc, np.where(sc["manifoldCount"] > 0, sm["pointCount"], 0)), f"{label}: point counts"
    mask = np.arange(4)[None, :] < pc[:, None]
    for f in ("n", "p1", "p2", "normalImpulse", "key"):
        assert np.array_equal(rm["points"][f][mask], sm["points"][f][mask]), f"{label}: manifold {f} differs"
    has = pc > 0
    for f in ("tangentImpulse", "motorImpulse"):
        assert np.array_equal(rm[f][has], sm[f][has]), f"{label}: {f} differs"
    return len(rp), int(np.count_nonzero(rp[:, 2] & 1))


def run_steps(oracle_mod, sc, steps, filter_modulus=0):
    ref = oracle_mod.RefWorld.stepping(sc, 32)
    shim = oracle_mod.RefWorld.stepping(sc, "shim")
    if filter_modulus:
        ref.set_filter(filter_modulus, 1)
        shim.set_filter(filter_modulus, 1)
    touching = asleep = 0
    for k in range(steps):
        ref.step()
        shim.step()
        _, t = compare_worlds(ref, shim, f"step {k}")
        touching = max(touching, t)
        asleep = max(asleep, int(np.count_nonzero(ref.awake() == 0)))
    assert oracle_mod.lib("shim").b3g_shim_failures() == 0
    ref.close()
    shim.close()
    return touching, asleep


def test_world_step_with_gpu_contacts_matches_stock_bounce(oracle_mod):
    sc = falling_scene()
    touching, asleep = run_steps(oracle_mod, sc, 300)
    assert touching > 300, touching
    assert asleep > 10, asleep


def test_world_step_with_contact_filter(oracle_mod):
    """The world's b3ContactFilter goes through the device's filter round trip."""
    sc = falling_scene(seed=47)
    touching, _ = run_steps(oracle_mod, sc, 60, filter_modulus=4)
    assert touching > 100, touching

"""GPU parity at the sizes the benchmark is quoted on, against the reference's
own FP32 collision pass (oracle/_ref), bit for bit:

* the benchmark's 65,536-body mixed world itself (same seed, cube, capacity,
  wall-reflected motion and centres of mass as `bench.py`), pass after pass:
  fat AABBs, contact list in list order, destroyed contacts, touching flags,
  manifolds, feature ids, impulses and hull feature caches;
* the 1,024-world batched scene (worlds of 16-4,096 bodies in one context),
  a sample of 130 worlds compared world by world with one reference world
  each;
* a hull pile of 16,384 hulls (128 columns of 128) over the benchmark pile's
  full 512 x 512-vertex mesh ground.

These runs reach what smaller scenes do not: leaves with more overlaps than
their scratch slots (the traversal's overflow list), many worlds sharing one
tree with wide ground proxies sorted last in each world, the hash and contact
capacities the benchmark sizes, and the mesh midphase on a 522,242-triangle
tree.
"""
import numpy as np
import pytest

import bench
from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline
from tests.parity import (BatchedPass, WorldView, compare_contacts, compare_ended, compare_fat_aabbs,
                          compare_order)

pytestmark = pytest.mark.gpu


def test_mixed_65536_benchmark_world(oracle_mod):
    sc = bench.build_scene(bench.N_BODIES, bench.SEED)
    walls = bench.scene_half(sc)
    rw = oracle_mod.RefWorld(sc)
    rw.set_local_centers(sc.local_center)  # as the benchmark drives the reference
    drv = S.KinematicDriver(sc, walls=walls)
    pipe = CollisionPipeline(sc, max_contacts=max(2_000_000, 40 * sc.n_bodies))
    prev = None
    overflow = 0
    for k in range(6):
        if k:
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
        c = pipe.counts()
        assert c["status"] == 0, c
        label = f"mixed-65536 pass {k}"
        compare_fat_aabbs(pipe, rw, label)
        st = compare_contacts(pipe, rw, label)
        compare_order(pipe, rw, label)
        cur = rw.pairs()
        if prev is not None:
            compare_ended(pipe, prev, cur, label)
        prev = cur
        overflow = max(overflow, pipe.pass_stats()["trav_overflow"])
    assert st["contacts"] > 600_000 and st["touching"] > 120_000, st
    print("mixed-65536 last pass:", st, "largest traversal overflow list:", overflow)
    pipe.close()
    rw.close()


def test_batched_1024_worlds_against_reference(oracle_mod):
    sc, counts = S.batched_scene(seed=3, n_worlds=1024, lo=16, hi=4096, cube=20.0)
    sc.finalize()
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    sample = sorted(set(range(0, 1024, 8)) | {int(np.argmin(counts)), int(np.argmax(counts))})
    worlds = []
    for w in sample:
        sub, bodies, fixtures = sc.world_subset(w)
        rw = oracle_mod.RefWorld(sub)
        rw.set_local_centers(sub.local_center)
        worlds.append((w, rw, fixtures))
    prev = {}
    touching = 0
    for k in range(4):
        if k:
            drv.advance()
        pipe.collide(drv.state17())
        assert pipe.counts()["status"] == 0
        bp = BatchedPass(pipe, sc)
        sw = drv.sweeps14().reshape(-1, 14)
        touching = 0
        for w, rw, fixtures in worlds:
            if k:
                rw.set_sweeps(np.ascontiguousarray(sw[sc.body_world == w].reshape(-1)))
                rw.step_pass()
            else:
                rw.first_pass()
            view = WorldView(bp, w, fixtures)
            label = f"batched pass {k} world {w} ({counts[w]} bodies)"
            compare_fat_aabbs(view, rw, label)
            touching += compare_contacts(view, rw, label)["touching"]
            compare_order(view, rw, label)
            cur = rw.pairs()
            if w in prev:
                compare_ended(view, prev[w], cur, label)
            prev[w] = cur
    assert len(worlds) >= 128 and touching > 10_000, touching
    for _, rw, _ in worlds:
        rw.close()
    pipe.close()


def test_pile_over_full_mesh_ground(oracle_mod):
    sc = S.pile_scene(seed=bench.PILE_SEED, columns=128, per_column=128, grid=512).finalize()
    rw = oracle_mod.RefWorld(sc)
    rw.set_local_centers(sc.local_center)
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc, max_contacts=4 * sc.n_bodies)
    prev = None
    for k in range(10):
        if k:
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
        assert pipe.counts()["status"] == 0
        label = f"pile-16384 pass {k}"
        compare_fat_aabbs(pipe, rw, label)
        st = compare_contacts(pipe, rw, label)
        compare_order(pipe, rw, label)
        cur = rw.pairs()
        if prev is not None:
            compare_ended(pipe, prev, cur, label)
        prev = cur
    stats = pipe.pass_stats()
    assert stats["mesh_items"] > 0 and st["touching"] > 10_000, (stats, st)
    print("pile-16384 last pass:", st, stats)
    pipe.close()
    rw.close()

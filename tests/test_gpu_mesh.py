"""Triangle meshes on the GPU against the reference, bit for bit:

* the edge wings that b3g_set_meshes builds equal b3Mesh::BuildAdjacency's
  (mesh.cpp:36-119), on two meshes in one upload, one of them with
  non-manifold edges (three triangles on one edge), and
* collision passes of spheres, capsules and hulls over a static mesh terrain
  (b3MeshContact, mesh_contact.cpp): contact list (order included), fat AABBs,
  manifold counts, every manifold's points and ids (triangle keys included).
"""
import numpy as np
import pytest

from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline
from tests.parity import compare_contacts, compare_fat_aabbs
from tests.parity import compare_order

pytestmark = pytest.mark.gpu


def two_meshes(seed=11):
    """A grid terrain and a small mesh whose triangles repeat one edge three
    times and come in a shuffled order."""
    rng = np.random.default_rng(seed)
    v0, t0 = S.grid_mesh(9, 7, 1.0, seed)
    v1, t1 = S.grid_mesh(4, 4, 0.5, seed + 1)
    t1 = np.concatenate([t1, t1[:2, ::-1], t1[3:4]])  # duplicated triangles: non-manifold edges
    t1 = t1[rng.permutation(len(t1))]
    desc = np.array([0, len(v0), 0, len(t0), len(v0), len(v1), len(t0), len(t1)], np.uint32)
    verts = np.concatenate([v0, v1]).reshape(-1).astype(np.float32)
    tris = np.concatenate([t0, t1]).reshape(-1).astype(np.uint32)
    return dict(desc=desc, verts=verts, tris=tris), (len(t0), len(t1))


def test_mesh_adjacency_matches_reference(oracle_mod):
    arrays, counts = two_meshes()
    sc = S.Scene()
    sc.mesh_arrays = arrays
    g = sc.add_body(0, S.N.BODY_STATIC, (0, 0, 0), (0, 0, 0, 1))
    sc.add_fixture(g, S.N.SHAPE_MESH, [1.0, 1.0, 1.0, 0.0], hull=0)
    sc.add_fixture(g, S.N.SHAPE_MESH, [2.0, 1.0, 0.5, 0.0], hull=1)
    sc.finalize()
    ref = oracle_mod.RefHulls(sc.hull_arrays, mesh_arrays=arrays)
    pipe = CollisionPipeline(sc)
    for m, n in enumerate(counts):
        assert np.array_equal(pipe.mesh_wings(m, n), ref.mesh_wings(m, n)), f"mesh {m}"
    pipe.close()


@pytest.mark.parametrize("scale", [(1.0, 1.0, 1.0), (1.3, 0.8, 0.9)])
def test_mesh_terrain_passes_match_reference(oracle_mod, scale):
    sc = S.mesh_terrain_scene(seed=5, n=600, scale=scale).finalize()
    rw = oracle_mod.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    multi = 0
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
        compare_fat_aabbs(pipe, rw, f"mesh pass {k}")
        compare_contacts(pipe, rw, f"mesh pass {k}")
        compare_order(pipe, rw, f"mesh pass {k}")
        c = pipe.contacts()
        mc = (c[:, 2] >> 8) & 0xFF
        multi += int(np.sum(mc > 1))
        touching = c[(c[:, 2] & 1) == 1]
        kinds |= set(zip(sc.fix_type[touching[:, 0]].tolist(), sc.fix_type[touching[:, 1]].tolist()))
    assert {(4, 0), (4, 1), (3, 4)} <= kinds, kinds
    assert multi > 0
    pipe.close()


def test_hull_pile_passes_match_reference(oracle_mod):
    """A small hull-heavy pile (hulls of 12-64 vertices stacked in columns over
    a sines mesh ground) settling for 10 passes."""
    sc = S.pile_scene(seed=4, columns=4, per_column=64, grid=48).finalize()
    rw = oracle_mod.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    touching = []
    for k in range(10):
        if k:
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            rw.step_pass()
        else:
            rw.first_pass()
        pipe.collide(drv.state17())
        assert pipe.counts()["status"] == 0
        compare_fat_aabbs(pipe, rw, f"pile pass {k}")
        touching.append(compare_contacts(pipe, rw, f"pile pass {k}")["touching"])
        compare_order(pipe, rw, f"pile pass {k}")
    assert touching[-1] > 150, touching
    pipe.close()


def test_warm_start_from_solver_impulses(oracle_mod):
    """Impulses handed back after each pass (b3g_load_impulses for manifold 0,
    b3g_load_mesh_impulses for manifolds 1 and 2) warm-start the next pass's
    matching points exactly as in the reference, on convex, hull and mesh
    contacts."""
    sc = S.mesh_terrain_scene(seed=8, n=500).finalize()
    rw = oracle_mod.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    rng = np.random.default_rng(1)
    persisting = 0
    for k in range(8):
        if k:
            n = pipe.counts()["contacts"]
            assert n == rw.contact_count()
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
        compare_contacts(pipe, rw, f"warm pass {k}")
        compare_order(pipe, rw, f"warm pass {k}")
        _, man = pipe.touching()
        persisting += int(np.sum(man["points"]["persisting"]))
    assert persisting > 100
    pipe.close()

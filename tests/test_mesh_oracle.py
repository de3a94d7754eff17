"""The oracle's mesh adjacency (b3Mesh::BuildAdjacency, mesh.cpp:36-119) on a
height-field grid equals the grid's own topology: the wing of edge
(v[i], v[i+1]) of a triangle is the third vertex of the other triangle on
that edge, B3_MAX_U32 on the border."""
import numpy as np

from bounce_b200 import scene as S


def test_grid_adjacency(oracle_mod):
    V, T = S.grid_mesh(9, 7, 1.0, 11)
    arrays = dict(desc=np.array([0, len(V), 0, len(T)], np.uint32),
                  verts=np.ascontiguousarray(V.reshape(-1), np.float32),
                  tris=np.ascontiguousarray(T.reshape(-1), np.uint32))
    sc = S.Scene().finalize()
    w = oracle_mod.RefHulls(sc.hull_arrays, mesh_arrays=arrays).mesh_wings(0, len(T))
    owner = {}
    for t, tri in enumerate(T):
        for e in range(3):
            owner.setdefault(frozenset((tri[e], tri[(e + 1) % 3])), []).append(t)
    for t, tri in enumerate(T):
        for e in range(3):
            a, b = tri[e], tri[(e + 1) % 3]
            other = [u for u in owner[frozenset((a, b))] if u != t]
            if other:
                third = [x for x in T[other[0]] if x not in (a, b)][0]
                assert w[t, e] == third
            else:
                assert w[t, e] == 0xFFFFFFFF

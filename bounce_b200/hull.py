"""Convex hulls for scene input in pure Python: the same incremental algorithm,
operation order and output layout as the native builder
(bounce_b200/csrc/hull_builder.cpp, include/b3g_hull.h), so both give the same
arrays bit for bit (double-precision hull, single-precision planes).

Scene input only, never on the per-step path. It exists so that a process can
build the seeded scenes without mapping the CUDA library: the reference arm of
the benchmark builds its hulls here, and runs the reference's CPU pass on the
same hulls the device pass sees.

Layout (b3Hull, include/bounce/collision/geometry/hull.h:24-72): vertices
(3 floats each, in first-use order of the face loops), half-edges (origin,
twin, face, prev, next; each undirected edge owns 2k / 2k+1), faces (first
half-edge), planes (normal, offset; b3Plane(A, B, C) of the face's first three
vertices, plane.h:43-48) and a volume centroid.
"""
import math

import numpy as np

F = np.float32
MAX_POINTS = 256


def _tri(p, a, b, c):
    """Triangle a, b, c: unit normal (double) and plane offset."""
    ax, ay, az = p[a]
    bx, by, bz = p[b]
    cx, cy, cz = p[c]
    ux, uy, uz = bx - ax, by - ay, bz - az
    vx, vy, vz = cx - ax, cy - ay, cz - az
    nx = uy * vz - uz * vy
    ny = uz * vx - ux * vz
    nz = ux * vy - uy * vx
    l = math.sqrt(nx * nx + ny * ny + nz * nz)
    if l > 0:
        nx /= l
        ny /= l
        nz /= l
    return [(a, b, c), (nx, ny, nz), nx * ax + ny * ay + nz * az, True]


def _emit(pts, loops):
    """Face loops (vertex indices, counter-clockwise from outside) -> arrays."""
    remap = [-1] * len(pts)
    nv = 0
    for L in loops:
        for v in L:
            if remap[v] < 0:
                remap[v] = nv
                nv += 1
    fv = np.zeros((nv, 3), F)
    for i, q in enumerate(pts):
        if remap[i] >= 0:
            fv[remap[i]] = q
    he = []  # [origin, twin, face, prev, next]
    index = {}
    face_first = []
    for f, L in enumerate(loops):
        m = len(L)
        ids = []
        for i in range(m):
            a, b = remap[L[i]], remap[L[(i + 1) % m]]
            idx = index.get((a, b))
            if idx is None:
                base = len(he)
                he.append([a, base + 1, 0, 0, 0])
                he.append([b, base, 0, 0, 0])
                index[(a, b)] = base
                index[(b, a)] = base + 1
                idx = base
            ids.append(idx)
        for i in range(m):
            e = he[ids[i]]
            e[2] = f
            e[4] = ids[(i + 1) % m]
            e[3] = ids[(i + m - 1) % m]
        face_first.append(ids[0])

    # Planes in single precision, elementwise in the native builder's order.
    first3 = np.array([[remap[L[0]], remap[L[1]], remap[L[2]]] for L in loops], np.int64)
    A, B, C = fv[first3[:, 0]], fv[first3[:, 1]], fv[first3[:, 2]]
    e1 = B - A
    e2 = C - A
    nx = e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1]
    ny = e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2]
    nz = e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]
    l = np.sqrt((nx * nx + ny * ny) + nz * nz)
    big = l > F(1.1920928955078125e-7)
    s = np.where(big, F(1) / np.where(big, l, F(1)), F(1)).astype(F)
    nx = np.where(big, s * nx, nx)
    ny = np.where(big, s * ny, ny)
    nz = np.where(big, s * nz, nz)
    planes = np.stack([nx, ny, nz, (nx * A[:, 0] + ny * A[:, 1]) + nz * A[:, 2]], axis=1).astype(F)

    # Volume centroid (fan of tetrahedra from vertex 0), in double.
    fd = fv.astype(np.float64).tolist()
    ox, oy, oz = fd[0]
    vol = cx = cy = cz = 0.0
    for L in loops:
        a = fd[remap[L[0]]]
        for i in range(1, len(L) - 1):
            b = fd[remap[L[i]]]
            c = fd[remap[L[i + 1]]]
            ax, ay, az = a[0] - ox, a[1] - oy, a[2] - oz
            bx, by, bz = b[0] - ox, b[1] - oy, b[2] - oz
            qx, qy, qz = c[0] - ox, c[1] - oy, c[2] - oz
            kx = by * qz - bz * qy
            ky = bz * qx - bx * qz
            kz = bx * qy - by * qx
            v6 = ax * kx + ay * ky + az * kz
            vol += v6
            cx += v6 * (ox + a[0] + b[0] + c[0]) / 4
            cy += v6 * (oy + a[1] + b[1] + c[1]) / 4
            cz += v6 * (oz + a[2] + b[2] + c[2]) / 4
    if vol > 0:
        centroid = np.array([cx / vol, cy / vol, cz / vol], np.float64).astype(F)
    else:
        centroid = np.zeros(3, F)
    return (fv.reshape(-1), np.asarray(he, np.uint32).reshape(-1), np.asarray(face_first, np.uint32),
            planes.reshape(-1), centroid, (nv, len(he), len(loops)))


def _len3(x, y, z):
    return math.sqrt(x * x + y * y + z * z)


def hull_from_points(points):
    """Hull of n points (n x 3 float32): (verts, edges, faces, planes,
    centroid, (nv, ne, nf)). Raises ValueError for fewer than 4 points, more
    than MAX_POINTS, or a degenerate (collinear / coplanar) set."""
    pts = np.ascontiguousarray(points, F).reshape(-1, 3)
    n = len(pts)
    if n < 4 or n > MAX_POINTS:
        raise ValueError("degenerate hull point set")
    p = [tuple(float(c) for c in q) for q in pts.tolist()]
    ext = 0.0
    for q in p:
        ext = max(ext, max(abs(q[0]), max(abs(q[1]), abs(q[2]))))
    eps = 1e-9 * (ext if ext > 0 else 1) * 8

    # Initial tetrahedron: farthest point from p0, farthest from that line,
    # farthest from that plane (first maximum wins, as in the native builder).
    i0, i1, i2, i3 = 0, -1, -1, -1
    x0, y0, z0 = p[i0]
    best = 0.0
    for i in range(1, n):
        d = _len3(p[i][0] - x0, p[i][1] - y0, p[i][2] - z0)
        if d > best:
            best, i1 = d, i
    if i1 < 0 or best <= eps:
        raise ValueError("degenerate hull point set")
    ux, uy, uz = p[i1][0] - x0, p[i1][1] - y0, p[i1][2] - z0
    best = 0.0
    for i in range(n):
        vx, vy, vz = p[i][0] - x0, p[i][1] - y0, p[i][2] - z0
        d = _len3(uy * vz - uz * vy, uz * vx - ux * vz, ux * vy - uy * vx)
        if d > best:
            best, i2 = d, i
    if i2 < 0 or best <= eps:
        raise ValueError("degenerate hull point set")
    vx, vy, vz = p[i2][0] - x0, p[i2][1] - y0, p[i2][2] - z0
    nx, ny, nz = uy * vz - uz * vy, uz * vx - ux * vz, ux * vy - uy * vx
    best = 0.0
    for i in range(n):
        d = abs(nx * (p[i][0] - x0) + ny * (p[i][1] - y0) + nz * (p[i][2] - z0))
        if d > best:
            best, i3 = d, i
    if i3 < 0 or best <= eps * _len3(nx, ny, nz):
        raise ValueError("degenerate hull point set")

    if nx * (p[i3][0] - x0) + ny * (p[i3][1] - y0) + nz * (p[i3][2] - z0) > 0:
        tris = [_tri(p, i0, i2, i1), _tri(p, i0, i1, i3), _tri(p, i1, i2, i3), _tri(p, i2, i0, i3)]
    else:
        tris = [_tri(p, i0, i1, i2), _tri(p, i0, i3, i1), _tri(p, i1, i3, i2), _tri(p, i2, i3, i0)]

    for pi in range(n):
        if pi in (i0, i1, i2, i3):
            continue
        qx, qy, qz = p[pi]
        visible = []
        for t, tr in enumerate(tris):
            if tr[3]:
                tn = tr[1]
                if (tn[0] * qx + tn[1] * qy + tn[2] * qz) - tr[2] > eps:
                    visible.append(t)
        if not visible:
            continue
        # Horizon: directed edges of visible faces whose reverse edge belongs
        # to no visible face, in face order then edge order.
        vis_edges = set()
        for t in visible:
            v = tris[t][0]
            vis_edges.update(((v[0], v[1]), (v[1], v[2]), (v[2], v[0])))
        horizon = []
        for t in visible:
            v = tris[t][0]
            for k in range(3):
                a, b = v[k], v[(k + 1) % 3]
                if (b, a) not in vis_edges:
                    horizon.append((a, b))
        for t in visible:
            tris[t][3] = False
        for a, b in horizon:
            tris.append(_tri(p, a, b, pi))
    loops = [list(tr[0]) for tr in tris if tr[3]]
    return _emit(p, loops)


def hull_box(ex, ey, ez):
    """Box hull with half extents (ex, ey, ez): 8 vertices, 24 half-edges, 6
    quad faces, centroid at the origin (b3g_hull_box)."""
    ex, ey, ez = float(F(ex)), float(F(ey)), float(F(ez))
    p = [(-ex, -ey, -ez), (ex, -ey, -ez), (ex, ey, -ez), (-ex, ey, -ez),
         (-ex, -ey, ez), (ex, -ey, ez), (ex, ey, ez), (-ex, ey, ez)]
    loops = [[0, 4, 7, 3], [1, 2, 6, 5], [0, 1, 5, 4], [3, 7, 6, 2], [0, 3, 2, 1], [4, 5, 6, 7]]
    v, e, f, pl, _, counts = _emit(p, loops)
    return v, e, f, pl, np.zeros(3, F), counts

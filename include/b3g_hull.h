/*
 * b3g_hull.h - host-side convex hull construction in the b3Hull half-edge
 * layout consumed by b3g_set_hulls (include/b3g.h).
 *
 * Scene input only, not part of the per-step path. The reference builds
 * hulls with the vendored quickhull (src/quickhull/quickhull.c, converted by
 * examples/testbed/framework/test.cpp:38-96) or the hand-written box
 * (include/bounce/collision/geometry/box_hull.h); this builder produces the
 * same kind of structure (half-edge pairs at 2k / 2k+1, triangle faces for
 * points in general position, one plane per face, a volume centroid) from
 * its own incremental hull algorithm.
 */
#ifndef B3G_HULL_H
#define B3G_HULL_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* Sizes needed for a hull of n input points: at most n vertices,
 * 6n - 12 half-edges and 2n - 4 faces (n >= 4). */
#define B3G_HULL_MAX_POINTS 256

/* Builds the convex hull of n points (3 floats each). Outputs go to
 * caller-provided arrays sized for the bounds above; counts are written to
 * counts[3] = {vertexCount, edgeCount, faceCount}. Returns 0 or a negative
 * status (-1: fewer than 4 points or all points coplanar). */
int b3g_hull_from_points(const float* points, uint32_t n, float* verts, uint32_t* edges,
	uint32_t* faces, float* planes, float* centroid, uint32_t* counts);

/* Box hull with half extents (ex, ey, ez), centred at the origin: 8 vertices,
 * 24 half-edges, 6 quad faces (the shape of b3BoxHull::SetExtents). */
int b3g_hull_box(float ex, float ey, float ez, float* verts, uint32_t* edges,
	uint32_t* faces, float* planes, float* centroid, uint32_t* counts);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* B3G_HULL_H */

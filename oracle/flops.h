// Floating-point operations of the reference's narrowphase, per loop trip:
// the constants the flop count of the FP64 oracle run (flop_count.cpp) uses.
// TEST INFRASTRUCTURE: the count is the algorithmic work of the reference's
// collision routines, the numerator of the device narrowphase's roofline.
//
// A flop is one add, subtract, multiply, divide or square root (compares and
// sign flips are not counted). The constants come from the expressions of the
// cited lines; the building blocks:
//   DOT    b3Dot                           3 mul + 2 add            =  5
//   CROSS  b3Cross                         6 mul + 3 sub            =  9
//   LEN    b3Length                        DOT + sqrt               =  6
//   ROT    b3Mul(b3Quat, b3Vec3)           t = 2 (v x p): 12; v + s t: 6;
//          (quat.h)                        + v x t: 9; + 3 add      = 30
//   XFP    b3Mul(b3Transform, b3Vec3)      ROT + 3 add              = 33
//   XFXF   b3MulT(b3Transform, b3Transform) quat product 28,
//                                          rotation of the offset 33 = 61
//   PLANE  b3Mul(b3Transform, b3Plane)     ROT + DOT + 1 add        = 36
//   DIST   b3Distance(point, plane)        DOT + 1 sub              =  6
// One term is an estimate, not an expression count: the simplex solve of a
// GJK iteration (Solve2 / Solve3 / Solve4, gjk.cpp:276-650), taken as
// FL_GJK_SOLVE per iteration whatever the simplex size.
#ifndef ORACLE_FLOPS_H
#define ORACLE_FLOPS_H

// b3QueryFaceSeparation, hull-hull (sat.cpp:33-58): XFXF once; per plane of
// hull 1 PLANE + DIST; per (plane, vertex of hull 2) one DOT
// (b3Hull::GetSupportVertex, hull.h:105-119).
#define FL_FACE_SETUP 61
#define FL_FACE_PLANE 42
#define FL_FACE_TRIP 5

// b3QueryFaceSeparation, hull-capsule (sat_hull_edge.cpp:29-55): XFXF + 2 XFP
// once; per plane two DIST (the segment's support).
#define FL_FACE_SEG_SETUP 127
#define FL_FACE_SEG_PLANE 12

// b3QueryEdgeSeparation, hull-hull (sat.cpp:111-174): XFXF + XFP (centroid)
// once; per edge of hull 1: P1, Q1 (XFP each), E1 (3), U1, V1 (ROT each);
// per edge pair: E2 (3) + b3IsMinkowskiFace (4 DOT + 3 mul); per pair that
// passes the Gauss-map test, b3Project (sat.cpp:73-109): 3 LEN, CROSS,
// tolerance (2), scale (1 div + 3 mul), 2 sub-vectors (6), 2 DOT.
#define FL_EDGE_SETUP 94
#define FL_EDGE_OUTER 129
#define FL_EDGE_PAIR 26
#define FL_EDGE_QUALIFIED 49

// b3QueryEdgeSeparation, hull-capsule (sat_hull_edge.cpp:92-146): XFXF + 2 XFP
// + 3 once; per hull edge E1 (3) + 2 DOT + 1 mul; qualified b3ProjectEdge 49.
#define FL_EDGE_SEG_SETUP 130
#define FL_EDGE_SEG_PAIR 14
#define FL_EDGE_SEG_QUALIFIED 49

// Clipping to the reference face's side planes (clip.cpp:100-150, :202-281):
// per side plane b3Hull::GetEdgeSidePlane (edge 3, CROSS, normalise 9,
// offset DOT; hull.h:137-152) + radius (1) + PLANE; per input vertex DIST; per
// edge that crosses the plane the intersection (fraction 2, lerp 9).
#define FL_CLIP_PLANE 63
#define FL_CLIP_VERTEX 6
#define FL_CLIP_CROSSING 11

// b3GJK (gjk.cpp:654-812): per call the cache read and the output (closest
// points, distance, radii); per iteration the closest point and its DOT, the
// search direction, two direction rotations (ROT), two support points (XFP),
// their difference, and the simplex solve (estimate); per proxy vertex of
// each support search one DOT (b3GJKProxy::GetSupportIndex, gjk_proxy.h:72-86).
#define FL_GJK_CALL 50
#define FL_GJK_ITER 159
#define FL_GJK_SOLVE 100
#define FL_GJK_SUPPORT_VERTEX 5

// Closed-form parts of the collide routines, per call (the loops above are
// counted separately):
//   spheres          collide_spheres.cpp:22-52        2 XFP, offset, DOT, normalise
//   capsule-sphere   collide_capsule_sphere.cpp:23-120 3 XFP, 2 DOT region tests, closest point, normal
//   capsules         collide_capsules.cpp:47-123      4 XFP, b3ClosestPointsOnSegments
//                                                     (collision.cpp:145-215), parallel test, side-plane clip
//   hull-sphere      collide_hull_sphere.cpp:26-97     2 XFP (sphere centre into the hull frame), point
//   hull-capsule     collide_hull_capsule.cpp:108-190  support face, parallel test, points
//   hulls            collide_hulls.cpp:355-534         cache state test and manifold points
#define FL_SPHERES 84
#define FL_CAPSULE_SPHERE 130
#define FL_CAPSULES 270
#define FL_HULL_SPHERE 90
#define FL_HULL_SPHERE_PLANE 6
#define FL_HULL_CAPSULE 60
#define FL_HULLS 60

// b3FeatureCache reads (sat.cpp:178-282): ReadFace re-projects the cached face
// (PLANE + DIST + one DOT per vertex of the other hull); ReadEdges re-projects
// the cached edge pair (2 edges transformed, b3Project); ReadState tests the
// cached separation sign (a face or edge projection, taken as ReadEdges).
#define FL_CACHE_FACE 42
#define FL_CACHE_EDGES 180

// b3ReducePolygon (cluster.cpp:59-200): per input polygon vertex the deepest /
// farthest / area scans (about 4 DOT and a CROSS).
#define FL_REDUCE_VERTEX 30

#endif

// Thread-per-pair narrowphase for the rounded convex pairs:
//   b3CollideSpheres          collide_spheres.cpp:22-52
//   b3CollideCapsuleAndSphere collide_capsule_sphere.cpp:23-120
//   b3CollideCapsules         collide_capsules.cpp:25-123
//   b3CollideHullAndSphere    collide_hull_sphere.cpp:26-97
//   b3CollideHullAndCapsule   collide_hull_capsule.cpp:29-190, sat_hull_edge.cpp:29-146
// and the sensor path b3TestOverlap (collision.cpp:104-113). Each routine
// evaluates the reference's operations in the reference's order.

#include "collide_common.cuh"

namespace {

struct ShapeP
{
	uint32_t type;
	float4 p0, p1, p2;
	uint32_t hull;
};

__device__ __forceinline__ ShapeP load_shape(const DevScene& S, uint32_t fix)
{
	ShapeP s;
	s.type = S.fixType[fix];
	s.p0 = S.fixParams[3 * fix + 0];
	s.p1 = S.fixParams[3 * fix + 1];
	s.p2 = S.fixParams[3 * fix + 2];
	s.hull = S.fixHull[fix];
	return s;
}

__device__ __forceinline__ V3 sph_center(const ShapeP& s) { return V3{s.p0.x, s.p0.y, s.p0.z}; }
__device__ __forceinline__ float sph_radius(const ShapeP& s) { return s.p0.w; }
__device__ __forceinline__ V3 cap_v1(const ShapeP& s) { return V3{s.p0.x, s.p0.y, s.p0.z}; }
__device__ __forceinline__ V3 cap_v2(const ShapeP& s) { return V3{s.p0.w, s.p1.x, s.p1.y}; }
__device__ __forceinline__ float cap_radius(const ShapeP& s) { return s.p1.z; }
__device__ __forceinline__ float hull_radius(const ShapeP& s) { return s.p0.x; }

__device__ void collide_spheres(DevManifold& m, const XF& xf1, const ShapeP& s1, const XF& xf2, const ShapeP& s2)
{
	V3 c1 = xmul(xf1, sph_center(s1));
	float r1 = sph_radius(s1);
	V3 c2 = xmul(xf2, sph_center(s2));
	float r2 = sph_radius(s2);
	V3 d = c2 - c1;
	float dd = dot(d, d);
	float totalRadius = r1 + r2;
	if (dd > totalRadius * totalRadius)
		return;
	float distance = len(d);
	V3 normal = V3{0.0f, 1.0f, 0.0f};
	if (distance > B3G_EPSILON)
		normal = d / distance;
	m.pointCount = 1;
	set_point(m.points[0], rotc(xf1.q, normal), sph_center(s1), sph_center(s2));
	set_id0(m.points[0]);
}

__device__ void collide_capsule_sphere(DevManifold& m, const XF& xf1, const ShapeP& c1, const XF& xf2,
	const ShapeP& s2)
{
	V3 Q = xmult(xf1, xmul(xf2, sph_center(s2)));
	V3 A = cap_v1(c1), B = cap_v2(c1);
	V3 AB = B - A;
	float u = dot(B - Q, AB);
	float v = dot(Q - A, AB);
	float radius = cap_radius(c1) + sph_radius(s2);
	if (v <= 0.0f || u <= 0.0f)
	{
		V3 P = v <= 0.0f ? A : B;
		V3 d = Q - P;
		float dd = dot(d, d);
		if (dd > radius * radius)
			return;
		V3 n = V3{0.0f, 1.0f, 0.0f};
		float l = len(d);
		if (l > B3G_EPSILON)
			n = d / l;
		m.pointCount = 1;
		set_point(m.points[0], n, P, sph_center(s2));
		set_id0(m.points[0]);
		return;
	}
	float s = dot(AB, AB);
	V3 P = (u * A + v * B) / s;
	V3 d = Q - P;
	float dd = dot(d, d);
	if (dd > radius * radius)
		return;
	V3 AQ = Q - A;
	V3 AB_x_AQ = cross(AB, AQ);
	V3 n = cross(AB_x_AQ, AB);
	if (dot(n, AQ) < 0.0f)
		n = -n;
	normalize_inplace(n);
	m.pointCount = 1;
	set_point(m.points[0], n, P, sph_center(s2));
	set_id0(m.points[0]);
}

// b3AreParalell (collide_capsules.cpp:25-45).
__device__ __forceinline__ bool are_parallel(V3 a1, V3 a2, V3 b1, V3 b2)
{
	V3 E1 = a2 - a1;
	float L1 = len(E1);
	if (L1 < B3G_LINEAR_SLOP)
		return false;
	V3 E2 = b2 - b1;
	float L2 = len(E2);
	if (L2 < B3G_LINEAR_SLOP)
		return false;
	const float kTol = 0.005f;
	V3 N = cross(E1, E2);
	return len(N) < (kTol * L1) * L2;
}

__device__ void collide_capsules(DevManifold& m, const XF& xf1, const ShapeP& k1, const XF& xf2, const ShapeP& k2)
{
	V3 s1a = xmul(xf1, cap_v1(k1)), s1b = xmul(xf1, cap_v2(k1));
	V3 s2a = xmul(xf2, cap_v1(k2)), s2b = xmul(xf2, cap_v2(k2));
	V3 point1, point2;
	closest_on_segments(point1, point2, s1a, s1b, s2a, s2b);
	float distance = len(point1 - point2);
	float r1 = cap_radius(k1), r2 = cap_radius(k2);
	float totalRadius = r1 + r2;
	if (distance > totalRadius)
		return;
	if (distance > 0.0f && are_parallel(s1a, s1b, s2a, s2b))
	{
		ClipV in1[2];
		build_segment(in1, s1a, s1b);
		ClipV clip1[2];
		uint32_t clipCount = clip_segment_to_segment_side_planes(clip1, in1, s2a, s2b);
		if (clipCount == 2)
		{
			V3 cp1 = closest_on_segment(clip1[0].pos, s2a, s2b);
			V3 cp2 = closest_on_segment(clip1[1].pos, s2a, s2b);
			float d1 = len(clip1[0].pos - cp1);
			float d2 = len(clip1[1].pos - cp2);
			if (d1 > B3G_EPSILON && d1 <= totalRadius && d2 > B3G_EPSILON && d2 <= totalRadius)
			{
				V3 n1 = (cp1 - clip1[0].pos) / d1;
				V3 n2 = (cp2 - clip1[1].pos) / d2;
				m.pointCount = 2;
				set_point(m.points[0], rotc(xf1.q, n1), xmult(xf1, clip1[0].pos), xmult(xf2, cp1));
				set_id(m.points[0], clip1[0].pair);
				set_point(m.points[1], rotc(xf1.q, n2), xmult(xf1, clip1[1].pos), xmult(xf2, cp2));
				set_id(m.points[1], clip1[1].pair);
				return;
			}
		}
	}
	if (distance > 0.0f)
	{
		V3 normal = (point2 - point1) / distance;
		m.pointCount = 1;
		set_point(m.points[0], rotc(xf1.q, normal), xmult(xf1, point1), xmult(xf2, point2));
		set_id0(m.points[0]);
	}
}

__device__ __forceinline__ GProxy hull_proxy(const HullRef& h, float r)
{
	GProxy p;
	p.gv = h.v;
	p.count = h.vCnt;
	p.radius = r;
	return p;
}

// b3CollideHullAndSphere (collide_hull_sphere.cpp:26-97), first part: the
// scan of the hull's faces for the sphere centre. False when that settles
// the manifold (empty: a face farther than the radii; one point: the centre
// inside the hull); true when the routine goes on to its GJK
// (hull_sphere_gjk).
__device__ __forceinline__ bool hull_sphere_faces(DevManifold& m, const DevScene& S, const XF& xf1,
	const ShapeP& hs, const XF& xf2, const ShapeP& s2)
{
	float radius = hull_radius(hs) + sph_radius(s2);
	HullRef h1 = hull_ref(S, hs.hull);
	V3 cLocal = xmult(xf1, xmul(xf2, sph_center(s2)));
	uint32_t faceIndex = 0;
	float separation = -B3G_MAX_SCALAR;
	for (uint32_t i = 0; i < h1.fCnt; ++i)
	{
		PL plane = hp(h1, i);
		float s = pdist(cLocal, plane);
		if (s > radius)
			return false;
		if (s > separation)
		{
			faceIndex = i;
			separation = s;
		}
	}
	if (separation < 0.0f)
	{
		PL lp = hp(h1, faceIndex);
		V3 c1 = pclosest(cLocal, lp);
		m.pointCount = 1;
		set_point(m.points[0], lp.n, c1, sph_center(s2));
		set_id0(m.points[0]);
		return false;
	}
	return true;
}

// The rest of b3CollideHullAndSphere: GJK between the hull and the centre.
__device__ __forceinline__ void hull_sphere_gjk(DevManifold& m, const DevScene& S, const XF& xf1, const ShapeP& hs,
	const XF& xf2, const ShapeP& s2)
{
	float radius = hull_radius(hs) + sph_radius(s2);
	HullRef h1 = hull_ref(S, hs.hull);
	GProxy p1 = hull_proxy(h1, hull_radius(hs));
	GProxy p2;
	p2.gv = nullptr;
	p2.lv[0] = sph_center(s2);
	p2.count = 1;
	p2.radius = sph_radius(s2);
	GJKOut q = gjk(xf1, p1, xf2, p2, false);
	if (q.distance > radius)
		return;
	if (q.distance > 0.0f)
	{
		V3 normal = (q.point2 - q.point1) / q.distance;
		m.pointCount = 1;
		set_point(m.points[0], rotc(xf1.q, normal), xmult(xf1, q.point1), sph_center(s2));
		set_id0(m.points[0]);
	}
}

// First maximum of (v, idx) over the G lanes of a lane group (lanes
// [k*G, k*G + G) of the warp, gmask): the largest value, and among equal
// values the lowest index, which is what the reference's serial scans keep
// with their strict "greater" test. Every lane of the group ends with it.
template <int G>
__device__ __forceinline__ void group_argmax(float& v, uint32_t& idx, uint32_t gmask)
{
#pragma unroll
	for (int o = G / 2; o > 0; o >>= 1)
	{
		float ov = __shfl_xor_sync(gmask, v, o, G);
		uint32_t oi = __shfl_xor_sync(gmask, idx, o, G);
		if (ov > v || (ov == v && oi < idx))
		{
			v = ov;
			idx = oi;
		}
	}
}

// b3Hull::GetSupportFace (hull.h:121-135) with the faces spread over the
// group's lanes (lane gl takes faces gl, gl + G, ...).
template <int G>
__device__ __forceinline__ uint32_t group_support_face(const HullRef& h, V3 d, uint32_t gl, uint32_t gmask)
{
	if (G == 1)
		return hull_support_face(h, d);
	float best = -INFINITY;
	uint32_t bi = 0xFFFFFFFFu;
	for (uint32_t i = gl; i < h.fCnt; i += G)
	{
		float proj = dot(d, hp(h, i).n);
		if (bi == 0xFFFFFFFFu || proj > best)
		{
			best = proj;
			bi = i;
		}
	}
	group_argmax<G>(best, bi, gmask);
	return bi;
}

// b3QueryFaceSeparation(hull, capsule) (sat_hull_edge.cpp:29-59), faces
// spread over the group's lanes. A lane that finds no separation above the
// start value keeps (-max, 0), so the group's answer is (-max, 0) exactly
// when the serial scan's is.
template <int G>
__device__ void query_face_hull_capsule(const HullRef& h1, V3 lv1, V3 lv2, uint32_t& index, float& sep,
	uint32_t gl, uint32_t gmask)
{
	uint32_t maxIndex = 0;
	float maxSep = -B3G_MAX_SCALAR;
	for (uint32_t i = gl; i < h1.fCnt; i += G)
	{
		PL plane = hp(h1, i);
		V3 d = -plane.n;
		V3 support = dot(d, lv1) > dot(d, lv2) ? lv1 : lv2; // b3Capsule::GetSupportVertex
		float s = pdist(support, plane);
		if (s > maxSep)
		{
			maxIndex = i;
			maxSep = s;
		}
	}
	group_argmax<G>(maxSep, maxIndex, gmask);
	index = maxIndex;
	sep = maxSep;
}

// b3ProjectEdge (sat_hull_edge.cpp:68-100).
__device__ __forceinline__ float project_edge_capsule(V3 P1, V3 E1, V3 C1, V3 P2, V3 E2)
{
	float L1 = len(E1);
	if (L1 < B3G_LINEAR_SLOP)
		return -B3G_MAX_SCALAR;
	float L2 = len(E2);
	if (L2 < B3G_LINEAR_SLOP)
		return -B3G_MAX_SCALAR;
	const float kTol = 0.005f;
	V3 E1_x_E2 = cross(E1, E2);
	float L = len(E1_x_E2);
	if (L < (kTol * L1) * L2)
		return -B3G_MAX_SCALAR;
	V3 N = (1.0f / L) * E1_x_E2;
	if (dot(N, P1 - C1) < 0.0f)
		N = -N;
	return dot(N, P2 - P1);
}

// b3QueryEdgeSeparation(hull, capsule) (sat_hull_edge.cpp:102-146), the
// hull's edges (half-edge pairs i, i + 1) spread over the group's lanes.
template <int G>
__device__ void query_edge_hull_capsule(const HullRef& h1, V3 P2, V3 Q2, uint32_t& index, float& sep,
	uint32_t gl, uint32_t gmask)
{
	uint32_t maxIndex = 0;
	float maxSep = -B3G_MAX_SCALAR;
	V3 C1 = h1.centroid;
	V3 E2 = Q2 - P2;
	for (uint32_t i = 2 * gl; i < h1.eCnt; i += 2 * G)
	{
		uint4 e1 = h1.e[i], t1 = h1.e[i + 1];
		V3 P1 = hv(h1, e1.x);
		V3 Q1 = hv(h1, t1.x);
		V3 E1 = Q1 - P1;
		V3 U1 = hp(h1, e1.y).n;
		V3 V1 = hp(h1, t1.y).n;
		// b3IsMinkowskiFace(E2, U1, V1)
		if (dot(E2, U1) * dot(E2, V1) < 0.0f)
		{
			float s = project_edge_capsule(P1, E1, C1, P2, E2);
			if (s > maxSep)
			{
				maxSep = s;
				maxIndex = i;
			}
		}
	}
	group_argmax<G>(maxSep, maxIndex, gmask);
	index = maxIndex;
	sep = maxSep;
}

__device__ void hull_capsule_edge_contact(DevManifold& m, const XF& xf1, const HullRef& h1, uint32_t index1,
	const XF& xf2, V3 v1, V3 v2)
{
	uint4 e1 = h1.e[index1], t1 = h1.e[index1 + 1];
	V3 C1 = xmul(xf1, h1.centroid);
	V3 P1 = xmul(xf1, hv(h1, e1.x));
	V3 Q1 = xmul(xf1, hv(h1, t1.x));
	V3 E1 = Q1 - P1;
	V3 P2 = xmul(xf2, v1);
	V3 Q2 = xmul(xf2, v2);
	V3 E2 = Q2 - P2;
	V3 N = cross(E1, E2);
	normalize_inplace(N);
	if (dot(N, P1 - C1) < 0.0f)
		N = -N;
	V3 point1, point2;
	closest_on_segments(point1, point2, P1, Q1, P2, Q2);
	m.pointCount = 1;
	set_point(m.points[0], rotc(xf1.q, N), xmult(xf1, point1), xmult(xf2, point2));
	set_id(m.points[0], mkpair(index1, index1 + 1, 0, 1));
}

__device__ void hull_capsule_face_contact(DevManifold& m, const XF& xf1, const HullRef& h1, uint32_t index1,
	float r1, const XF& xf2, V3 v1, V3 v2, float r2)
{
	ClipV seg[2];
	build_segment(seg, xmul(xf2, v1), xmul(xf2, v2));
	ClipV clip2[2];
	uint32_t clipCount = clip_segment_to_face_side_planes(clip2, seg, xf1, r1, index1, h1);
	PL localPlane1 = hp(h1, index1);
	PL plane1 = pmul(xf1, localPlane1);
	float totalRadius = r1 + r2;
	uint32_t pointCount = 0;
	for (uint32_t i = 0; i < clipCount; ++i)
	{
		V3 c2 = clip2[i].pos;
		float s = pdist(c2, plane1);
		if (s <= totalRadius)
		{
			V3 c1 = pclosest(c2, plane1);
			DevPoint& mp = m.points[pointCount];
			set_point(mp, localPlane1.n, xmult(xf1, c1), xmult(xf2, c2));
			set_id(mp, clip2[i].pair);
			++pointCount;
		}
	}
	m.pointCount = pointCount;
}

// b3CollideHullAndCapsule (collide_hull_capsule.cpp:29-190), first part:
// the GJK distance between the hull and the capsule's segment. False when it
// is above the radii (an empty manifold); else the rest of the routine
// (hull_capsule_after_gjk) builds the manifold from q.
__device__ __forceinline__ bool hull_capsule_gjk(const DevScene& S, const XF& xf1, const ShapeP& hs, const XF& xf2,
	const ShapeP& k2, GJKOut& q)
{
	float r1 = hull_radius(hs), r2 = cap_radius(k2);
	float totalRadius = r1 + r2;
	HullRef h1 = hull_ref(S, hs.hull);
	GProxy p1 = hull_proxy(h1, r1);
	GProxy p2;
	p2.gv = nullptr;
	p2.lv[0] = cap_v1(k2);
	p2.lv[1] = cap_v2(k2);
	p2.count = 2;
	p2.radius = r2;
	q = gjk(xf1, p1, xf2, p2, false);
	return !(q.distance > totalRadius);
}

// The rest of b3CollideHullAndCapsule after its GJK, run by a group of G
// lanes (gl the lane in the group): the support face or the SAT queries
// spread over the lanes, the contact points built by lane 0, which alone
// writes m.
template <int G>
__device__ void hull_capsule_after_gjk(DevManifold& m, const DevScene& S, const XF& xf1, const ShapeP& hs,
	const XF& xf2, const ShapeP& k2, const GJKOut& q, uint32_t gl, uint32_t gmask)
{
	float r1 = hull_radius(hs), r2 = cap_radius(k2);
	float totalRadius = r1 + r2;
	HullRef h1 = hull_ref(S, hs.hull);
	V3 v1 = cap_v1(k2), v2 = cap_v2(k2);
	if (q.distance > 0.0f)
	{
		V3 c1 = q.point1, c2 = q.point2;
		float d = q.distance;
		V3 N1 = (c2 - c1) / d;
		V3 localN1 = rotc(xf1.q, N1);
		uint32_t index1 = group_support_face<G>(h1, localN1, gl, gmask);
		if (gl != 0)
			return;
		V3 localFaceN1 = hp(h1, index1).n;
		const float kTol = 0.005f;
		V3 N = cross(localN1, localFaceN1);
		float L = dot(N, N);
		if (L < kTol * kTol)
		{
			hull_capsule_face_contact(m, xf1, h1, index1, r1, xf2, v1, v2, r2);
			if (m.pointCount == 2)
				return;
		}
		m.pointCount = 1;
		set_point(m.points[0], localN1, xmult(xf1, c1), xmult(xf2, c2));
		set_id0(m.points[0]);
		return;
	}
	// Deep overlap: SAT on the hull against the capsule segment.
	XF xf = xmult(xf1, xf2);
	V3 lv1 = xmul(xf, v1), lv2 = xmul(xf, v2);
	uint32_t faceIndex;
	float faceSep;
	query_face_hull_capsule<G>(h1, lv1, lv2, faceIndex, faceSep, gl, gmask);
	if (faceSep > totalRadius)
		return;
	uint32_t edgeIndex;
	float edgeSep;
	query_edge_hull_capsule<G>(h1, lv1, lv2, edgeIndex, edgeSep, gl, gmask);
	if (edgeSep > totalRadius || gl != 0)
		return;
	const float kRelEdgeTol = 0.90f;
	const float kAbsTol = 0.5f * B3G_LINEAR_SLOP;
	if (edgeSep > kRelEdgeTol * faceSep + kAbsTol)
		hull_capsule_edge_contact(m, xf1, h1, edgeIndex, xf2, v1, v2);
	else
		hull_capsule_face_contact(m, xf1, h1, faceIndex, r1, xf2, v1, v2, r2);
}

// ---------------------------------------------------------------------------
// Triangles (with optional edge wings for smooth edges).

struct TriWings
{
	V3 e[3];
	bool has[3];
};

__device__ __forceinline__ TriWings load_wings(const DevScene& S, uint32_t fix)
{
	TriWings w;
	for (int k = 0; k < 3; ++k)
	{
		float4 x = S.fixWing[3 * (size_t)fix + k];
		w.e[k] = V3{x.x, x.y, x.z};
		w.has[k] = x.w != 0.0f;
	}
	return w;
}

__device__ __forceinline__ V3 tri_v1(const ShapeP& s) { return V3{s.p0.x, s.p0.y, s.p0.z}; }
__device__ __forceinline__ V3 tri_v2(const ShapeP& s) { return V3{s.p0.w, s.p1.x, s.p1.y}; }
__device__ __forceinline__ V3 tri_v3(const ShapeP& s) { return V3{s.p1.z, s.p1.w, s.p2.x}; }
__device__ __forceinline__ float tri_radius(const ShapeP& s) { return s.p2.y; }

// One point from P on the triangle to the sphere centre (every region of
// b3CollideTriangleAndSphere ends this way).
__device__ __forceinline__ bool tri_sphere_point(DevManifold& m, V3 P, V3 Q, float radius, V3 center2)
{
	V3 d = Q - P;
	float dd = dot(d, d);
	if (dd > radius * radius)
		return false;
	V3 n = V3{0.0f, 1.0f, 0.0f};
	float l = len(d);
	if (l > B3G_EPSILON)
		n = d / l;
	m.pointCount = 1;
	set_point(m.points[0], n, P, center2);
	set_id0(m.points[0]);
	return true;
}

// Is Q in the face region of the wing triangle (A1, B1, C1)?
__device__ __forceinline__ bool in_wing_face(V3 A1, V3 B1, V3 C1, V3 Q)
{
	float w[4];
	barycentric_triangle(w, A1, B1, C1, Q);
	return w[0] > 0.0f && w[1] > 0.0f && w[2] > 0.0f;
}

// b3CollideTriangleAndSphere (collide_triangle_sphere.cpp:24-296): Voronoi
// regions of the triangle, edge regions suppressed when the sphere lies in
// the face region of the triangle across a winged edge.
__device__ void collide_triangle_sphere(DevManifold& m, const XF& xf1, const ShapeP& t1, const TriWings& wg,
	const XF& xf2, const ShapeP& s2)
{
	V3 center2 = sph_center(s2);
	V3 Q = xmult(xf1, xmul(xf2, center2));
	V3 A = tri_v1(t1), B = tri_v2(t1), C = tri_v3(t1);
	float radius = tri_radius(t1) + sph_radius(s2);
	float wAB[3], wBC[3], wCA[3];
	barycentric_segment(wAB, A, B, Q);
	barycentric_segment(wBC, B, C, Q);
	barycentric_segment(wCA, C, A, Q);
	// vertex regions
	if (wAB[1] <= 0.0f && wCA[0] <= 0.0f)
	{
		tri_sphere_point(m, A, Q, radius, center2);
		return;
	}
	if (wAB[0] <= 0.0f && wBC[1] <= 0.0f)
	{
		tri_sphere_point(m, B, Q, radius, center2);
		return;
	}
	if (wBC[0] <= 0.0f && wCA[1] <= 0.0f)
	{
		tri_sphere_point(m, C, Q, radius, center2);
		return;
	}
	float wABC[4];
	barycentric_triangle(wABC, A, B, C, Q);
	// edge regions
	if (wAB[0] > 0.0f && wAB[1] > 0.0f && wABC[3] * wABC[2] <= 0.0f)
	{
		float den = 1.0f / wAB[2];
		V3 P = den * (wAB[0] * A + wAB[1] * B);
		V3 d = Q - P;
		if (dot(d, d) > radius * radius)
			return;
		if (wg.has[0] && in_wing_face(wg.e[0], B, A, Q))
			return;
		tri_sphere_point(m, P, Q, radius, center2);
		return;
	}
	if (wBC[0] > 0.0f && wBC[1] > 0.0f && wABC[3] * wABC[0] <= 0.0f)
	{
		float den = 1.0f / wBC[2];
		V3 P = den * (wBC[0] * B + wBC[1] * C);
		V3 d = Q - P;
		if (dot(d, d) > radius * radius)
			return;
		if (wg.has[1] && in_wing_face(wg.e[1], C, B, Q))
			return;
		tri_sphere_point(m, P, Q, radius, center2);
		return;
	}
	if (wCA[0] > 0.0f && wCA[1] > 0.0f && wABC[3] * wABC[1] <= 0.0f)
	{
		float den = 1.0f / wCA[2];
		V3 P = den * (wCA[0] * C + wCA[1] * A);
		V3 d = Q - P;
		if (dot(d, d) > radius * radius)
			return;
		if (wg.has[2] && in_wing_face(wg.e[2], A, C, Q))
			return;
		tri_sphere_point(m, P, Q, radius, center2);
		return;
	}
	// face region
	if (wABC[3] == 0.0f)
		return;
	float den = 1.0f / wABC[3];
	V3 P = den * ((wABC[0] * A + wABC[1] * B) + wABC[2] * C);
	tri_sphere_point(m, P, Q, radius, center2);
}

// b3UniqueCount (gjk_feature_pair.cpp): distinct values among the first n.
__device__ __forceinline__ uint32_t unique_count(const uint32_t* v, uint32_t n)
{
	uint32_t u = 0;
	for (uint32_t i = 0; i < n; ++i)
	{
		bool seen = false;
		for (uint32_t j = 0; j < i; ++j)
			seen = seen || v[j] == v[i];
		u += seen ? 0u : 1u;
	}
	return u;
}

// The shape-1 edge of b3GetFeaturePair (gjk_feature_pair.cpp:20-236) when its
// count1 is 2: false otherwise.
__device__ bool feature_edge1(const GJKSimplexOut& sx, uint32_t& v1, uint32_t& v2)
{
	uint32_t n = sx.count;
	if (n != 2 && n != 3)
		return false;
	uint32_t u1 = unique_count(sx.index1, n), u2 = unique_count(sx.index2, n);
	if (n == 2)
	{
		// EE, then VE (count1 1), then EV
		if ((u1 == 2 && u2 == 2) || (u1 != 1 && u2 == 1))
		{
			v1 = sx.index1[0];
			v2 = sx.index1[1];
			return true;
		}
		return false;
	}
	// EE and EF: the two distinct shape-1 indices
	if (u1 == 2 && (u2 == 2 || u2 == 3))
	{
		v1 = sx.index1[0];
		v2 = sx.index1[0] == sx.index1[1] ? sx.index1[2] : sx.index1[1];
		return true;
	}
	return false;
}

// b3CollideTriangleAndCapsule (collide_triangle_capsule.cpp:104-278); h1 is
// the triangle's b3TriangleHull.
__device__ void collide_triangle_capsule(DevManifold& m, const HullRef& h1, const XF& xf1, const ShapeP& t1,
	const TriWings& wg, const XF& xf2, const ShapeP& k2)
{
	float r1 = tri_radius(t1), r2 = cap_radius(k2);
	float totalRadius = r1 + r2;
	GProxy p1;
	p1.gv = nullptr;
	p1.lv[0] = tri_v1(t1);
	p1.lv[1] = tri_v2(t1);
	p1.lv[2] = tri_v3(t1);
	p1.count = 3;
	p1.radius = r1;
	GProxy p2;
	p2.gv = nullptr;
	p2.lv[0] = cap_v1(k2);
	p2.lv[1] = cap_v2(k2);
	p2.count = 2;
	p2.radius = r2;
	GJKSimplexOut sx;
	GJKOut q = gjk(xf1, p1, xf2, p2, false, &sx);
	if (q.distance > totalRadius)
		return;
	V3 v1 = cap_v1(k2), v2 = cap_v2(k2);
	if (q.distance > 0.0f)
	{
		V3 c1 = q.point1, c2 = q.point2;
		float d = q.distance;
		V3 N1 = (c2 - c1) / d;
		V3 localN1 = rotc(xf1.q, N1);
		uint32_t index1 = hull_support_face(h1, localN1);
		V3 localFaceN1 = hp(h1, index1).n;
		const float kTol = 0.005f;
		V3 N = cross(localN1, localFaceN1);
		float L = dot(N, N);
		if (L < kTol * kTol)
		{
			hull_capsule_face_contact(m, xf1, h1, index1, r1, xf2, v1, v2, r2);
			if (m.pointCount == 2)
				return;
		}
		uint32_t e1, e2;
		if ((wg.has[0] || wg.has[1] || wg.has[2]) && feature_edge1(sx, e1, e2))
		{
			V3 vtx[3] = {tri_v1(t1), tri_v2(t1), tri_v3(t1)};
			int edgeIndex = -1;
			for (uint32_t i = 0; i < 3 && edgeIndex < 0; ++i)
			{
				uint32_t j = i + 1 < 3 ? i + 1 : 0;
				if ((e1 == i && e2 == j) || (e2 == i && e1 == j))
					edgeIndex = (int)i;
			}
			if (edgeIndex >= 0 && wg.has[edgeIndex])
			{
				uint32_t ev1 = (uint32_t)edgeIndex;
				uint32_t ev2 = ev1 + 1 < 3 ? ev1 + 1 : 0;
				V3 Q = xmult(xf1, c2);
				V3 A = wg.e[edgeIndex];
				V3 B = vtx[ev2];
				V3 C = vtx[ev1];
				float w[4];
				barycentric_triangle(w, A, B, C, Q);
				// In the adjacent face's region: no edge point (the manifold
				// keeps what the face-contact attempt left in it).
				if (w[0] > 0.0f && w[1] > 0.0f && w[2] > 0.0f)
					return;
				V3 center = ((A + B) + C) / 3.0f;
				PL plane = hp(h1, 0);
				float distance = pdist(center, plane);
				const float kCoplanarTol = 0.005f;
				if (distance > -kCoplanarTol && distance < kCoplanarTol)
				{
					V3 n = plane.n;
					if (dot(n, localN1) < 0.0f)
						n = -n;
					V3 nc2 = c1 + d * rot(xf1.q, n);
					localN1 = n;
					c2 = nc2;
				}
			}
		}
		m.pointCount = 1;
		set_point(m.points[0], localN1, xmult(xf1, c1), xmult(xf2, c2));
		set_id0(m.points[0]);
		return;
	}
	XF xf = xmult(xf1, xf2);
	V3 lv1 = xmul(xf, v1), lv2 = xmul(xf, v2);
	uint32_t faceIndex;
	float faceSep;
	query_face_hull_capsule<1>(h1, lv1, lv2, faceIndex, faceSep, 0, 1u);
	if (faceSep > totalRadius)
		return;
	uint32_t edgeIndex;
	float edgeSep;
	query_edge_hull_capsule<1>(h1, lv1, lv2, edgeIndex, edgeSep, 0, 1u);
	if (edgeSep > totalRadius)
		return;
	const float kRelEdgeTol = 0.90f;
	const float kAbsTol = 0.5f * B3G_LINEAR_SLOP;
	if (edgeSep > kRelEdgeTol * faceSep + kAbsTol)
		hull_capsule_edge_contact(m, xf1, h1, edgeIndex, xf2, v1, v2);
	else
		hull_capsule_face_contact(m, xf1, h1, faceIndex, r1, xf2, v1, v2, r2);
}

__device__ GProxy shape_proxy(const DevScene& S, const ShapeP& s)
{
	GProxy p;
	p.gv = nullptr;
	switch (s.type)
	{
	case B3G_SHAPE_SPHERE:
		p.lv[0] = sph_center(s);
		p.count = 1;
		p.radius = sph_radius(s);
		break;
	case B3G_SHAPE_CAPSULE:
		p.lv[0] = cap_v1(s);
		p.lv[1] = cap_v2(s);
		p.count = 2;
		p.radius = cap_radius(s);
		break;
	case B3G_SHAPE_TRIANGLE:
		p.lv[0] = V3{s.p0.x, s.p0.y, s.p0.z};
		p.lv[1] = V3{s.p0.w, s.p1.x, s.p1.y};
		p.lv[2] = V3{s.p1.z, s.p1.w, s.p2.x};
		p.count = 3;
		p.radius = s.p2.y;
		break;
	default:
	{
		HullRef h = hull_ref(S, s.hull);
		p = hull_proxy(h, hull_radius(s));
		break;
	}
	}
	return p;
}

// Contacts listed in one bucket, one thread each (spheres_apart: the exact
// cull of collide_common.cuh, repeated here for contacts that reach these
// kernels without k_bucket, i.e. wake-ups and b3g_collide_pairs).
template <int BUCKET>
__global__ void __launch_bounds__(128, 4) k_convex(NPArgs a)
{
	uint32_t n = *a.listCount;
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = a.list[t];
		uint32_t fa = a.pairA[c], fb = a.pairB[c];
		uint32_t ba = a.S.fixBody[fa], bb = a.S.fixBody[fb];
		XF xfA = a.exA ? load_xf7(a.exA + 7 * (size_t)c) : body_xf(a.S, ba);
		XF xfB = a.exB ? load_xf7(a.exB + 7 * (size_t)c) : body_xf(a.S, bb);
		DevManifold& m = a.man[c];
		man_clear(m);
		if (spheres_apart(a.S, fa, xfA, fb, xfB) ||
			(BUCKET == BK_HULL_CAPSULE && hull_capsule_apart(a.S, fa, xfA, fb, xfB)))
		{
			finish_convex(a, c, m);
			a.cache[c] = make_uint4(B3G_NULL, B3G_NULL, B3G_NULL, B3G_NULL);
			continue;
		}
		ShapeP sa = load_shape(a.S, fa), sb = load_shape(a.S, fb);
		if (BUCKET == BK_SPHERES)
			collide_spheres(m, xfA, sa, xfB, sb);
		else if (BUCKET == BK_CAPSULE_SPHERE)
			collide_capsule_sphere(m, xfA, sa, xfB, sb);
		else if (BUCKET == BK_CAPSULES)
			collide_capsules(m, xfA, sa, xfB, sb);
		else if (BUCKET == BK_HULL_SPHERE)
		{
			if (hull_sphere_faces(m, a.S, xfA, sa, xfB, sb))
			{
				// The GJK runs in k_hull_sphere_gjk, which finishes the contact.
				const uint32_t act = __activemask();
				const uint32_t lane = threadIdx.x & 31u;
				const uint32_t leader = __ffs(act) - 1;
				uint32_t base = 0;
				if (lane == leader)
					base = atomicAdd(a.hsPostCount, __popc(act));
				base = __shfl_sync(act, base, leader);
				a.hsPost[base + __popc(act & ((1u << lane) - 1u))] = c;
				continue;
			}
		}
		else if (BUCKET == BK_HULL_CAPSULE)
		{
			GJKOut q;
			if (hull_capsule_gjk(a.S, xfA, sa, xfB, sb, q))
			{
				// Within the radii: k_hull_capsule_post builds the manifold
				// and finishes the contact.
				const uint32_t act = __activemask();
				const uint32_t lane = threadIdx.x & 31u;
				const bool deep = !(q.distance > 0.0f);
				const uint32_t deepMask = __ballot_sync(act, deep);
				const uint32_t mine = deep ? deepMask : act & ~deepMask;
				const uint32_t leader = __ffs(mine) - 1;
				uint32_t base = 0;
				if (lane == leader)
					base = atomicAdd(a.hcPostCount + (deep ? 1 : 0), __popc(mine));
				base = __shfl_sync(mine, base, leader);
				const uint32_t k = base + __popc(mine & ((1u << lane) - 1u));
				const uint32_t j = deep ? a.hcPostCap - 1u - k : k;
				a.hcPost[2 * (size_t)j] = make_float4(q.point1.x, q.point1.y, q.point1.z, q.distance);
				a.hcPost[2 * (size_t)j + 1] = make_float4(q.point2.x, q.point2.y, q.point2.z, __uint_as_float(c));
				continue;
			}
		}
		else if (BUCKET == BK_TRIANGLE_SPHERE)
			collide_triangle_sphere(m, xfA, sa, load_wings(a.S, fa), xfB, sb);
		else if (BUCKET == BK_TRIANGLE_CAPSULE)
			collide_triangle_capsule(m, tri_ref(a.S, fa), xfA, sa, load_wings(a.S, fa), xfB, sb);
		finish_convex(a, c, m);
		a.cache[c] = make_uint4(B3G_NULL, B3G_NULL, B3G_NULL, B3G_NULL);
	}
}

// Hull-sphere contacts whose face scan left the GJK to run
// (k_convex<BK_HULL_SPHERE> lists them), one thread each: the warps that run
// a GJK no longer wait on the face scans of the others.
__global__ void __launch_bounds__(128, 4) k_hull_sphere_gjk(NPArgs a)
{
	const uint32_t n = *a.hsPostCount;
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = a.hsPost[t];
		uint32_t fa = a.pairA[c], fb = a.pairB[c];
		uint32_t ba = a.S.fixBody[fa], bb = a.S.fixBody[fb];
		XF xfA = a.exA ? load_xf7(a.exA + 7 * (size_t)c) : body_xf(a.S, ba);
		XF xfB = a.exB ? load_xf7(a.exB + 7 * (size_t)c) : body_xf(a.S, bb);
		ShapeP sa = load_shape(a.S, fa), sb = load_shape(a.S, fb);
		DevManifold& m = a.man[c];
		hull_sphere_gjk(m, a.S, xfA, sa, xfB, sb);
		finish_convex(a, c, m);
		a.cache[c] = make_uint4(B3G_NULL, B3G_NULL, B3G_NULL, B3G_NULL);
	}
}

// Lanes per contact and blocks per SM of k_hull_capsule_post.
constexpr int HC_POST_LANES = 8;
constexpr int HC_POST_BLOCKS = 6;

// Hull-capsule contacts past their GJK (k_convex<BK_HULL_CAPSULE> lists them),
// G lanes per contact: the support-face and SAT scans run on the group's
// lanes, so a warp no longer walks, one lane at a time, the faces and edges
// of every hull in it that needs them.
template <int G>
__global__ void __launch_bounds__(128, HC_POST_BLOCKS) k_hull_capsule_post(NPArgs a)
{
	// The contacts at a distance first, then the overlapping ones, so the
	// groups of a warp mostly take the same branch.
	const uint32_t nSep = a.hcPostCount[0];
	const uint32_t n = nSep + a.hcPostCount[1];
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t gl = lane % G;
	const uint32_t gmask = G == 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (lane - gl));
	const uint32_t groups = gridDim.x * (blockDim.x / G);
	for (uint32_t t = blockIdx.x * (blockDim.x / G) + threadIdx.x / G; t < n; t += groups)
	{
		const uint32_t j = t < nSep ? t : a.hcPostCap - 1u - (t - nSep);
		float4 q0 = a.hcPost[2 * (size_t)j], q1 = a.hcPost[2 * (size_t)j + 1];
		uint32_t c = __float_as_uint(q1.w);
		GJKOut q;
		q.point1 = V3{q0.x, q0.y, q0.z};
		q.point2 = V3{q1.x, q1.y, q1.z};
		q.distance = q0.w;
		q.iterations = 0;
		uint32_t fa = a.pairA[c], fb = a.pairB[c];
		uint32_t ba = a.S.fixBody[fa], bb = a.S.fixBody[fb];
		XF xfA = a.exA ? load_xf7(a.exA + 7 * (size_t)c) : body_xf(a.S, ba);
		XF xfB = a.exB ? load_xf7(a.exB + 7 * (size_t)c) : body_xf(a.S, bb);
		ShapeP sa = load_shape(a.S, fa), sb = load_shape(a.S, fb);
		DevManifold& m = a.man[c];
		hull_capsule_after_gjk<G>(m, a.S, xfA, sa, xfB, sb, q, gl, gmask);
		if (gl == 0)
		{
			finish_convex(a, c, m);
			a.cache[c] = make_uint4(B3G_NULL, B3G_NULL, B3G_NULL, B3G_NULL);
		}
	}
}

// Sensor contacts: touching = b3TestOverlap (collision.cpp:104-113), no manifolds.
__global__ void k_sensor(NPArgs a)
{
	uint32_t n = *a.listCount;
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = a.list[t];
		uint32_t fa = a.pairA[c], fb = a.pairB[c];
		XF xfA = body_xf(a.S, a.S.fixBody[fa]), xfB = body_xf(a.S, a.S.fixBody[fb]);
		GProxy pa = shape_proxy(a.S, load_shape(a.S, fa));
		GProxy pb = shape_proxy(a.S, load_shape(a.S, fb));
		GJKOut q = gjk(xfA, pa, xfB, pb, true);
		const float kTol = 10.0f * B3G_EPSILON;
		uint32_t touching = q.distance <= kTol ? 1u : 0u;
		int32_t prev = a.prevIndex[c];
		uint32_t begun = prev < 0 ? 1u : 0u;
		a.cstate[c] = touching | (begun << 16);
		man_clear(a.man[c]);
		// A hull-hull sensor contact keeps the b3FeatureCache it was built
		// with: e_empty (sat.h:69), the other fields unset.
		bool hulls = a.S.fixType[fa] == B3G_SHAPE_HULL && a.S.fixType[fb] == B3G_SHAPE_HULL;
		a.cache[c] = make_uint4(hulls ? 0u : B3G_NULL, B3G_NULL, B3G_NULL, B3G_NULL);
	}
}

// Convex contacts k_bucket found apart (spheres_apart): the routine would
// return no point, so the manifold is empty; warm start and flags as in k_convex.
__global__ void k_apart(NPArgs a)
{
	uint32_t n = *a.listCount;
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = a.list[t];
		DevManifold& m = a.man[c];
		man_clear(m);
		finish_convex(a, c, m);
		a.cache[c] = make_uint4(B3G_NULL, B3G_NULL, B3G_NULL, B3G_NULL);
	}
}

// Contacts whose bodies are both inactive keep their state (contact_manager.cpp:262-268).
__global__ void k_inactive(NPArgs a)
{
	uint32_t n = *a.listCount;
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = a.list[t];
		int32_t prev = a.prevIndex[c];
		if (prev >= 0)
		{
			a.cstate[c] = a.prevState[prev] & ~(1u << 16);
			a.cache[c] = a.prevCache[prev];
			a.man[c] = a.prevMan[prev];
			if (a.impN && ((a.prevState[prev] >> 8) & 0xFFu) > 0)
			{
				// The host solver's impulses live in the skipped contact's
				// manifold as it does in the reference's.
				DevManifold& m = a.man[c];
				m.tangentImpulse[0] = a.impT[2 * prev + 0];
				m.tangentImpulse[1] = a.impT[2 * prev + 1];
				m.motorImpulse = a.impM[prev];
				for (uint32_t j = 0; j < m.pointCount && j < 4; ++j)
					m.points[j].normalImpulse = a.impN[4 * prev + j];
			}
			if (a.extraCur && ((a.prevState[prev] >> 8) & 0xFFu) > 1)
			{
				a.extraCur[2 * (size_t)c] = a.extraPrev[2 * (size_t)prev];
				a.extraCur[2 * (size_t)c + 1] = a.extraPrev[2 * (size_t)prev + 1];
			}
		}
		else
		{
			a.cstate[c] = 1u << 16;
			a.cache[c] = make_uint4(0, B3G_NULL, B3G_NULL, B3G_NULL);
			man_clear(a.man[c]);
		}
	}
}

// Mesh work items whose other shape is a sphere or a capsule (the mesh is
// fixture A, the primary order): one triangle each (b3MeshAndSphereContact /
// b3MeshAndCapsuleContact::Evaluate, mesh_sphere_contact.cpp:42-50,
// mesh_capsule_contact.cpp:42-50), points tagged with the triangle
// (mesh_contact.cpp:343-356). Sensor contacts record the triangle's overlap
// (b3TestOverlap with the child index, collision.cpp:104-113) in pointCount.
__global__ void __launch_bounds__(128) k_mesh_items_convex(NPArgs a, Buffers B)
{
	uint32_t n = min(B.counters[CTR_MESH_PAIRS], B.meshPairCap);
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		uint32_t c = B.meshPairC[i], t = B.meshPairT[i];
		uint32_t fa = a.pairA[c], fb = a.pairB[c];
		uint32_t tb = a.S.fixType[fb];
		if (a.S.fixType[fa] != B3G_SHAPE_MESH || (tb != B3G_SHAPE_SPHERE && tb != B3G_SHAPE_CAPSULE))
			continue;
		XF xfA = body_xf(a.S, a.S.fixBody[fa]), xfB = body_xf(a.S, a.S.fixBody[fb]);
		MeshTri tri;
		mesh_triangle(a.S, fa, t, tri);
		ShapeP st;
		st.type = B3G_SHAPE_TRIANGLE;
		st.p0 = make_float4(tri.v[0].x, tri.v[0].y, tri.v[0].z, tri.v[1].x);
		st.p1 = make_float4(tri.v[1].y, tri.v[1].z, tri.v[2].x, tri.v[2].y);
		st.p2 = make_float4(tri.v[2].z, tri.radius, 0.0f, 0.0f);
		st.hull = 0;
		ShapeP sb = load_shape(a.S, fb);
		DevManifold& m = B.meshPairMan[i];
		man_clear(m);
		if ((a.S.fixFlags[fa] | a.S.fixFlags[fb]) & B3G_FIXTURE_SENSOR)
		{
			GJKOut q = gjk(xfA, shape_proxy(a.S, st), xfB, shape_proxy(a.S, sb), true);
			m.pointCount = q.distance <= 10.0f * B3G_EPSILON ? 1u : 0u;
			continue;
		}
		TriWings wg;
		for (int k = 0; k < 3; ++k)
		{
			wg.e[k] = V3{tri.wing[k].x, tri.wing[k].y, tri.wing[k].z};
			wg.has[k] = tri.wing[k].w != 0.0f;
		}
		if (tb == B3G_SHAPE_SPHERE)
			collide_triangle_sphere(m, xfA, st, wg, xfB, sb);
		else
			collide_triangle_capsule(m, mesh_tri_ref(tri), xfA, st, wg, xfB, sb);
		for (uint32_t j = 0; j < m.pointCount; ++j)
			m.points[j].triangleKey = t;
	}
}

} // namespace

// Bucket kernel k of launch_convex_buckets (the order of B3G_TUNE_CONVEX).
void launch_convex_one(int k, const NPArgs& base, const uint32_t* lists, const uint32_t* counts, uint32_t cap,
	const Tune& tune, cudaStream_t s)
{
	static const uint32_t buckets[B3G_CONVEX_KERNELS] = {BK_SPHERES, BK_CAPSULE_SPHERE, BK_CAPSULES,
		BK_TRIANGLE_SPHERE, BK_TRIANGLE_CAPSULE, BK_HULL_SPHERE, BK_HULL_CAPSULE, BK_SENSOR, BK_INACTIVE};
	const uint32_t bk = buckets[k];
	NPArgs a = base;
	a.list = lists + (size_t)bk * cap;
	a.listCount = counts + bk;
	const int blocks = persistent_blocks((int)tune.v[B3G_TUNE_CONVEX + k]);
	switch (k)
	{
	case 0:
		k_convex<BK_SPHERES><<<blocks, 128, 0, s>>>(a);
		break;
	case 1:
		k_convex<BK_CAPSULE_SPHERE><<<blocks, 128, 0, s>>>(a);
		break;
	case 2:
		k_convex<BK_CAPSULES><<<blocks, 128, 0, s>>>(a);
		break;
	case 3:
		k_convex<BK_TRIANGLE_SPHERE><<<blocks, 128, 0, s>>>(a);
		break;
	case 4:
		k_convex<BK_TRIANGLE_CAPSULE><<<blocks, 128, 0, s>>>(a);
		break;
	case 5:
		cudaMemsetAsync(a.hsPostCount, 0, sizeof(uint32_t), s);
		k_convex<BK_HULL_SPHERE><<<blocks, 128, 0, s>>>(a);
		k_hull_sphere_gjk<<<persistent_blocks(4), 128, 0, s>>>(a);
		break;
	case 6:
		cudaMemsetAsync(a.hcPostCount, 0, 2 * sizeof(uint32_t), s);
		k_convex<BK_HULL_CAPSULE><<<blocks, 128, 0, s>>>(a);
		k_hull_capsule_post<HC_POST_LANES><<<persistent_blocks(HC_POST_BLOCKS), 128, 0, s>>>(a);
		break;
	case 7:
		k_sensor<<<blocks, 128, 0, s>>>(a);
		break;
	default:
		k_inactive<<<blocks, 128, 0, s>>>(a);
		break;
	}
}

void launch_convex_buckets(const NPArgs& base, const uint32_t* lists, const uint32_t* counts, uint32_t cap,
	const Tune& tune, cudaStream_t s)
{
	for (int k = 0; k < B3G_CONVEX_KERNELS; ++k)
		launch_convex_one(k, base, lists, counts, cap, tune, s);
}

void launch_apart(const NPArgs& base, const uint32_t* list, const uint32_t* count, cudaStream_t s)
{
	NPArgs a = base;
	a.list = list;
	a.listCount = count;
	k_apart<<<persistent_blocks(4), 128, 0, s>>>(a);
}

void launch_mesh_items_convex(const NPArgs& a, const Buffers& B, cudaStream_t s)
{
	k_mesh_items_convex<<<persistent_blocks(4), 128, 0, s>>>(a, B);
}

// Loop-trip counters of the reference's narrowphase, for the algorithmic flop
// count of a collision pass. TEST INFRASTRUCTURE, linked into the FP64 oracle
// build only (oracle/Makefile: libb3ref64.so), never into the product.
//
// The reference's functions stay unmodified: the linker's --wrap sends every
// call between translation units of the reference to the __wrap_ function
// here, which adds up trips from its arguments (hull sizes, iteration counts
// returned, or a recount with the reference's own primitives) and calls the
// reference's function (__real_). Flops per trip are the constants of
// flops.h. Calls inside one reference translation unit (e.g. ReadFace from
// ReadState) are not wrapped; their callers' wrappers count them.
//
// refc_reset() clears the counters, refc_read() copies them out
// (RC_COUNT doubles, the RC_* order below).

#include <stdint.h>
#include <string.h>

#include <bounce/bounce.h>
#include <bounce/collision/clip.h>
#include <bounce/collision/cluster.h>
#include <bounce/collision/gjk/gjk.h>
#include <bounce/collision/gjk/gjk_proxy.h>
#include <bounce/collision/sat/sat.h>
#include <bounce/collision/geometry/capsule.h>
#include <bounce/collision/sat/sat_hull_edge.h>

#include "flops.h"

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {

enum
{
	RC_FLOPS = 0,      // total flops (flops.h constants x trips)
	RC_SPHERES,        // b3Collide* calls per routine
	RC_CAPSULE_SPHERE,
	RC_CAPSULES,
	RC_HULL_SPHERE,
	RC_HULL_CAPSULE,
	RC_HULLS,
	RC_FACE_QUERIES,   // b3QueryFaceSeparation calls (hull-hull)
	RC_FACE_TRIPS,     // (plane, vertex) trips
	RC_EDGE_QUERIES,   // b3QueryEdgeSeparation calls (hull-hull)
	RC_EDGE_PAIRS,     // edge pairs tested
	RC_EDGE_QUALIFIED, // edge pairs past the Gauss-map test
	RC_GJK_CALLS,
	RC_GJK_ITERS,
	RC_CLIP_PLANES,
	RC_CLIP_VERTICES,
	RC_CACHE_READS,
	RC_HULL_SPHERE_PLANES,
	RC_FLOPS_SAT,      // flops of the hull-hull and hull-capsule SAT queries
	RC_FLOPS_GJK,
	RC_FLOPS_CLIP,     // clipping and reduction
	RC_COUNT
};

double g_rc[RC_COUNT];

inline void add(int what, double n) { g_rc[what] += n; }
inline void flops(double f, int part = -1)
{
	g_rc[RC_FLOPS] += f;
	if (part >= 0)
		g_rc[part] += f;
}

// b3IsMinkowskiFace of sat.cpp:60-71, restated for the count of qualified
// edge pairs (the reference's copy is file-static).
inline bool minkowski(const b3Vec3& A, const b3Vec3& B, const b3Vec3& BxA, const b3Vec3& C, const b3Vec3& D,
	const b3Vec3& DxC)
{
	scalar ADC = b3Dot(A, DxC), BDC = b3Dot(B, DxC);
	scalar CBA = b3Dot(C, BxA), DBA = b3Dot(D, BxA);
	return CBA * DBA < scalar(0) && ADC * BDC < scalar(0) && CBA * BDC > scalar(0);
}

// Qualified edge pairs of b3QueryEdgeSeparation (sat.cpp:111-174), with its
// loop structure and the same Gauss-map test.
double qualified_pairs(const b3Transform& xf1, const b3Hull* h1, const b3Transform& xf2, const b3Hull* h2)
{
	b3Transform xf = b3MulT(xf2, xf1);
	double q = 0;
	for (uint32 i = 0; i < h1->edgeCount; i += 2)
	{
		const b3HalfEdge* e1 = h1->GetEdge(i);
		const b3HalfEdge* t1 = h1->GetEdge(i + 1);
		b3Vec3 P1 = xf * h1->GetVertex(e1->origin);
		b3Vec3 Q1 = xf * h1->GetVertex(t1->origin);
		b3Vec3 E1 = Q1 - P1;
		b3Vec3 U1 = b3Mul(xf.rotation, h1->GetPlane(e1->face).normal);
		b3Vec3 V1 = b3Mul(xf.rotation, h1->GetPlane(t1->face).normal);
		for (uint32 j = 0; j < h2->edgeCount; j += 2)
		{
			const b3HalfEdge* e2 = h2->GetEdge(j);
			const b3HalfEdge* t2 = h2->GetEdge(j + 1);
			b3Vec3 E2 = h2->GetVertex(t2->origin) - h2->GetVertex(e2->origin);
			b3Vec3 U2 = h2->GetPlane(e2->face).normal;
			b3Vec3 V2 = h2->GetPlane(t2->face).normal;
			if (minkowski(U1, V1, -E1, -U2, -V2, -E2))
				q += 1;
		}
	}
	return q;
}

} // namespace

REF_API void refc_reset() { memset(g_rc, 0, sizeof(g_rc)); }

REF_API uint32_t refc_read(double* out, uint32_t capacity)
{
	uint32_t n = capacity < RC_COUNT ? capacity : RC_COUNT;
	memcpy(out, g_rc, sizeof(double) * n);
	return n;
}

// Declarations of the real and wrapping symbols, by mangled name (the FP64
// build: scalar = double).
#define WRAPPED(ret, mangled, ...)                   \
	extern "C" ret __real_##mangled(__VA_ARGS__);   \
	extern "C" ret __wrap_##mangled(__VA_ARGS__)

// --- SAT queries -----------------------------------------------------------

WRAPPED(b3FaceQuery, _Z21b3QueryFaceSeparationRK11b3TransformPK6b3HullS1_S4_, const b3Transform& xf1,
	const b3Hull* h1, const b3Transform& xf2, const b3Hull* h2)
{
	add(RC_FACE_QUERIES, 1);
	double trips = (double)h1->faceCount * h2->vertexCount;
	add(RC_FACE_TRIPS, trips);
	flops(FL_FACE_SETUP + (double)FL_FACE_PLANE * h1->faceCount + FL_FACE_TRIP * trips, RC_FLOPS_SAT);
	return __real__Z21b3QueryFaceSeparationRK11b3TransformPK6b3HullS1_S4_(xf1, h1, xf2, h2);
}

WRAPPED(b3EdgeQuery, _Z21b3QueryEdgeSeparationRK11b3TransformPK6b3HullS1_S4_, const b3Transform& xf1,
	const b3Hull* h1, const b3Transform& xf2, const b3Hull* h2)
{
	add(RC_EDGE_QUERIES, 1);
	double outer = h1->edgeCount / 2, pairs = outer * (h2->edgeCount / 2);
	double q = qualified_pairs(xf1, h1, xf2, h2);
	add(RC_EDGE_PAIRS, pairs);
	add(RC_EDGE_QUALIFIED, q);
	flops(FL_EDGE_SETUP + FL_EDGE_OUTER * outer + FL_EDGE_PAIR * pairs + FL_EDGE_QUALIFIED * q, RC_FLOPS_SAT);
	return __real__Z21b3QueryEdgeSeparationRK11b3TransformPK6b3HullS1_S4_(xf1, h1, xf2, h2);
}

WRAPPED(b3FaceQuery, _Z21b3QueryFaceSeparationRK11b3TransformPK6b3HullS1_PK9b3Capsule, const b3Transform& xf1,
	const b3Hull* h1, const b3Transform& xf2, const b3Capsule* c2)
{
	flops(FL_FACE_SEG_SETUP + (double)FL_FACE_SEG_PLANE * h1->faceCount, RC_FLOPS_SAT);
	return __real__Z21b3QueryFaceSeparationRK11b3TransformPK6b3HullS1_PK9b3Capsule(xf1, h1, xf2, c2);
}

WRAPPED(b3EdgeQuery, _Z21b3QueryEdgeSeparationRK11b3TransformPK6b3HullS1_PK9b3Capsule, const b3Transform& xf1,
	const b3Hull* h1, const b3Transform& xf2, const b3Capsule* c2)
{
	// Every hull edge past the Gauss-map test is projected (an upper bound of
	// the qualified count: at most the edges whose faces straddle the segment).
	double pairs = h1->edgeCount / 2;
	flops(FL_EDGE_SEG_SETUP + FL_EDGE_SEG_PAIR * pairs + FL_EDGE_SEG_QUALIFIED * 2.0, RC_FLOPS_SAT);
	return __real__Z21b3QueryEdgeSeparationRK11b3TransformPK6b3HullS1_PK9b3Capsule(xf1, h1, xf2, c2);
}

WRAPPED(b3CacheType, _ZN14b3FeatureCache9ReadStateERK11b3TransformPK6b3HullS2_S5_d, b3FeatureCache* self,
	const b3Transform& xf1, const b3Hull* h1, const b3Transform& xf2, const b3Hull* h2, scalar r)
{
	add(RC_CACHE_READS, 1);
	b3FeatureType t = self->cacheType == b3CacheType::e_empty ? b3FeatureType::e_face1 : self->featureType;
	if (t == b3FeatureType::e_edges)
		flops(FL_CACHE_EDGES, RC_FLOPS_SAT);
	else if (t == b3FeatureType::e_face1)
		flops(FL_FACE_SETUP + FL_CACHE_FACE + (double)FL_FACE_TRIP * h2->vertexCount, RC_FLOPS_SAT);
	else if (t == b3FeatureType::e_face2)
		flops(FL_FACE_SETUP + FL_CACHE_FACE + (double)FL_FACE_TRIP * h1->vertexCount, RC_FLOPS_SAT);
	return __real__ZN14b3FeatureCache9ReadStateERK11b3TransformPK6b3HullS2_S5_d(self, xf1, h1, xf2, h2, r);
}

// --- GJK -------------------------------------------------------------------

static void gjk_flops(const b3GJKProxy& p1, const b3GJKProxy& p2, uint32 iters)
{
	add(RC_GJK_CALLS, 1);
	add(RC_GJK_ITERS, iters);
	flops(FL_GJK_CALL + (double)iters * (FL_GJK_ITER + FL_GJK_SOLVE +
		FL_GJK_SUPPORT_VERTEX * (double)(p1.m_count + p2.m_count)), RC_FLOPS_GJK);
}

WRAPPED(b3GJKOutput, _Z5b3GJKRK11b3TransformRK10b3GJKProxyS1_S4_b, const b3Transform& xf1, const b3GJKProxy& p1,
	const b3Transform& xf2, const b3GJKProxy& p2, bool applyRadius)
{
	b3GJKOutput o = __real__Z5b3GJKRK11b3TransformRK10b3GJKProxyS1_S4_b(xf1, p1, xf2, p2, applyRadius);
	gjk_flops(p1, p2, o.iterations);
	return o;
}

WRAPPED(b3GJKOutput, _Z5b3GJKRK11b3TransformRK10b3GJKProxyS1_S4_bP14b3SimplexCache, const b3Transform& xf1,
	const b3GJKProxy& p1, const b3Transform& xf2, const b3GJKProxy& p2, bool applyRadius, b3SimplexCache* cache)
{
	b3GJKOutput o = __real__Z5b3GJKRK11b3TransformRK10b3GJKProxyS1_S4_bP14b3SimplexCache(xf1, p1, xf2, p2,
		applyRadius, cache);
	gjk_flops(p1, p2, o.iterations);
	return o;
}

// --- Clipping and reduction ------------------------------------------------

// b3ClipPolygonToFaceSidePlanes (clip.cpp:244-281): its face loop is run again
// with the reference's b3ClipPolygonToPlane to count the vertices each side
// plane sees and the edges that cross it.
WRAPPED(void, _Z29b3ClipPolygonToFaceSidePlanesR7b3ArrayI12b3ClipVertexERKS1_RK11b3TransformdjPK6b3Hull,
	b3ClipPolygon& pOut, const b3ClipPolygon& pIn, const b3Transform& xf, scalar r, uint32 index, const b3Hull* hull)
{
	b3StackArray<b3ClipVertex, 32> cur;
	cur = pIn;
	const b3Face* face = hull->GetFace(index);
	const b3HalfEdge* begin = hull->GetEdge(face->edge);
	const b3HalfEdge* edge = begin;
	do
	{
		uint32 edgeId = uint32(hull->GetEdge(edge->twin)->twin);
		b3Plane plane = hull->GetEdgeSidePlane(edgeId);
		plane.offset += r;
		b3ClipPlane cp;
		cp.edge = edgeId;
		cp.plane = b3Mul(xf, plane);
		uint32 n = cur.Count();
		double crossings = 0;
		scalar d1 = b3Distance(cur.Back().position, cp.plane);
		for (uint32 i = 0; i < n; ++i)
		{
			scalar d2 = b3Distance(cur[i].position, cp.plane);
			if ((d1 <= scalar(0)) != (d2 <= scalar(0)))
				crossings += 1;
			d1 = d2;
		}
		add(RC_CLIP_PLANES, 1);
		add(RC_CLIP_VERTICES, n);
		flops(FL_CLIP_PLANE + FL_CLIP_VERTEX * (double)n + FL_CLIP_CROSSING * crossings, RC_FLOPS_CLIP);
		b3StackArray<b3ClipVertex, 32> next;
		b3ClipPolygonToPlane(next, cur, cp);
		cur = next;
		if (cur.IsEmpty())
			break;
		edge = hull->GetEdge(edge->next);
	} while (edge != begin);
	__real__Z29b3ClipPolygonToFaceSidePlanesR7b3ArrayI12b3ClipVertexERKS1_RK11b3TransformdjPK6b3Hull(pOut, pIn, xf,
		r, index, hull);
}

// b3ClipSegmentToFaceSidePlanes (clip.cpp:202-242): a segment of two vertices
// against each side plane of the face (crossings taken as one per plane).
WRAPPED(uint32, _Z29b3ClipSegmentToFaceSidePlanesP12b3ClipVertexPKS_RK11b3TransformdjPK6b3Hull, b3ClipVertex* vOut,
	const b3ClipVertex* vIn, const b3Transform& xf, scalar r, uint32 index, const b3Hull* hull)
{
	const b3Face* face = hull->GetFace(index);
	const b3HalfEdge* begin = hull->GetEdge(face->edge);
	const b3HalfEdge* edge = begin;
	double planes = 0;
	do
	{
		planes += 1;
		edge = hull->GetEdge(edge->next);
	} while (edge != begin);
	add(RC_CLIP_PLANES, planes);
	add(RC_CLIP_VERTICES, 2 * planes);
	flops(planes * (FL_CLIP_PLANE + 2 * FL_CLIP_VERTEX + FL_CLIP_CROSSING), RC_FLOPS_CLIP);
	return __real__Z29b3ClipSegmentToFaceSidePlanesP12b3ClipVertexPKS_RK11b3TransformdjPK6b3Hull(vOut, vIn, xf, r,
		index, hull);
}

WRAPPED(void, _Z15b3ReducePolygonR7b3ArrayI15b3ClusterVertexERKS1_RK6b3Vec3j, b3ClusterPolygon& pOut,
	const b3ClusterPolygon& pIn, const b3Vec3& normal, uint32 initialPoint)
{
	flops(FL_REDUCE_VERTEX * (double)pIn.Count(), RC_FLOPS_CLIP);
	__real__Z15b3ReducePolygonR7b3ArrayI15b3ClusterVertexERKS1_RK6b3Vec3j(pOut, pIn, normal, initialPoint);
}

// --- Collide routines: calls and closed-form parts -------------------------

WRAPPED(void, _Z16b3CollideSpheresR10b3ManifoldRK11b3TransformPK13b3SphereShapeS3_S6_, b3Manifold& m,
	const b3Transform& xf1, const b3SphereShape* s1, const b3Transform& xf2, const b3SphereShape* s2)
{
	add(RC_SPHERES, 1);
	flops(FL_SPHERES);
	__real__Z16b3CollideSpheresR10b3ManifoldRK11b3TransformPK13b3SphereShapeS3_S6_(m, xf1, s1, xf2, s2);
}

WRAPPED(void, _Z25b3CollideCapsuleAndSphereR10b3ManifoldRK11b3TransformPK14b3CapsuleShapeS3_PK13b3SphereShape,
	b3Manifold& m, const b3Transform& xf1, const b3CapsuleShape* s1, const b3Transform& xf2, const b3SphereShape* s2)
{
	add(RC_CAPSULE_SPHERE, 1);
	flops(FL_CAPSULE_SPHERE);
	__real__Z25b3CollideCapsuleAndSphereR10b3ManifoldRK11b3TransformPK14b3CapsuleShapeS3_PK13b3SphereShape(m, xf1,
		s1, xf2, s2);
}

WRAPPED(void, _Z17b3CollideCapsulesR10b3ManifoldRK11b3TransformPK14b3CapsuleShapeS3_S6_, b3Manifold& m,
	const b3Transform& xf1, const b3CapsuleShape* s1, const b3Transform& xf2, const b3CapsuleShape* s2)
{
	add(RC_CAPSULES, 1);
	flops(FL_CAPSULES);
	__real__Z17b3CollideCapsulesR10b3ManifoldRK11b3TransformPK14b3CapsuleShapeS3_S6_(m, xf1, s1, xf2, s2);
}

// The face loop of b3CollideHullAndSphere (collide_hull_sphere.cpp:39-54)
// leaves at the first plane farther than the radius: its trips are recounted
// with the same test.
WRAPPED(void, _Z22b3CollideHullAndSphereR10b3ManifoldRK11b3TransformPK11b3HullShapeS3_PK13b3SphereShape,
	b3Manifold& m, const b3Transform& xf1, const b3HullShape* s1, const b3Transform& xf2, const b3SphereShape* s2)
{
	add(RC_HULL_SPHERE, 1);
	scalar radius = s1->m_radius + s2->m_radius;
	const b3Hull* h = s1->m_hull;
	b3Vec3 c = b3MulT(xf1, b3Mul(xf2, s2->m_center));
	double trips = 0;
	for (uint32 i = 0; i < h->faceCount; ++i)
	{
		trips += 1;
		if (b3Distance(c, h->GetPlane(i)) > radius)
			break;
	}
	add(RC_HULL_SPHERE_PLANES, trips);
	flops(FL_HULL_SPHERE + FL_HULL_SPHERE_PLANE * trips);
	__real__Z22b3CollideHullAndSphereR10b3ManifoldRK11b3TransformPK11b3HullShapeS3_PK13b3SphereShape(m, xf1, s1,
		xf2, s2);
}

WRAPPED(void, _Z23b3CollideHullAndCapsuleR10b3ManifoldRK11b3TransformPK11b3HullShapeS3_PK14b3CapsuleShape,
	b3Manifold& m, const b3Transform& xf1, const b3HullShape* s1, const b3Transform& xf2, const b3CapsuleShape* s2)
{
	add(RC_HULL_CAPSULE, 1);
	flops(FL_HULL_CAPSULE);
	__real__Z23b3CollideHullAndCapsuleR10b3ManifoldRK11b3TransformPK11b3HullShapeS3_PK14b3CapsuleShape(m, xf1, s1,
		xf2, s2);
}

WRAPPED(void, _Z14b3CollideHullsR10b3ManifoldRK11b3TransformPK11b3HullShapeS3_S6_R14b3FeatureCacheS3_S3_,
	b3Manifold& m, const b3Transform& xf1, const b3HullShape* s1, const b3Transform& xf2, const b3HullShape* s2,
	b3FeatureCache& cache, const b3Transform& xf01, const b3Transform& xf02)
{
	add(RC_HULLS, 1);
	flops(FL_HULLS);
	__real__Z14b3CollideHullsR10b3ManifoldRK11b3TransformPK11b3HullShapeS3_S6_R14b3FeatureCacheS3_S3_(m, xf1, s1,
		xf2, s2, cache, xf01, xf02);
}

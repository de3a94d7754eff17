// Shared narrowphase pieces: hull accessors, clipping (clip.cpp), manifold
// initialisation and warm-start matching (collision.cpp:23-61, contact.cpp:399-501).
#pragma once

#include "b3g_internal.cuh"
#include "gjk.cuh"

#define B3G_NULL_EDGE 0xFFFFFFFFu
#define B3G_NULL_TRIANGLE 0xFFFFFFFFu
#define B3G_MAX_POLY 64 // b3StackArray<b3ClipVertex, 32> grows; 64 bounds every hull here

struct HullRef
{
	const float4* v;
	const uint4* e; // origin, face, prev, next; twin = i ^ 1
	const uint32_t* f;
	const float4* p;
	uint32_t vCnt, eCnt, fCnt;
	V3 centroid;
};

__device__ __forceinline__ HullRef hull_ref(const DevScene& S, uint32_t h)
{
	HullDesc d = S.hulls[h];
	HullRef r;
	r.v = S.hverts + d.vOff;
	r.e = S.hedges + d.eOff;
	r.f = S.hfaces + d.fOff;
	r.p = S.hplanes + d.fOff;
	r.vCnt = d.vCnt;
	r.eCnt = d.eCnt;
	r.fCnt = d.fCnt;
	r.centroid = V3{d.cx, d.cy, d.cz};
	return r;
}

// b3TriangleHull (triangle_hull.h:26-70): every triangle hull has the same
// topology, two faces of three half-edges each (twin = i ^ 1; origin, face,
// prev, next), so only its vertices, planes and centroid are stored per
// fixture.
__device__ const uint4 kTriEdges[6] = {
	{0, 0, 4, 2}, {1, 1, 3, 5}, {1, 0, 0, 4}, {2, 1, 5, 1}, {2, 0, 2, 0}, {0, 1, 1, 3}};
__device__ const uint32_t kTriFaces[2] = {0, 1};

__device__ __forceinline__ HullRef tri_ref(const DevScene& S, uint32_t fix)
{
	const float4* t = S.fixTri + 6 * (size_t)fix;
	HullRef r;
	r.v = t;
	r.e = kTriEdges;
	r.f = kTriFaces;
	r.p = t + 3;
	r.vCnt = 3;
	r.eCnt = 6;
	r.fCnt = 2;
	float4 c = t[5];
	r.centroid = V3{c.x, c.y, c.z};
	return r;
}

__device__ __forceinline__ V3 hv(const HullRef& h, uint32_t i)
{
	float4 w = h.v[i];
	return V3{w.x, w.y, w.z};
}
__device__ __forceinline__ PL hp(const HullRef& h, uint32_t i)
{
	float4 w = h.p[i];
	return PL{V3{w.x, w.y, w.z}, w.w};
}
__device__ __forceinline__ uint32_t he_origin(const HullRef& h, uint32_t i) { return h.e[i].x; }
__device__ __forceinline__ uint32_t he_face(const HullRef& h, uint32_t i) { return h.e[i].y; }
__device__ __forceinline__ uint32_t he_prev(const HullRef& h, uint32_t i) { return h.e[i].z; }
__device__ __forceinline__ uint32_t he_next(const HullRef& h, uint32_t i) { return h.e[i].w; }

// b3Hull::GetSupportVertex (hull.h:105-119): first maximum.
__device__ __forceinline__ uint32_t hull_support_vertex(const HullRef& h, V3 d)
{
	uint32_t maxIndex = 0;
	float maxProj = dot(d, hv(h, 0));
	for (uint32_t i = 1; i < h.vCnt; ++i)
	{
		float proj = dot(d, hv(h, i));
		if (proj > maxProj)
		{
			maxIndex = i;
			maxProj = proj;
		}
	}
	return maxIndex;
}

// b3Hull::GetSupportFace (hull.h:121-135).
__device__ __forceinline__ uint32_t hull_support_face(const HullRef& h, V3 d)
{
	uint32_t maxIndex = 0;
	float maxProj = dot(d, hp(h, 0).n);
	for (uint32_t i = 1; i < h.fCnt; ++i)
	{
		float proj = dot(d, hp(h, i).n);
		if (proj > maxProj)
		{
			maxIndex = i;
			maxProj = proj;
		}
	}
	return maxIndex;
}

// b3Hull::GetEdgeSidePlane (hull.h:137-152).
__device__ __forceinline__ PL hull_edge_side_plane(const HullRef& h, uint32_t index)
{
	uint4 e = h.e[index];
	uint32_t twinOrigin = h.e[index ^ 1u].x;
	PL face = hp(h, e.y);
	V3 P = hv(h, e.x);
	V3 Q = hv(h, twinOrigin);
	V3 E = Q - P;
	V3 D = cross(E, face.n);
	PL pl;
	pl.n = normalized(D);
	pl.d = dot(pl.n, P);
	return pl;
}

// ---------------------------------------------------------------------------
// Clipping (clip.cpp).

struct FPair
{
	uint32_t inEdge1, outEdge1, inEdge2, outEdge2;
};

struct ClipV
{
	V3 pos;
	FPair pair;
};

__device__ __forceinline__ FPair mkpair(uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
	return FPair{a, b, c, d};
}

// b3ClipSegmentToPlane (clip.cpp:62-98).
__device__ __forceinline__ uint32_t clip_segment_to_plane(ClipV vOut[2], const ClipV vIn[2], PL plane,
	uint32_t edge)
{
	uint32_t numOut = 0;
	float d1 = pdist(vIn[0].pos, plane);
	float d2 = pdist(vIn[1].pos, plane);
	if (d1 <= 0.0f)
		vOut[numOut++] = vIn[0];
	if (d2 <= 0.0f)
		vOut[numOut++] = vIn[1];
	if (d1 <= 0.0f && d2 > 0.0f)
	{
		float fraction = d1 / (d1 - d2);
		vOut[numOut].pos = vIn[0].pos + fraction * (vIn[1].pos - vIn[0].pos);
		vOut[numOut].pair = mkpair(edge, B3G_NULL_EDGE, vIn[0].pair.outEdge2, B3G_NULL_EDGE);
		++numOut;
	}
	else if (d1 > 0.0f && d2 <= 0.0f)
	{
		float fraction = d1 / (d1 - d2);
		vOut[numOut].pos = vIn[0].pos + fraction * (vIn[1].pos - vIn[0].pos);
		vOut[numOut].pair = mkpair(B3G_NULL_EDGE, edge, B3G_NULL_EDGE, vIn[1].pair.inEdge2);
		++numOut;
	}
	return numOut;
}

// b3BuildSegment (clip.cpp:24-30).
__device__ __forceinline__ void build_segment(ClipV v[2], V3 a, V3 b)
{
	v[0].pos = a;
	v[0].pair = mkpair(B3G_NULL_EDGE, B3G_NULL_EDGE, 0, 0);
	v[1].pos = b;
	v[1].pair = mkpair(B3G_NULL_EDGE, B3G_NULL_EDGE, 1, 0);
}

// b3ClipSegmentToSegmentSidePlanes (clip.cpp:153-199).
__device__ __forceinline__ uint32_t clip_segment_to_segment_side_planes(ClipV vOut[2], const ClipV vIn[2],
	V3 P1, V3 Q1)
{
	vOut[0] = vIn[0];
	vOut[1] = vIn[1];
	V3 E1 = Q1 - P1;
	PL plane1;
	plane1.n = normalized(E1);
	plane1.d = dot(plane1.n, Q1);
	ClipV c1[2] = {vOut[0], vOut[1]};
	uint32_t numOut = clip_segment_to_plane(c1, vOut, plane1, 0);
	vOut[0] = c1[0];
	vOut[1] = c1[1];
	if (numOut < 2)
		return numOut;
	PL plane2;
	plane2.n = -plane1.n;
	plane2.d = dot(plane2.n, P1);
	ClipV c2[2] = {vOut[0], vOut[1]};
	numOut = clip_segment_to_plane(c2, vOut, plane2, 1);
	vOut[0] = c2[0];
	vOut[1] = c2[1];
	return numOut;
}

// b3ClipSegmentToFaceSidePlanes (clip.cpp:202-241).
__device__ __forceinline__ uint32_t clip_segment_to_face_side_planes(ClipV vOut[2], const ClipV vIn[2],
	const XF& xf, float r, uint32_t index, const HullRef& h)
{
	vOut[0] = vIn[0];
	vOut[1] = vIn[1];
	uint32_t numOut = 0;
	uint32_t begin = h.f[index];
	uint32_t edge = begin;
	uint32_t guard = 0;
	do
	{
		if (++guard > h.eCnt)
			return 0; // face loops are validated on upload; never loop forever
		uint32_t edgeId = edge; // twin of the twin
		PL plane = hull_edge_side_plane(h, edgeId);
		plane.d += r;
		PL cp = pmul(xf, plane);
		ClipV cs[2] = {vOut[0], vOut[1]};
		numOut = clip_segment_to_plane(cs, vOut, cp, edgeId);
		vOut[0] = cs[0];
		vOut[1] = cs[1];
		if (numOut == 0)
			return 0;
		edge = he_next(h, edge);
	} while (edge != begin);
	return numOut;
}

struct Poly
{
	ClipV v[B3G_MAX_POLY];
	uint32_t n;
};

// b3BuildPolygon (clip.cpp:33-58).
__device__ __forceinline__ bool build_polygon(Poly& out, const XF& xf, uint32_t index, const HullRef& h)
{
	out.n = 0;
	uint32_t begin = h.f[index];
	uint32_t edge = begin;
	do
	{
		if (out.n >= B3G_MAX_POLY)
			return false;
		uint32_t inEdge = he_prev(h, edge);
		uint32_t outEdge = edge;
		ClipV& cv = out.v[out.n++];
		cv.pos = xmul(xf, hv(h, he_origin(h, edge)));
		cv.pair = mkpair(B3G_NULL_EDGE, B3G_NULL_EDGE, inEdge, outEdge);
		edge = he_next(h, edge);
	} while (edge != begin);
	return true;
}

// b3ClipPolygonToPlane (clip.cpp:101-150).
__device__ __forceinline__ bool clip_polygon_to_plane(Poly& out, const Poly& in, PL plane, uint32_t edge)
{
	out.n = 0;
	ClipV v1 = in.v[in.n - 1];
	float d1 = pdist(v1.pos, plane);
	for (uint32_t i = 0; i < in.n; ++i)
	{
		ClipV v2 = in.v[i];
		float d2 = pdist(v2.pos, plane);
		if (d1 <= 0.0f && d2 <= 0.0f)
		{
			if (out.n >= B3G_MAX_POLY)
				return false;
			out.v[out.n++] = v2;
		}
		else if (d1 <= 0.0f && d2 > 0.0f)
		{
			if (out.n >= B3G_MAX_POLY)
				return false;
			float fraction = d1 / (d1 - d2);
			ClipV& vx = out.v[out.n++];
			vx.pos = v1.pos + fraction * (v2.pos - v1.pos);
			vx.pair = mkpair(edge, B3G_NULL_EDGE, v1.pair.outEdge2, B3G_NULL_EDGE);
		}
		else if (d1 > 0.0f && d2 <= 0.0f)
		{
			if (out.n + 2 > B3G_MAX_POLY)
				return false;
			float fraction = d1 / (d1 - d2);
			ClipV& vx = out.v[out.n++];
			vx.pos = v1.pos + fraction * (v2.pos - v1.pos);
			vx.pair = mkpair(B3G_NULL_EDGE, edge, B3G_NULL_EDGE, v2.pair.inEdge2);
			out.v[out.n++] = v2;
		}
		v1 = v2;
		d1 = d2;
	}
	return true;
}

// b3ClipPolygonToFaceSidePlanes (clip.cpp:244-281). Ping-pongs between two
// polygons; returns a pointer to the one holding the result.
__device__ __forceinline__ Poly* clip_polygon_to_face_side_planes(Poly& a, Poly& b, const XF& xf, float r,
	uint32_t index, const HullRef& h, bool& ok)
{
	Poly* in = &a;
	Poly* out = &b;
	uint32_t begin = h.f[index];
	uint32_t edge = begin;
	ok = true;
	uint32_t guard = 0;
	do
	{
		if (++guard > h.eCnt)
		{
			ok = false;
			return in;
		}
		uint32_t edgeId = edge;
		PL plane = hull_edge_side_plane(h, edgeId);
		plane.d += r;
		PL cp = pmul(xf, plane);
		if (!clip_polygon_to_plane(*out, *in, cp, edgeId))
		{
			ok = false;
			return out;
		}
		Poly* t = in;
		in = out;
		out = t;
		if (in->n == 0)
			return in;
		edge = he_next(h, edge);
	} while (edge != begin);
	return in;
}

// ---------------------------------------------------------------------------
// Polygon reduction (cluster.cpp:24-200).

struct CV
{
	V3 pos;
	uint32_t clipIndex;
};

__device__ __forceinline__ bool is_ccw(V3 A, V3 B, V3 C, V3 N)
{
	V3 n = cross(B - A, C - A);
	return dot(n, N) > 0.0f;
}

// b3SortPolygon (cluster.cpp:34-57). B is read once per i, before the swaps.
__device__ __forceinline__ void sort_polygon(CV* p, uint32_t n, V3 N)
{
	V3 A = p[0].pos;
	for (uint32_t i = 1; i < n; ++i)
	{
		V3 B = p[i].pos;
		for (uint32_t j = i + 1; j < n; ++j)
		{
			V3 C = p[j].pos;
			if (!is_ccw(A, B, C, N))
			{
				CV t = p[i];
				p[i] = p[j];
				p[j] = t;
			}
		}
	}
}

// b3ReducePolygon (cluster.cpp:59-200). out holds at most 4 vertices, so the
// reference's per-vertex chosen flags are kept as a list of at most 4
// indices.
__device__ __forceinline__ uint32_t reduce_polygon(CV out[4], const CV* in, uint32_t n, V3 N, uint32_t initialPoint)
{
	if (n <= 4)
	{
		for (uint32_t i = 0; i < n; ++i)
			out[i] = in[i];
		sort_polygon(out, n, N);
		return n;
	}
	uint32_t chosen[4];
	uint32_t nChosen = 0;
	auto isChosen = [&](uint32_t i) {
		bool r = false;
		for (uint32_t k = 0; k < nChosen; ++k)
			r |= chosen[k] == i;
		return r;
	};
	auto choose = [&](uint32_t i) { chosen[nChosen++] = i; };
	uint32_t cnt = 0;
	out[cnt++] = in[initialPoint];
	choose(initialPoint);
	{
		V3 A = out[0].pos;
		uint32_t index = 0;
		float mx = -B3G_MAX_SCALAR;
		for (uint32_t i = 0; i < n; ++i)
		{
			if (isChosen(i))
				continue;
			V3 d = in[i].pos - A;
			float dd = dot(d, d);
			if (dd > mx)
			{
				mx = dd;
				index = i;
			}
		}
		if (mx < B3G_EPSILON * B3G_EPSILON)
			return cnt;
		out[cnt++] = in[index];
		choose(index);
	}
	{
		V3 A = out[0].pos;
		V3 B = out[1].pos;
		uint32_t index = 0;
		float mx = -B3G_MAX_SCALAR;
		for (uint32_t i = 0; i < n; ++i)
		{
			if (isChosen(i))
				continue;
			V3 C = in[i].pos;
			V3 Nn = cross(B - A, C - A);
			float sa2 = dot(Nn, N);
			float a2 = fabsr(sa2);
			if (a2 > mx)
			{
				mx = a2;
				index = i;
			}
		}
		const float kAreaTol = 0.01f;
		if (mx < 2.0f * kAreaTol)
			return cnt;
		V3 C = in[index].pos;
		if (!is_ccw(A, B, C, N))
		{
			CV t = out[0];
			out[0] = out[1];
			out[1] = t;
		}
		out[cnt++] = in[index];
		choose(index);
	}
	{
		V3 A = out[0].pos;
		V3 B = out[1].pos;
		uint32_t index = 0;
		float mn = B3G_MAX_SCALAR;
		for (uint32_t i = 0; i < n; ++i)
		{
			if (isChosen(i))
				continue;
			V3 D = in[i].pos;
			V3 Nn = cross(B - A, D - A);
			float sa2 = dot(Nn, N);
			if (sa2 < mn)
			{
				mn = sa2;
				index = i;
			}
		}
		const float kAreaTol = 0.01f;
		if (fabsr(mn) < 2.0f * kAreaTol)
			return cnt;
		out[cnt++] = in[index];
		choose(index);
	}
	sort_polygon(out, cnt, N);
	return cnt;
}

// ---------------------------------------------------------------------------
// Manifolds.

// b3Manifold::Initialize() (collision.cpp:23-38): the 32-byte header
// (pointCount, impulses, speeds) is zeroed with two 16-byte stores; every
// point a collide routine produces is written whole by set_point. As in the
// reference, which reuses the manifold memory of a contact from step to step,
// points at or beyond pointCount keep unspecified older contents.
__device__ __forceinline__ void man_clear(DevManifold& m)
{
	uint4* w = reinterpret_cast<uint4*>(&m.pointCount);
	w[0] = make_uint4(0u, 0u, 0u, 0u);
	w[1] = make_uint4(0u, 0u, 0u, 0u);
}

// Writes a produced point: geometry here, the id by set_id / set_id0;
// normalImpulse, persisting and edgeContact start cleared (Initialize()).
__device__ __forceinline__ void set_point(DevPoint& p, V3 n, V3 p1, V3 p2)
{
	p.normalImpulse = 0.0f;
	p.pad0 = 0;
	p.persisting = 0;
	p.edgeContact = 0;
	for (int k = 0; k < 6; ++k)
		p.pad1[k] = 0;
	p.n[0] = n.x;
	p.n[1] = n.y;
	p.n[2] = n.z;
	p.p1[0] = p1.x;
	p.p1[1] = p1.y;
	p.p1[2] = p1.z;
	p.p2[0] = p2.x;
	p.p2[1] = p2.y;
	p.p2[2] = p2.z;
}

// b3MakeID(key1, key2) with key1 = key2 = 0, and b3MakeID(pair) (collision.h:80-95).
__device__ __forceinline__ void set_id0(DevPoint& p)
{
	p.triangleKey = B3G_NULL_TRIANGLE;
	p.key[0] = p.key[1] = p.key[2] = p.key[3] = 0;
}
__device__ __forceinline__ void set_id(DevPoint& p, FPair f)
{
	p.triangleKey = B3G_NULL_TRIANGLE;
	p.key[0] = f.inEdge1;
	p.key[1] = f.outEdge1;
	p.key[2] = f.inEdge2;
	p.key[3] = f.outEdge2;
}

__device__ __forceinline__ bool id_equal(const DevPoint& a, const DevPoint& b)
{
	return a.triangleKey == b.triangleKey && a.key[0] == b.key[0] && a.key[1] == b.key[1] &&
		a.key[2] == b.key[2] && a.key[3] == b.key[3];
}

// Per-pass context passed to the narrowphase kernels.
struct NPArgs
{
	DevScene S;
	uint32_t* pairA;
	uint32_t* pairB;
	uint32_t* cstate;
	uint4* cache;
	DevManifold* man;
	const uint32_t* prevState;
	const uint4* prevCache;
	const DevManifold* prevMan;
	const int32_t* prevIndex;
	const uint32_t* list;
	const uint32_t* listCount;
	uint32_t* status;
	int warmStarting;
	int convexCache;
	// warm-start overrides from the host solver (indexed by previous contact)
	const float* impN;
	const float* impT;
	const float* impM;
	// explicit transforms per contact (7 floats), used instead of the body
	// state when set (stand-alone narrowphase)
	const float* exA;
	const float* exB;
	const float* ex0A;
	const float* ex0B;
	// hull-hull pairs the feature cache could not resolve
	uint32_t* missList;
	uint32_t* missCount;
	// manifolds 1 and 2 of mesh contacts (null without meshes)
	DevManifold* extraCur;
	const DevManifold* extraPrev;
	// hull-capsule contacts whose GJK distance is within the radii: two
	// float4 per entry (point1, distance; point2, contact index); those with a
	// positive distance fill the entries from the front, the overlapping ones
	// from the back (hcPostCap entries), counted in hcPostCount[0] and [1]
	float4* hcPost;
	uint32_t* hcPostCount;
	uint32_t hcPostCap;
	// hull-sphere contacts whose face scan leaves the GJK to run, and their count
	uint32_t* hsPost;
	uint32_t* hsPostCount;
};

// ---------------------------------------------------------------------------
// Pair hash tables (one per pass): open addressing, fixture pair -> contact.

constexpr unsigned long long B3G_EMPTY_KEY = 0xFFFFFFFFFFFFFFFFull;

__device__ __forceinline__ unsigned long long pair_key(uint32_t a, uint32_t b)
{
	return ((unsigned long long)a << 32) | b;
}

__device__ __forceinline__ uint32_t pair_hash(unsigned long long k)
{
	k ^= k >> 33;
	k *= 0xff51afd7ed558ccdull;
	k ^= k >> 33;
	k *= 0xc4ceb9fe1a85ec53ull;
	k ^= k >> 33;
	return (uint32_t)k;
}

// Contact index of `key`, or -1.
__device__ __forceinline__ int32_t pair_hash_find(const unsigned long long* keys, const uint32_t* vals,
	uint32_t capPow2, unsigned long long key)
{
	uint32_t mask = capPow2 - 1u;
	uint32_t h = pair_hash(key) & mask;
	for (uint32_t probe = 0; probe <= mask; ++probe)
	{
		unsigned long long k = keys[h];
		if (k == key)
			return (int32_t)vals[h];
		if (k == B3G_EMPTY_KEY)
			return -1;
		h = (h + 1) & mask;
	}
	return -1;
}

// False when the table is full.
__device__ __forceinline__ bool pair_hash_insert(unsigned long long* keys, uint32_t* vals, uint32_t capPow2,
	unsigned long long key, uint32_t value)
{
	uint32_t mask = capPow2 - 1u;
	uint32_t h = pair_hash(key) & mask;
	for (uint32_t probe = 0; probe <= mask; ++probe)
	{
		unsigned long long old = atomicCAS(&keys[h], B3G_EMPTY_KEY, key);
		if (old == B3G_EMPTY_KEY || old == key)
		{
			vals[h] = value;
			return true;
		}
		h = (h + 1) & mask;
	}
	return false;
}

// Shape-type pair -> narrowphase bucket (A carries the primary type;
// contact.cpp:60-68).
__device__ __forceinline__ uint32_t bucket_of(uint32_t ta, uint32_t tb)
{
	if (ta == B3G_SHAPE_SPHERE)
		return BK_SPHERES;
	if (ta == B3G_SHAPE_CAPSULE)
		return tb == B3G_SHAPE_SPHERE ? BK_CAPSULE_SPHERE : BK_CAPSULES;
	if (ta == B3G_SHAPE_TRIANGLE)
		return tb == B3G_SHAPE_SPHERE ? BK_TRIANGLE_SPHERE : BK_TRIANGLE_CAPSULE;
	if (ta == B3G_SHAPE_HULL)
	{
		if (tb == B3G_SHAPE_SPHERE)
			return BK_HULL_SPHERE;
		if (tb == B3G_SHAPE_CAPSULE)
			return BK_HULL_CAPSULE;
		if (tb == B3G_SHAPE_TRIANGLE)
			return BK_HULL_TRIANGLE;
		return BK_HULLS;
	}
	return BK_COUNT; // mesh pairs: not handled by these buckets
}

// ---------------------------------------------------------------------------
// Shape AABBs.

__device__ __forceinline__ XF load_xf(const float* s)
{
	XF x;
	x.p = V3{s[0], s[1], s[2]};
	x.q = Q4{V3{s[3], s[4], s[5]}, s[6]};
	return x;
}

// b3Shape::ComputeAABB for one transform (hull_shape.cpp:160-164,
// sphere_shape.cpp:51-57, capsule_shape.cpp:124-131, triangle_shape.cpp:59-67)
// of a shape given by its type, parameters (the fixture layout) and hull.
// Two transforms are handled in one vertex loop for hulls.
__device__ inline void compute_shape_aabbs(const DevScene& S, uint32_t type, float4 p0, float4 p1, float4 p2,
	uint32_t hull, const XF& xa, const XF& xb, bool two, AABB& a, AABB& b)
{
	if (type == B3G_SHAPE_SPHERE)
	{
		V3 c = V3{p0.x, p0.y, p0.z};
		float r = p0.w;
		V3 rv = V3{r, r, r};
		V3 ca = xmul(xa, c);
		a.lo = ca - rv;
		a.hi = ca + rv;
		if (two)
		{
			V3 cb = xmul(xb, c);
			b.lo = cb - rv;
			b.hi = cb + rv;
		}
	}
	else if (type == B3G_SHAPE_CAPSULE)
	{
		V3 v1 = V3{p0.x, p0.y, p0.z};
		V3 v2 = V3{p0.w, p1.x, p1.y};
		float r = p1.z;
		V3 rv = V3{r, r, r};
		V3 c1 = xmul(xa, v1), c2 = xmul(xa, v2);
		a.lo = vmin(c1, c2) - rv;
		a.hi = vmax(c1, c2) + rv;
		if (two)
		{
			c1 = xmul(xb, v1);
			c2 = xmul(xb, v2);
			b.lo = vmin(c1, c2) - rv;
			b.hi = vmax(c1, c2) + rv;
		}
	}
	else if (type == B3G_SHAPE_TRIANGLE)
	{
		// The reference ignores the transform here (triangle_shape.cpp:59-67).
		V3 v1 = V3{p0.x, p0.y, p0.z};
		V3 v2 = V3{p0.w, p1.x, p1.y};
		V3 v3_ = V3{p1.z, p1.w, p2.x};
		float r = p2.y;
		V3 rv = V3{r, r, r};
		a.lo = vmin(v1, vmin(v2, v3_)) - rv;
		a.hi = vmax(v1, vmax(v2, v3_)) + rv;
		b = a;
	}
	else // hull
	{
		const HullDesc h = S.hulls[hull];
		const float4* hv = S.hverts + h.vOff;
		float4 w = hv[0];
		V3 v = V3{w.x, w.y, w.z};
		V3 ta = xmul(xa, v);
		a.lo = ta;
		a.hi = ta;
		V3 tb;
		if (two)
		{
			tb = xmul(xb, v);
			b.lo = tb;
			b.hi = tb;
		}
		for (uint32_t i = 1; i < h.vCnt; ++i)
		{
			w = hv[i];
			v = V3{w.x, w.y, w.z};
			ta = xmul(xa, v);
			a.lo = vmin(a.lo, ta);
			a.hi = vmax(a.hi, ta);
			if (two)
			{
				tb = xmul(xb, v);
				b.lo = vmin(b.lo, tb);
				b.hi = vmax(b.hi, tb);
			}
		}
		float r = p0.x;
		aabb_extend(a, r);
		if (two)
			aabb_extend(b, r);
	}
}

// b3AABB::Scale (aabb.h:287-294).
__device__ __forceinline__ AABB aabb_scaled(const AABB& a, V3 s)
{
	V3 l = vmul(s, a.lo), u = vmul(s, a.hi);
	AABB r;
	r.lo = vmin(l, u);
	r.hi = vmax(l, u);
	return r;
}

// b3GJKProxy::Set (gjk.cpp:37-95) for a convex shape given by type,
// parameters (the fixture layout) and hull.
__device__ inline GProxy convex_proxy(const DevScene& S, uint32_t type, float4 p0, float4 p1, float4 p2, uint32_t hull)
{
	GProxy g;
	g.gv = nullptr;
	g.lv[0] = g.lv[1] = g.lv[2] = V3{0.0f, 0.0f, 0.0f};
	switch (type)
	{
	case B3G_SHAPE_SPHERE:
		g.lv[0] = V3{p0.x, p0.y, p0.z};
		g.count = 1;
		g.radius = p0.w;
		break;
	case B3G_SHAPE_CAPSULE:
		g.lv[0] = V3{p0.x, p0.y, p0.z};
		g.lv[1] = V3{p0.w, p1.x, p1.y};
		g.count = 2;
		g.radius = p1.z;
		break;
	case B3G_SHAPE_TRIANGLE:
		g.lv[0] = V3{p0.x, p0.y, p0.z};
		g.lv[1] = V3{p0.w, p1.x, p1.y};
		g.lv[2] = V3{p1.z, p1.w, p2.x};
		g.count = 3;
		g.radius = p2.y;
		break;
	default:
	{
		const HullDesc h = S.hulls[hull];
		g.gv = S.hverts + h.vOff;
		g.count = h.vCnt;
		g.radius = p0.x;
		break;
	}
	}
	return g;
}

// The same for fixture fix.
__device__ inline void compute_aabbs(const DevScene& S, uint32_t fix, const XF& xa, const XF& xb, bool two, AABB& a,
	AABB& b)
{
	compute_shape_aabbs(S, S.fixType[fix], S.fixParams[3 * fix + 0], S.fixParams[3 * fix + 1],
		S.fixParams[3 * fix + 2], S.fixHull[fix], xa, xb, two, a, b);
}

// Exact cull, not in the reference: every convex routine (sphere, capsule,
// triangle-sphere/capsule, hull-sphere/capsule) returns no point when the
// shapes are farther apart than their radii sum (the sphere
// and capsule routines compare closest-point distances with the radii; the
// hull routines' face loop or GJK, whose witness points lie on the shapes,
// then report a distance above the radii). Bounding spheres (fixture-local
// centre, conservative radius from b3g_set_fixtures) separated by more than
// the radii plus a margin that dominates the FP32 rounding of those
// distances (1e-3 m + 1e-5 of the coordinate magnitude) therefore mean an
// empty manifold, and the routine can be skipped without changing the output.
__device__ __forceinline__ bool spheres_apart(const DevScene& S, uint32_t fa, const XF& xfA, uint32_t fb,
	const XF& xfB)
{
	float4 ba = S.fixBound[fa], bb = S.fixBound[fb];
	V3 ca = xmul(xfA, V3{ba.x, ba.y, ba.z});
	V3 cb = xmul(xfB, V3{bb.x, bb.y, bb.z});
	V3 d = cb - ca;
	float mag = fmaxf(fmaxf(fmaxf(fabsf(ca.x), fabsf(ca.y)), fabsf(ca.z)),
		fmaxf(fmaxf(fabsf(cb.x), fabsf(cb.y)), fabsf(cb.z)));
	float reach = (ba.w + bb.w) + (1e-3f + 1e-5f * mag);
	return dot(d, d) > reach * reach;
}

// The same cull for a hull (bounding sphere) against a capsule's segment:
// the hull lies inside its bounding sphere, so its distance to the segment is
// at least the centre's distance minus the sphere radius; farther than the
// capsule radius plus the margin means b3CollideHullAndCapsule's GJK reports
// a distance above the radii and the manifold is empty.
__device__ __forceinline__ bool hull_capsule_apart(const DevScene& S, uint32_t fh, const XF& xfH, uint32_t fc,
	const XF& xfC)
{
	float4 bh = S.fixBound[fh];
	float4 p0 = S.fixParams[3 * fc], p1 = S.fixParams[3 * fc + 1];
	V3 c = xmul(xfH, V3{bh.x, bh.y, bh.z});
	V3 a = xmul(xfC, V3{p0.x, p0.y, p0.z});
	V3 b = xmul(xfC, V3{p0.w, p1.x, p1.y});
	V3 d = b - a;
	float dd = dot(d, d);
	float t = dd > 0.0f ? dot(c - a, d) / dd : 0.0f;
	t = fminf(fmaxf(t, 0.0f), 1.0f);
	V3 e = c - (a + t * d);
	float mag = fmaxf(fmaxf(fmaxf(fabsf(c.x), fabsf(c.y)), fabsf(c.z)),
		fmaxf(fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fabsf(a.z)), fmaxf(fmaxf(fabsf(b.x), fabsf(b.y)), fabsf(b.z))));
	float reach = (bh.w + p1.z) + (1e-3f + 1e-5f * mag);
	return dot(e, e) > reach * reach;
}

// ---------------------------------------------------------------------------
// Meshes.

// b3StaticTree::QueryAABB (static_tree.h:114-150): depth-first from the root
// with a LIFO stack (child1 pushed, then child2, so child2 is searched
// first), reporting each overlapping leaf's triangle in that order. False if
// the stack overflowed (the query stops).
template <class F>
__device__ inline bool mesh_query(const DevScene& S, const MeshDesc& md, const AABB& box, F&& report)
{
	constexpr uint32_t STACK = 64;
	uint32_t stack[STACK];
	uint32_t sp = 0;
	stack[sp++] = md.root;
	while (sp > 0)
	{
		uint32_t id = stack[--sp];
		if (id == B3G_NULL_NODE)
			continue;
		float4 lo = S.meshNodes[2 * (size_t)(md.nOff + id)], hi = S.meshNodes[2 * (size_t)(md.nOff + id) + 1];
		bool overlap = !(hi.x < box.lo.x || lo.x > box.hi.x || hi.y < box.lo.y || lo.y > box.hi.y ||
			hi.z < box.lo.z || lo.z > box.hi.z);
		if (!overlap)
			continue;
		uint32_t child1 = __float_as_uint(lo.w), other = __float_as_uint(hi.w);
		if (child1 == B3G_NULL_NODE)
			report(other);
		else
		{
			if (sp + 2 > STACK)
				return false;
			stack[sp++] = child1;
			stack[sp++] = other;
		}
	}
	return true;
}

// b3MeshShape::GetChildTriangle (mesh_shape.cpp:151-183): the scaled
// vertices, the mesh radius and the wings of the triangle's edges, with its
// b3TriangleHull (triangle_hull.h:36-69).
struct MeshTri
{
	V3 v[3];
	float4 wing[3]; // wing vertex, w = 1 when the edge has one
	float radius;
	float4 hv[3];   // hull vertices
	float4 hp[2];   // hull planes
	V3 centroid;
};

__device__ inline void mesh_triangle(const DevScene& S, uint32_t meshFix, uint32_t t, MeshTri& out)
{
	const MeshDesc md = S.meshes[S.fixHull[meshFix]];
	float4 sp = S.fixParams[3 * meshFix];
	V3 sc = V3{sp.x, sp.y, sp.z};
	uint4 tri = S.meshTris[md.tOff + t];
	uint4 w = S.meshWings[md.tOff + t];
	auto vert = [&](uint32_t i) {
		float4 a = S.meshVerts[md.vOff + i];
		return vmul(sc, V3{a.x, a.y, a.z});
	};
	out.v[0] = vert(tri.x);
	out.v[1] = vert(tri.y);
	out.v[2] = vert(tri.z);
	uint32_t wi[3] = {w.x, w.y, w.z};
	for (int k = 0; k < 3; ++k)
	{
		if (wi[k] != B3G_NULL)
		{
			V3 e = vert(wi[k]);
			out.wing[k] = make_float4(e.x, e.y, e.z, 1.0f);
		}
		else
			out.wing[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	}
	out.radius = sp.w;
	V3 A = out.v[0], B = out.v[1], C = out.v[2];
	V3 cen = ((A + B) + C) / 3.0f;
	V3 N = normalized(cross(B - A, C - A));
	V3 M = -N;
	out.hv[0] = make_float4(A.x, A.y, A.z, 0.0f);
	out.hv[1] = make_float4(B.x, B.y, B.z, 0.0f);
	out.hv[2] = make_float4(C.x, C.y, C.z, 0.0f);
	out.hp[0] = make_float4(N.x, N.y, N.z, dot(N, cen));
	out.hp[1] = make_float4(M.x, M.y, M.z, dot(M, cen));
	out.centroid = cen;
}

__device__ __forceinline__ HullRef mesh_tri_ref(const MeshTri& t)
{
	HullRef r;
	r.v = t.hv;
	r.e = kTriEdges;
	r.f = kTriFaces;
	r.p = t.hp;
	r.vCnt = 3;
	r.eCnt = 6;
	r.fCnt = 2;
	r.centroid = t.centroid;
	return r;
}

void scan_exclusive_device(uint32_t* data, const uint32_t* nPtr, uint32_t cap, uint32_t* aux, uint32_t* total,
	uint32_t* err, cudaStream_t s);
void launch_apart(const NPArgs& a, const uint32_t* list, const uint32_t* count, cudaStream_t s);
void launch_mesh_items_convex(const NPArgs& a, const Buffers& B, cudaStream_t s);
void launch_mesh_items_hull(const NPArgs& a, const Buffers& B, uint32_t maxUE, const Tune& tune, cudaStream_t s);

// Narrowphase arguments of the current pass (contact arrays of c->cur).
NPArgs make_np_args(b3g_ctx* c);
void launch_convex_buckets(const NPArgs& base, const uint32_t* lists, const uint32_t* counts, uint32_t cap,
	const Tune& tune, cudaStream_t s);
void launch_convex_one(int k, const NPArgs& base, const uint32_t* lists, const uint32_t* counts, uint32_t cap,
	const Tune& tune, cudaStream_t s);
// Whether convex bucket kernel k (the order of B3G_TUNE_CONVEX) can have
// contacts in this context's pass: the triangle buckets need triangle
// fixtures, the sensor bucket sensors, the inactive bucket a sleeping body.
bool convex_bucket_possible(const b3g_ctx* c, int k);
void launch_hulls(const NPArgs& base, const uint32_t* list, const uint32_t* count, uint32_t maxUE, const Tune& tune,
	cudaStream_t s);
void launch_hulls_probe(const NPArgs& base, const uint32_t* list, const uint32_t* count, const Tune& tune,
	cudaStream_t s);
void launch_hulls_sat(const NPArgs& a, uint32_t maxUE, const Tune& tune, cudaStream_t s);
void launch_hull_triangles(const NPArgs& base, const uint32_t* list, const uint32_t* count, uint32_t maxUE,
	const Tune& tune, cudaStream_t s);
void scan_exclusive(uint32_t* data, uint32_t n, uint32_t* aux, uint32_t* total, uint32_t* err, cudaStream_t s);
uint32_t scan_aux_words(uint32_t n);
uint32_t radix_sort_scratch_words(uint32_t n, int bits);
bool radix_sort_pairs(unsigned long long* keys, uint32_t* vals, unsigned long long* keysTmp, uint32_t* valsTmp,
	uint32_t n, int bits, uint32_t* scratch, uint32_t* err, cudaStream_t s);

__device__ __forceinline__ XF load_xf7(const float* s)
{
	XF x;
	x.p = V3{s[0], s[1], s[2]};
	x.q = Q4{V3{s[3], s[4], s[5]}, s[6]};
	return x;
}

// The tail of b3Contact::Update for a convex contact (contact.cpp:424-465):
// warm start from the previous manifold as b3Manifold::Initialize(old) does
// (collision.cpp:40-61: tangent and motor impulses copied, normal impulses
// copied to points whose b3ContactID matches), touching flag, manifold count 1.
// m is the contact's output record (device memory); the previous record is
// read field by field.
__device__ __forceinline__ void finish_convex(const NPArgs& a, uint32_t c, DevManifold& m)
{
	int32_t prev = a.prevIndex[c];
	uint32_t oldCount = prev >= 0 ? ((a.prevState[prev] >> 8) & 0xFFu) : 0u;
	uint32_t pc = m.pointCount;
	if (a.warmStarting && oldCount > 0)
	{
		const DevManifold& old = a.prevMan[prev];
		if (a.impN)
		{
			m.tangentImpulse[0] = a.impT[2 * prev + 0];
			m.tangentImpulse[1] = a.impT[2 * prev + 1];
			m.motorImpulse = a.impM[prev];
		}
		else
		{
			m.tangentImpulse[0] = old.tangentImpulse[0];
			m.tangentImpulse[1] = old.tangentImpulse[1];
			m.motorImpulse = old.motorImpulse;
		}
		uint32_t opc = old.pointCount;
		for (uint32_t i = 0; i < pc; ++i)
		{
			DevPoint& p1 = m.points[i];
			for (uint32_t j = 0; j < opc; ++j)
			{
				const DevPoint& p2 = old.points[j];
				if (p2.triangleKey == p1.triangleKey && p2.key[0] == p1.key[0] && p2.key[1] == p1.key[1] &&
					p2.key[2] == p1.key[2] && p2.key[3] == p1.key[3])
				{
					p1.normalImpulse = a.impN ? a.impN[4 * prev + j] : p2.normalImpulse;
					p1.persisting = 1;
					break;
				}
			}
		}
	}
	uint32_t touching = pc > 0 ? 1u : 0u;
	uint32_t begun = prev < 0 ? 1u : 0u;
	a.cstate[c] = touching | (1u << 8) | (begun << 16);
}

// Per-body transforms prepared once per pass by k_body_prep (two float4 each:
// translation + rotation.x, rotation.yzw).
__device__ __forceinline__ XF unpack_xf(const float4* t, uint32_t body)
{
	float4 a = t[2 * (size_t)body], b = t[2 * (size_t)body + 1];
	XF x;
	x.p = V3{a.x, a.y, a.z};
	x.q = Q4{V3{a.w, b.x, b.y}, b.z};
	return x;
}
__device__ __forceinline__ void pack_xf(float4* t, uint32_t body, const XF& x)
{
	t[2 * (size_t)body] = make_float4(x.p.x, x.p.y, x.p.z, x.q.v.x);
	t[2 * (size_t)body + 1] = make_float4(x.q.v.y, x.q.v.z, x.q.s, 0.0f);
}

// b3Body::m_xf.
__device__ __forceinline__ XF body_xf(const DevScene& S, uint32_t body) { return unpack_xf(S.bodyXf, body); }

// b3Sweep::GetTransform(0), as b3HullContact::Evaluate uses it (hull_contact.cpp:43-44).
__device__ __forceinline__ XF body_xf0(const DevScene& S, uint32_t body) { return unpack_xf(S.bodyXf0, body); }

// b3Sweep::GetTransform(0) (sweep.h:43-63) from the stored sweep start.
__device__ __forceinline__ XF sweep_xf0(const DevScene& S, uint32_t body)
{
	const float* s = S.bodyState + 17 * (size_t)body;
	Q4 q1 = Q4{V3{s[10], s[11], s[12]}, s[13]};
	Q4 q2 = Q4{V3{s[3], s[4], s[5]}, s[6]};
	V3 c0 = V3{s[7], s[8], s[9]};
	V3 lc = V3{s[14], s[15], s[16]};
	if (qdot(q1, q2) < 0.0f)
		q1 = qneg(q1);
	// (1 - 0) * c0 + 0 * c and (1 - 0) * q1 + 0 * q2 reduce to c0 and q1.
	Q4 q = q1;
	qnormalize_inplace(q);
	XF x;
	x.p = c0 - rot(q, lc);
	x.q = q;
	return x;
}

// World queries on the device: b3World::QueryAABB, RayCast, RayCastSingle,
// ShapeCast and ShapeCastSingle (world.cpp:452-878) over the LBVH and fat
// AABBs of the last pass, with each shape's own ray cast:
//   b3SphereShape::RayCast    sphere_shape.cpp:69-122
//   b3CapsuleShape::RayCast   capsule_shape.cpp:180-322
//   b3HullShape::RayCast      hull_shape.cpp:189-275
//   b3TriangleShape::RayCast  triangle_shape.cpp:95-180
//   b3MeshShape::RayCast      mesh_shape.cpp:81-146, over b3StaticTree::RayCast
//                             (static_tree.h:150-292)
//
// One thread per query walks the LBVH from the root along its ropes. The
// reference walks its dynamic tree instead; the set of proxies a query meets
// is the same (fat AABBs overlapping the box, or the segment), only the order
// differs: QueryAABB and RayCast (every hit) are returned per query in LBVH
// order, and RayCastSingle keeps the smallest fraction, the smaller fixture
// index on an exact tie (the reference keeps the first one its tree meets).

#include <vector>

#include "collide_common.cuh"

namespace {

constexpr uint32_t SENT = 0xFFFFFFFFu;

struct RayIn
{
	V3 p1, p2;
	float maxFraction;
};

struct RayOut
{
	float fraction;
	V3 normal;
};

__device__ __forceinline__ V3 vabs(V3 v) { return V3{fabsf(v.x), fabsf(v.y), fabsf(v.z)}; }

// The segment tests of b3DynamicTree::RayCast / b3StaticTree::RayCast
// (static_tree.h:185-262): the segment's AABB overlaps the node's, and no
// axis of the box or of cross(e_i, r) separates them.
struct SegTest
{
	V3 p1, q2, r;
	AABB box;

	__device__ void init(V3 a, V3 b, float maxFraction)
	{
		p1 = a;
		r = b - a;
		normalize_inplace(r);
		q2 = a + maxFraction * (b - a);
		box.lo = vmin(a, q2);
		box.hi = vmax(a, q2);
	}

	// Shortens the segment to [p1, p1 + f (b - p1)].
	__device__ void clip(V3 b, float f)
	{
		q2 = p1 + f * (b - p1);
		box.lo = vmin(p1, q2);
		box.hi = vmax(p1, q2);
	}

	__device__ bool pass(V3 lo, V3 hi) const
	{
		if (box.hi.x < lo.x || box.lo.x > hi.x || box.hi.y < lo.y || box.lo.y > hi.y || box.hi.z < lo.z ||
			box.lo.z > hi.z)
			return false;
		V3 c = 0.5f * (lo + hi);
		V3 h = 0.5f * (hi - lo);
		V3 s = p1 - c;
		V3 t = q2 - c;
		if (fabsf(s.x + t.x) - (fabsf(s.x - t.x) + 2.0f * h.x) > 0.0f)
			return false;
		if (fabsf(s.y + t.y) - (fabsf(s.y - t.y) + 2.0f * h.y) > 0.0f)
			return false;
		if (fabsf(s.z + t.z) - (fabsf(s.z - t.z) + 2.0f * h.z) > 0.0f)
			return false;
		V3 v1 = cross(V3{1.0f, 0.0f, 0.0f}, r);
		if (fabsf(dot(v1, s)) - dot(vabs(v1), h) > 0.0f)
			return false;
		V3 v2 = cross(V3{0.0f, 1.0f, 0.0f}, r);
		if (fabsf(dot(v2, s)) - dot(vabs(v2), h) > 0.0f)
			return false;
		V3 v3 = cross(V3{0.0f, 0.0f, 1.0f}, r);
		if (fabsf(dot(v3, s)) - dot(vabs(v3), h) > 0.0f)
			return false;
		return true;
	}
};

// Ray against a sphere of radius `radius` around m = p1 - centre.
__device__ __forceinline__ bool ray_sphere_at(RayOut& o, V3 m, V3 d, float a, float radius, float maxFraction)
{
	float b = dot(m, d);
	float c = dot(m, m) - radius * radius;
	float disc = b * b - a * c;
	if (disc < 0.0f)
		return false;
	float t = -b - sqrtf(disc);
	if (t > 0.0f && t <= maxFraction * a)
	{
		t /= a;
		o.fraction = t;
		o.normal = normalized(m + t * d);
		return true;
	}
	return false;
}

__device__ bool ray_sphere(RayOut& o, const RayIn& in, const XF& xf, V3 center, float radius)
{
	V3 d = in.p2 - in.p1;
	float a = dot(d, d);
	if (a < B3G_EPSILON * B3G_EPSILON)
		return false;
	V3 m = in.p1 - xmul(xf, center);
	return ray_sphere_at(o, m, d, a, radius, in.maxFraction);
}

__device__ bool ray_capsule(RayOut& o, const RayIn& in, const XF& xf, V3 v1, V3 v2, float radius)
{
	V3 A = in.p1, B = in.p2;
	V3 n = B - A;
	float nn = dot(n, n);
	if (nn < B3G_EPSILON * B3G_EPSILON)
		return false;
	V3 P = xmul(xf, v1), Q = xmul(xf, v2);
	V3 d = Q - P;
	float dd = dot(d, d);
	if (dd < B3G_EPSILON * B3G_EPSILON)
		return ray_sphere_at(o, A - P, n, nn, radius, in.maxFraction);
	V3 m = A - P;
	float nd = dot(n, d);
	float mm = dot(m, m);
	float md = dot(m, d);
	float mn = dot(m, n);
	float a = dd * nn - nd * nd;
	if (fabsf(a) < 2.0f * (B3G_EPSILON * B3G_EPSILON))
		return false;
	float b = dd * mn - nd * md;
	float c = dd * (mm - radius * radius) - md * md;
	float disc = b * b - a * c;
	if (disc < 0.0f)
		return false;
	float t = -b - sqrtf(disc);
	t /= a;
	if (t < 0.0f || t > 1.0f)
		return false;
	// Which part of the capsule the cylinder hit lies on.
	float tp = md + t * nd;
	V3 C;
	if (tp < 0.0f)
		C = P;
	else if (tp > dd)
		C = Q;
	else
	{
		V3 X = (1.0f - t) * A + t * B;
		V3 e2 = cross(d, X - P);
		V3 e3 = cross(e2, d);
		normalize_inplace(e3);
		o.fraction = t;
		o.normal = e3;
		return true;
	}
	// Hemisphere at C.
	return ray_sphere_at(o, A - C, n, nn, radius, in.maxFraction);
}

__device__ bool ray_hull(RayOut& o, const RayIn& in, const XF& xf, const HullRef& h)
{
	V3 p1 = rotc(xf.q, in.p1 - xf.p);
	V3 p2 = rotc(xf.q, in.p2 - xf.p);
	V3 d = p2 - p1;
	float lower = 0.0f, upper = in.maxFraction;
	uint32_t index = B3G_NULL;
	for (uint32_t i = 0; i < h.fCnt; ++i)
	{
		PL pl = hp(h, i);
		float numerator = pl.d - dot(pl.n, p1);
		float denominator = dot(pl.n, d);
		if (denominator == 0.0f)
		{
			if (numerator < 0.0f)
				return false;
		}
		else
		{
			if (denominator < 0.0f)
			{
				if (numerator < lower * denominator)
				{
					lower = numerator / denominator;
					index = i;
				}
			}
			else if (numerator < upper * denominator)
				upper = numerator / denominator;
			if (upper < lower)
				return false;
		}
	}
	if (index != B3G_NULL)
	{
		o.fraction = lower;
		o.normal = rot(xf.q, hp(h, index).n);
		return true;
	}
	return false;
}

__device__ bool ray_triangle(RayOut& o, const RayIn& in, const XF& xf, V3 v1, V3 v2, V3 v3)
{
	V3 p1 = xmult(xf, in.p1);
	V3 p2 = xmult(xf, in.p2);
	V3 d = p2 - p1;
	if (dot(d, d) < B3G_EPSILON * B3G_EPSILON)
		return false;
	V3 n = cross(v2 - v1, v3 - v1);
	float l = len(n);
	if (l == 0.0f)
		return false;
	float inv = 1.0f / l; // b3Vec3::operator/= scales by the reciprocal
	n = inv * n;
	float num = dot(n, v1 - p1);
	float den = dot(n, d);
	if (den == 0.0f)
		return false;
	float fraction = num / den;
	if (fraction < 0.0f || in.maxFraction < fraction)
		return false;
	V3 Q = p1 + fraction * d;
	V3 AB = v2 - v1, AC = v3 - v1;
	V3 QA = v1 - Q, QB = v2 - Q, QC = v3 - Q;
	V3 QB_x_QC = cross(QB, QC);
	V3 QC_x_QA = cross(QC, QA);
	V3 QA_x_QB = cross(QA, QB);
	V3 AB_x_AC = cross(AB, AC);
	float u = dot(QB_x_QC, AB_x_AC);
	float v = dot(QC_x_QA, AB_x_AC);
	float w = dot(QA_x_QB, AB_x_AC);
	if (u >= 0.0f && v >= 0.0f && w >= 0.0f)
	{
		o.fraction = fraction;
		o.normal = num > 0.0f ? rot(xf.q, -n) : rot(xf.q, n);
		return true;
	}
	return false;
}

// b3MeshShape::RayCast: the segment in the mesh's unscaled frame walks the
// static tree (depth first, child2 first, as b3StaticTree::RayCast's stack);
// each leaf's triangle (scaled) is ray cast with the original segment; the
// first smallest fraction wins.
__device__ bool ray_mesh(RayOut& o, const RayIn& in, const XF& xf, const DevScene& S, uint32_t fix, uint32_t* status)
{
	const MeshDesc md = S.meshes[S.fixHull[fix]];
	float4 sp = S.fixParams[3 * fix];
	V3 sc = V3{sp.x, sp.y, sp.z};
	V3 inv = V3{1.0f / sc.x, 1.0f / sc.y, 1.0f / sc.z};
	SegTest seg;
	seg.init(vmul(inv, xmult(xf, in.p1)), vmul(inv, xmult(xf, in.p2)), in.maxFraction);
	bool hit = false;
	o.fraction = B3G_MAX_SCALAR;
	constexpr uint32_t STACK = 64;
	uint32_t stack[STACK];
	uint32_t sp_ = 0;
	stack[sp_++] = md.root;
	while (sp_ > 0)
	{
		uint32_t id = stack[--sp_];
		if (id == B3G_NULL_NODE)
			continue;
		float4 lo = S.meshNodes[2 * (size_t)(md.nOff + id)], hi = S.meshNodes[2 * (size_t)(md.nOff + id) + 1];
		if (!seg.pass(V3{lo.x, lo.y, lo.z}, V3{hi.x, hi.y, hi.z}))
			continue;
		uint32_t child1 = __float_as_uint(lo.w), other = __float_as_uint(hi.w);
		if (child1 == B3G_NULL_NODE)
		{
			uint4 t = S.meshTris[md.tOff + other];
			auto vert = [&](uint32_t i) {
				float4 a = S.meshVerts[md.vOff + i];
				return vmul(sc, V3{a.x, a.y, a.z});
			};
			RayOut r;
			if (ray_triangle(r, in, xf, vert(t.x), vert(t.y), vert(t.z)) && r.fraction < o.fraction)
			{
				hit = true;
				o = r;
				// Triangle boxes are grown by B3_LINEAR_SLOP: a triangle hit no
				// later than this one is met by the shortened segment too.
				seg.clip(vmul(inv, xmult(xf, in.p2)), r.fraction);
			}
		}
		else
		{
			if (sp_ + 2 > STACK)
			{
				atomicOr(status, B3G_ST_POLY_OVERFLOW);
				return hit;
			}
			stack[sp_++] = child1;
			stack[sp_++] = other;
		}
	}
	return hit;
}

// b3Fixture::RayCast (fixture.h) at the body's transform of the last pass.
__device__ bool ray_fixture(RayOut& o, const RayIn& in, const DevScene& S, uint32_t f, uint32_t* status)
{
	XF xf = body_xf(S, S.fixBody[f]);
	float4 p0 = S.fixParams[3 * f], p1 = S.fixParams[3 * f + 1], p2 = S.fixParams[3 * f + 2];
	switch (S.fixType[f])
	{
	case B3G_SHAPE_SPHERE:
		return ray_sphere(o, in, xf, V3{p0.x, p0.y, p0.z}, p0.w);
	case B3G_SHAPE_CAPSULE:
		return ray_capsule(o, in, xf, V3{p0.x, p0.y, p0.z}, V3{p0.w, p1.x, p1.y}, p1.z);
	case B3G_SHAPE_TRIANGLE:
		return ray_triangle(o, in, xf, V3{p0.x, p0.y, p0.z}, V3{p0.w, p1.x, p1.y}, V3{p1.z, p1.w, p2.x});
	case B3G_SHAPE_HULL:
		return ray_hull(o, in, xf, hull_ref(S, S.fixHull[f]));
	case B3G_SHAPE_MESH:
		return ray_mesh(o, in, xf, S, f, status);
	default:
		return false;
	}
}

struct QueryCtx
{
	DevScene S;
	const float4* nodeLo;
	const float4* nodeHi;
	const float4* fatLo;
	const float4* fatHi;
	uint32_t leaves;
	uint32_t* status;
};

__device__ __forceinline__ bool query_takes(const QueryCtx& q, uint32_t f, uint32_t world)
{
	return q.S.fixLife[f] != FIX_DEAD && q.S.bodyWorld[q.S.fixBody[f]] == world;
}

// Rope walk of the LBVH from the root; visit(proxy) for every leaf `accept`
// lets through (internal nodes are descended when `accept` passes them).
template <class Accept, class Visit>
__device__ __forceinline__ void lbvh_walk(const QueryCtx& q, Accept&& accept, Visit&& visit)
{
	const uint32_t nodes = 2u * q.leaves - 1u;
	uint32_t node = 0;
	uint32_t steps = 0;
	while (node != SENT)
	{
		if (++steps > nodes + 1u || node >= nodes)
		{
			atomicOr(q.status, B3G_ST_WAIT_TIMEOUT);
			return;
		}
		float4 lo = q.nodeLo[node], hi = q.nodeHi[node];
		bool pass = accept(V3{lo.x, lo.y, lo.z}, V3{hi.x, hi.y, hi.z});
		if (pass && node < q.leaves - 1u)
		{
			node = __float_as_uint(lo.w);
			continue;
		}
		if (pass)
			visit(__float_as_uint(lo.w));
		node = __float_as_uint(hi.w);
	}
}

// b3World::QueryAABB: fat AABBs overlapping the box (b3TestOverlap, closed).
template <int MODE>
__global__ void k_query_aabb(QueryCtx q, const float* boxes, const uint32_t* worlds, uint32_t n, uint32_t* counts,
	uint2* out, uint32_t capacity)
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	AABB b;
	b.lo = V3{boxes[6 * i], boxes[6 * i + 1], boxes[6 * i + 2]};
	b.hi = V3{boxes[6 * i + 3], boxes[6 * i + 4], boxes[6 * i + 5]};
	uint32_t world = worlds ? worlds[i] : 0u;
	uint32_t k = MODE == 0 ? 0u : counts[i];
	auto overlap = [&](V3 lo, V3 hi) {
		return !(hi.x < b.lo.x || lo.x > b.hi.x || hi.y < b.lo.y || lo.y > b.hi.y || hi.z < b.lo.z || lo.z > b.hi.z);
	};
	lbvh_walk(q, overlap, [&](uint32_t f) {
		float4 lo = q.fatLo[f], hi = q.fatHi[f];
		if (!overlap(V3{lo.x, lo.y, lo.z}, V3{hi.x, hi.y, hi.z}) || !query_takes(q, f, world))
			return;
		if (MODE == 1 && k < capacity)
			out[k] = make_uint2(i, f);
		++k;
	});
	if (MODE == 0)
		counts[i] = k;
}

// b3World::RayCast with a listener that keeps every hit (MODE 0 counts,
// MODE 1 writes fixture + (point, normal, fraction)) and b3World::RayCastSingle
// (MODE 2: the smallest fraction).
template <int MODE>
__global__ void k_ray_cast(QueryCtx q, const float* rays, const uint32_t* worlds, uint32_t n, uint32_t* counts,
	uint2* outIdx, float* outHit, uint32_t capacity, uint32_t* outFix)
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	RayIn in;
	in.p1 = V3{rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]};
	in.p2 = V3{rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]};
	in.maxFraction = 1.0f;
	uint32_t world = worlds ? worlds[i] : 0u;
	uint32_t k = MODE == 1 ? counts[i] : 0u;
	uint32_t best = B3G_NULL;
	RayOut bestOut;
	bestOut.fraction = B3G_MAX_SCALAR;
	bestOut.normal = V3{0.0f, 0.0f, 0.0f};
	if (dot(in.p2 - in.p1, in.p2 - in.p1) > 0.0f)
	{
		SegTest seg;
		seg.init(in.p1, in.p2, in.maxFraction);
		lbvh_walk(q, [&](V3 lo, V3 hi) { return seg.pass(lo, hi); }, [&](uint32_t f) {
			if (!query_takes(q, f, world))
				return;
			RayOut o;
			if (!ray_fixture(o, in, q.S, f, q.status))
				return;
			if (MODE == 2)
			{
				if (o.fraction < bestOut.fraction || (o.fraction == bestOut.fraction && f < best))
				{
					best = f;
					bestOut = o;
					// A fixture hit at or before this fraction has the hit point
					// inside its shape's AABB, at least B3_AABB_EXTENSION inside its
					// fat AABB, so the walk may stop at the hit: the shapes are
					// still ray cast over the whole segment.
					seg.clip(in.p2, o.fraction);
				}
				return;
			}
			if (MODE == 1 && k < capacity)
			{
				V3 p = (1.0f - o.fraction) * in.p1 + o.fraction * in.p2;
				outIdx[k] = make_uint2(i, f);
				float* h = outHit + 7 * (size_t)k;
				h[0] = p.x, h[1] = p.y, h[2] = p.z;
				h[3] = o.normal.x, h[4] = o.normal.y, h[5] = o.normal.z;
				h[6] = o.fraction;
			}
			++k;
		});
	}
	if (MODE == 0)
		counts[i] = k;
	if (MODE == 2)
	{
		outFix[i] = best;
		float* h = outHit + 7 * (size_t)i;
		V3 p = best != B3G_NULL ? (1.0f - bestOut.fraction) * in.p1 + bestOut.fraction * in.p2 : V3{0.0f, 0.0f, 0.0f};
		h[0] = p.x, h[1] = p.y, h[2] = p.z;
		h[3] = bestOut.normal.x, h[4] = bestOut.normal.y, h[5] = bestOut.normal.z;
		h[6] = best != B3G_NULL ? bestOut.fraction : 0.0f;
	}
}

// ---------------------------------------------------------------------------
// Shape casts: b3World::ShapeCast / ShapeCastSingle (world.cpp:568-851), each
// candidate fixture (fat AABB overlapping the swept AABB of the cast shape)
// tested with the translational b3TimeOfImpact (time_of_impact.cpp:666-776)
// and the touching ones evaluated with b3GJK at the time of impact.

// b3TOIOutput::State (time_of_impact.h:40-47).
enum : uint32_t
{
	TOI_UNKNOWN = 0,
	TOI_FAILED,
	TOI_OVERLAPPED,
	TOI_TOUCHING,
	TOI_SEPARATED
};

struct TOIOut
{
	uint32_t state;
	float t;
};

// b3TimeOfImpact(xf1, proxy1, d1, xf2, proxy2, d2) (time_of_impact.cpp:666-776):
// Mirtich's conservative advancement along the translations, the GJK simplex
// carried from one iteration to the next, at most 20 iterations.
__device__ __noinline__ TOIOut toi_translate(const XF& xf1, const GProxy& p1, V3 d1, const XF& xf2, const GProxy& p2,
	V3 d2)
{
	const float totalRadius = p1.radius + p2.radius;
	const float target = fmaxr(B3G_LINEAR_SLOP, totalRadius - 3.0f * B3G_LINEAR_SLOP);
	const float tolerance = 0.25f * B3G_LINEAR_SLOP;
	GJKCache cache;
	cache.count = 0;
	cache.metric = 0.0f;
	for (int i = 0; i < 4; ++i)
		cache.index1[i] = cache.index2[i] = 0u;
	float t = 0.0f;
	XF xf1t = xf1, xf2t = xf2;
	for (uint32_t iteration = 0; iteration < 20u; ++iteration)
	{
		GJKOut q = gjk_cached(xf1t, p1, xf2t, p2, cache);
		if (q.distance == 0.0f)
			return TOIOut{TOI_OVERLAPPED, 0.0f};
		if (q.distance < target + tolerance)
			return TOIOut{TOI_TOUCHING, t};
		V3 n = (q.point2 - q.point1) / q.distance;
		float denominator = dot(d2 - d1, n);
		if (denominator >= 0.0f)
			return TOIOut{TOI_SEPARATED, 1.0f};
		float dt = (target - q.distance) / denominator;
		t += dt;
		if (t >= 1.0f)
			return TOIOut{TOI_SEPARATED, 1.0f};
		xf1t.p = xf1.p + t * d1;
		xf2t.p = xf2.p + t * d2;
	}
	return TOIOut{TOI_UNKNOWN, t};
}

// The proxy of a mesh fixture's triangle (gjk.cpp:75-89): its vertices
// scaled by the mesh scale, the mesh radius.
__device__ GProxy mesh_triangle_proxy(const DevScene& S, uint32_t fix, uint32_t tri)
{
	const MeshDesc md = S.meshes[S.fixHull[fix]];
	const float4 sp = S.fixParams[3 * fix];
	const V3 sc = V3{sp.x, sp.y, sp.z};
	const uint4 t = S.meshTris[md.tOff + tri];
	auto vert = [&](uint32_t i) {
		float4 a = S.meshVerts[md.vOff + i];
		return vmul(sc, V3{a.x, a.y, a.z});
	};
	GProxy g;
	g.gv = nullptr;
	g.lv[0] = vert(t.x);
	g.lv[1] = vert(t.y);
	g.lv[2] = vert(t.z);
	g.count = 3;
	g.radius = sp.w;
	return g;
}

// b3WorldShapeCastQueryWrapper::Evaluate (world.cpp:719-731).
__device__ __noinline__ void cast_evaluate(V3& point, V3& normal, const XF& xA, const GProxy& pA, const XF& xB,
	const GProxy& pB)
{
	GJKOut q = gjk(xA, pA, xB, pB, false);
	normal = normalized(q.point1 - q.point2);
	point = q.point2 + pB.radius * normal;
}

struct CastIn
{
	uint32_t type, hull, world;
	float4 p0, p1, p2;
	XF xf;
	V3 d;
};

// b3g_shape_cast_input: type, hull, world, pad, params[12], position[3],
// rotation[4], displacement[3], pad[2].
__device__ __forceinline__ CastIn load_cast(const float* in, uint32_t i)
{
	const float* r = in + 28 * (size_t)i;
	CastIn c;
	c.type = __float_as_uint(r[0]);
	c.hull = __float_as_uint(r[1]);
	c.world = __float_as_uint(r[2]);
	c.p0 = make_float4(r[4], r[5], r[6], r[7]);
	c.p1 = make_float4(r[8], r[9], r[10], r[11]);
	c.p2 = make_float4(r[12], r[13], r[14], r[15]);
	c.xf.p = V3{r[16], r[17], r[18]};
	c.xf.q = Q4{V3{r[19], r[20], r[21]}, r[22]};
	c.d = V3{r[23], r[24], r[25]};
	return c;
}

// The cast's end transform and swept AABB (world.cpp:759-768).
__device__ __forceinline__ AABB cast_sweep(const DevScene& S, const CastIn& in, XF& xf2)
{
	xf2 = in.xf;
	xf2.p = in.xf.p + in.d;
	AABB a1, a2;
	compute_shape_aabbs(S, in.type, in.p0, in.p1, in.p2, in.hull, in.xf, xf2, true, a1, a2);
	AABB sw;
	sw.lo = vmin(a1.lo, a2.lo);
	sw.hi = vmax(a1.hi, a2.hi);
	return sw;
}

__device__ __forceinline__ bool box_overlap(const AABB& b, float4 lo, float4 hi)
{
	return !(hi.x < b.lo.x || lo.x > b.hi.x || hi.y < b.lo.y || lo.y > b.hi.y || hi.z < b.lo.z || lo.z > b.hi.z);
}

// Mesh fixture f against cast `in`: the triangles under the swept box in the
// unscaled mesh frame (world.cpp:638-664), in the static tree's depth-first
// order; visit(triangle, toi, proxy) for each touching one.
template <class Visit>
__device__ __forceinline__ void cast_mesh(const QueryCtx& q, const CastIn& in, const GProxy& pA, const XF& xf2,
	uint32_t f, const XF& xfB, Visit&& visit)
{
	const DevScene& S = q.S;
	const MeshDesc md = S.meshes[S.fixHull[f]];
	const float4 sp = S.fixParams[3 * f];
	const V3 inv = V3{1.0f / sp.x, 1.0f / sp.y, 1.0f / sp.z};
	AABB m1, m2;
	compute_shape_aabbs(S, in.type, in.p0, in.p1, in.p2, in.hull, xmult(xfB, in.xf), xmult(xfB, xf2), true, m1, m2);
	m1 = aabb_scaled(m1, inv);
	m2 = aabb_scaled(m2, inv);
	AABB box;
	box.lo = vmin(m1.lo, m2.lo);
	box.hi = vmax(m1.hi, m2.hi);
	const V3 zero = V3{0.0f, 0.0f, 0.0f};
	constexpr uint32_t STACK = 64;
	uint32_t stack[STACK];
	uint32_t sp_ = 0;
	stack[sp_++] = md.root;
	while (sp_ > 0)
	{
		uint32_t id = stack[--sp_];
		if (id == B3G_NULL_NODE)
			continue;
		float4 nlo = S.meshNodes[2 * (size_t)(md.nOff + id)], nhi = S.meshNodes[2 * (size_t)(md.nOff + id) + 1];
		if (!box_overlap(box, nlo, nhi))
			continue;
		uint32_t child1 = __float_as_uint(nlo.w), other = __float_as_uint(nhi.w);
		if (child1 == B3G_NULL_NODE)
		{
			const GProxy pB = mesh_triangle_proxy(S, f, other);
			TOIOut r = toi_translate(in.xf, pA, in.d, xfB, pB, zero);
			if (r.state == TOI_TOUCHING)
				visit(other, r.t, pB);
		}
		else
		{
			if (sp_ + 2 > STACK)
			{
				atomicOr(q.status, B3G_ST_POLY_OVERFLOW);
				return;
			}
			stack[sp_++] = child1;
			stack[sp_++] = other;
		}
	}
}

// One (cast, fixture) candidate on one lane: the time of impact against a
// convex fixture, or against each triangle of a mesh fixture. MODE 0 counts
// the touching results in *count, MODE 1 writes them (slot base + a count
// taken from *count), MODE 2 lowers *best to (fraction bits, fixture).
template <int MODE>
__device__ __noinline__ void cast_candidate(const QueryCtx& q, const float* casts, uint32_t i, uint32_t f,
	uint32_t* count, uint32_t base, uint32_t* outIdx, float* outHit, uint32_t capacity, unsigned long long* best)
{
	const DevScene& S = q.S;
	const CastIn in = load_cast(casts, i);
	const GProxy pA = convex_proxy(S, in.type, in.p0, in.p1, in.p2, in.hull);
	const XF xfB = body_xf(S, S.fixBody[f]);
	auto act = [&](uint32_t child, float t, const GProxy& pB) {
		if (MODE == 2)
		{
			atomicMin(best, ((unsigned long long)__float_as_uint(t) << 32) | f);
			return;
		}
		const uint32_t slot = atomicAdd(count, 1u);
		if (MODE == 1 && base + slot < capacity)
		{
			XF xt;
			xt.q = in.xf.q;
			xt.p = in.xf.p + t * in.d;
			V3 point, normal;
			cast_evaluate(point, normal, xt, pA, xfB, pB);
			uint32_t* o = outIdx + 3 * (size_t)(base + slot);
			o[0] = i;
			o[1] = f;
			o[2] = child;
			float* h = outHit + 7 * (size_t)(base + slot);
			h[0] = point.x, h[1] = point.y, h[2] = point.z;
			h[3] = normal.x, h[4] = normal.y, h[5] = normal.z;
			h[6] = t;
		}
	};
	if (S.fixType[f] != B3G_SHAPE_MESH)
	{
		const GProxy pB =
			convex_proxy(S, S.fixType[f], S.fixParams[3 * f], S.fixParams[3 * f + 1], S.fixParams[3 * f + 2], S.fixHull[f]);
		TOIOut r = toi_translate(in.xf, pA, in.d, xfB, pB, V3{0.0f, 0.0f, 0.0f});
		if (r.state == TOI_TOUCHING)
			act(0u, r.t, pB);
		return;
	}
	XF xf2;
	cast_sweep(S, in, xf2);
	cast_mesh(q, in, pA, xf2, f, xfB, act);
}

// b3World::ShapeCast with a listener that returns 1 for every fixture
// (MODE 0 counts, MODE 1 writes (cast, fixture, triangle) + (point, normal,
// fraction), in no particular order within a cast) and
// b3World::ShapeCastSingle (MODE 2: the smallest fraction, then the smaller
// fixture and triangle on an exact tie).
//
// A warp holds 32 casts. Its lanes walk their casts' LBVH paths only until
// each finds its next candidate fixture (fat AABB overlapping the swept box)
// and push it into the warp's queue in shared memory; whenever 32 candidates
// are queued (or the walks are over) every lane takes one and runs its time
// of impact, so the lanes run the same GJK code on different candidates
// instead of each walking and testing its own cast alone. Per-cast results
// meet in shared memory (counts, or the smallest (fraction, fixture) key).
template <int MODE>
__global__ void __launch_bounds__(128) k_shape_cast(QueryCtx q, const float* casts, const uint32_t* order, uint32_t n,
	uint32_t* counts, uint32_t* outIdx, float* outHit, uint32_t capacity, uint32_t* outSingle)
{
	constexpr int WARPS = 4;
	__shared__ uint32_t qLane[WARPS][64], qFix[WARPS][64];
	__shared__ uint32_t sCount[WARPS][32];
	__shared__ unsigned long long sBest[WARPS][32];
	const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
	const uint32_t warpBase = blockIdx.x * blockDim.x + w * 32u;
	const uint32_t t = warpBase + lane;
	const bool active = t < n;
	// Casts are taken in the order of their Morton keys, so the lanes of a
	// warp walk neighbouring parts of the tree; results go to their own slots.
	const uint32_t i = active ? (order ? order[t] : t) : 0u;
	sCount[w][lane] = 0;
	sBest[w][lane] = ~0ull;
	__syncwarp();
	const DevScene& S = q.S;
	bool walking = false;
	uint32_t world = 0;
	AABB sw;
	sw.lo = sw.hi = V3{0.0f, 0.0f, 0.0f};
	if (active)
	{
		const CastIn in = load_cast(casts, i);
		// A mesh cannot be cast (world.cpp:755-760).
		walking = in.type != B3G_SHAPE_MESH;
		world = in.world;
		XF xf2;
		sw = cast_sweep(S, in, xf2);
	}
	const uint32_t nodes = 2u * q.leaves - 1u;
	uint32_t node = 0, steps = 0, qn = 0;
	for (;;)
	{
		uint32_t f = 0;
		bool got = false;
		while (walking && node != SENT)
		{
			if (++steps > nodes + 1u || node >= nodes)
			{
				atomicOr(q.status, B3G_ST_WAIT_TIMEOUT);
				node = SENT;
				break;
			}
			const float4 lo = q.nodeLo[node], hi = q.nodeHi[node];
			const bool pass = box_overlap(sw, lo, hi);
			if (pass && node < q.leaves - 1u)
			{
				node = __float_as_uint(lo.w);
				continue;
			}
			node = __float_as_uint(hi.w);
			if (pass)
			{
				const uint32_t proxy = __float_as_uint(lo.w);
				if (box_overlap(sw, q.fatLo[proxy], q.fatHi[proxy]) && query_takes(q, proxy, world))
				{
					f = proxy;
					got = true;
					break;
				}
			}
		}
		if (!got)
			walking = false;
		const uint32_t m = __ballot_sync(0xFFFFFFFFu, got);
		if (got)
		{
			const uint32_t pos = qn + __popc(m & ((1u << lane) - 1u));
			qLane[w][pos] = lane;
			qFix[w][pos] = f;
		}
		qn += __popc(m);
		const bool more = __any_sync(0xFFFFFFFFu, walking);
		if (qn >= 32u || (!more && qn > 0u))
		{
			__syncwarp();
			const uint32_t take = min(qn, 32u);
			if (lane < take)
			{
				const uint32_t e = qn - take + lane;
				const uint32_t cl = qLane[w][e];
				const uint32_t ci = order ? order[warpBase + cl] : warpBase + cl;
				cast_candidate<MODE>(q, casts, ci, qFix[w][e], &sCount[w][cl], MODE == 1 ? counts[ci] : 0u, outIdx,
					outHit, capacity, &sBest[w][cl]);
			}
			qn -= take;
			__syncwarp();
		}
		if (!more && qn == 0u)
			break;
	}
	__syncwarp();
	if (!active)
		return;
	if (MODE == 0)
		counts[i] = sCount[w][lane];
	if (MODE == 2)
	{
		const unsigned long long key = sBest[w][lane];
		uint32_t bestF = B3G_NULL, bestChild = B3G_NULL;
		float* h = outHit + 7 * (size_t)i;
		if (key != ~0ull)
		{
			bestF = (uint32_t)(key & 0xFFFFFFFFull);
			const float bestT = __uint_as_float((uint32_t)(key >> 32));
			const CastIn in = load_cast(casts, i);
			const GProxy pA = convex_proxy(S, in.type, in.p0, in.p1, in.p2, in.hull);
			const XF xfB = body_xf(S, S.fixBody[bestF]);
			GProxy pB;
			pB.gv = nullptr;
			pB.lv[0] = pB.lv[1] = pB.lv[2] = V3{0.0f, 0.0f, 0.0f};
			pB.count = 1;
			pB.radius = 0.0f;
			if (S.fixType[bestF] == B3G_SHAPE_MESH)
			{
				// The winning mesh's smallest triangle at that fraction.
				XF xf2;
				cast_sweep(S, in, xf2);
				cast_mesh(q, in, pA, xf2, bestF, xfB, [&](uint32_t tri, float tt, const GProxy& pt) {
					if (tt == bestT && tri < bestChild)
					{
						bestChild = tri;
						pB = pt;
					}
				});
			}
			else
			{
				bestChild = 0;
				pB = convex_proxy(S, S.fixType[bestF], S.fixParams[3 * bestF], S.fixParams[3 * bestF + 1],
					S.fixParams[3 * bestF + 2], S.fixHull[bestF]);
			}
			// b3World::ShapeCastSingle (world.cpp:828-848): evaluate the winner.
			XF xt;
			xt.q = in.xf.q;
			xt.p = in.xf.p + bestT * in.d;
			V3 point, normal;
			cast_evaluate(point, normal, xt, pA, xfB, pB);
			h[0] = point.x, h[1] = point.y, h[2] = point.z;
			h[3] = normal.x, h[4] = normal.y, h[5] = normal.z;
			h[6] = bestT;
		}
		else
		{
			for (int e = 0; e < 7; ++e)
				h[e] = 0.0f;
		}
		outSingle[2 * (size_t)i] = bestF;
		outSingle[2 * (size_t)i + 1] = bestChild;
	}
}

__device__ __forceinline__ uint32_t cast_expand10(uint32_t v)
{
	v = (v * 0x00010001u) & 0xFF0000FFu;
	v = (v * 0x00000101u) & 0x0F00F00Fu;
	v = (v * 0x00000011u) & 0xC30C30C3u;
	v = (v * 0x00000005u) & 0x49249249u;
	return v;
}

// Sort keys of the casts: world, then the 30-bit Morton code of the middle of
// the sweep within the tree's root box.
__global__ void k_cast_keys(const float* casts, uint32_t n, const float4* nodeLo, const float4* nodeHi,
	unsigned long long* keys, uint32_t* vals)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const float* r = casts + 28 * (size_t)i;
	const float4 lo = nodeLo[0], hi = nodeHi[0];
	const float c[3] = {r[16] + 0.5f * r[23], r[17] + 0.5f * r[24], r[18] + 0.5f * r[25]};
	const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
	uint32_t qv[3];
	for (int k = 0; k < 3; ++k)
	{
		float ext = h[k] - l[k];
		float t = ext > 0.0f ? (c[k] - l[k]) / ext : 0.0f;
		t = fminf(fmaxf(t, 0.0f), 1.0f);
		qv[k] = min((uint32_t)(t * 1024.0f), 1023u);
	}
	const uint32_t code = (cast_expand10(qv[0]) << 2) | (cast_expand10(qv[1]) << 1) | cast_expand10(qv[2]);
	keys[i] = ((unsigned long long)__float_as_uint(r[2]) << 30) | code;
	vals[i] = i;
}

int qfail(b3g_ctx* c, int code, const char* msg)
{
	c->err = msg;
	return code;
}

// Device scratch of the query calls, grown on demand.
bool q_reserve(b3g_ctx* c, size_t bytes)
{
	if (c->qScratchBytes >= bytes)
		return true;
	if (c->qScratch)
		cudaFree(c->qScratch);
	c->qScratch = nullptr;
	c->qScratchBytes = 0;
	size_t want = bytes < ((size_t)1 << 20) ? ((size_t)1 << 20) : bytes;
	if (cudaMalloc(&c->qScratch, want) != cudaSuccess)
		return false;
	c->qScratchBytes = want;
	return true;
}

int q_begin(b3g_ctx* c, uint32_t n, const void* in, size_t inBytes, const uint32_t* worlds, QueryCtx& q,
	size_t extraBytes, char*& base, const uint32_t*& dWorlds, const void*& dIn)
{
	if (!c->havePass || c->treeLeaves == 0)
		return qfail(c, B3G_E_STATE, "world query: no collision pass yet");
	if (n > std::max(c->cfg.max_proxies, c->cfg.max_contacts))
		return qfail(c, B3G_E_CAPACITY, "world query: more queries than max(max_proxies, max_contacts) per call");
	if (cudaSetDevice(c->device) != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "world query: device");
	auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
	size_t need = al(inBytes) + al(4 * (size_t)n) + extraBytes;
	if (!q_reserve(c, need))
		return qfail(c, B3G_E_CUDA, "world query: device allocation failed");
	base = (char*)c->qScratch;
	dIn = base;
	if (cudaMemcpyAsync(base, in, inBytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "world query: copy");
	base += al(inBytes);
	dWorlds = nullptr;
	if (worlds)
	{
		if (cudaMemcpyAsync(base, worlds, 4 * (size_t)n, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
			return qfail(c, B3G_E_CUDA, "world query: copy");
		dWorlds = (const uint32_t*)base;
	}
	base += al(4 * (size_t)n);
	q.S = c->scene;
	q.nodeLo = c->buf.nodeLo;
	q.nodeHi = c->buf.nodeHi;
	q.fatLo = c->buf.fatLo;
	q.fatHi = c->buf.fatHi;
	q.leaves = c->treeLeaves;
	q.status = c->buf.counters + CTR_SCRATCH;
	return B3G_OK;
}

int q_status(b3g_ctx* c)
{
	uint32_t st = 0;
	if (cudaMemcpyAsync(&st, c->buf.counters + CTR_SCRATCH, 4, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
		cudaStreamSynchronize(c->stream) != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "world query: kernel failed");
	if (st)
		return qfail(c, st & B3G_ST_WAIT_TIMEOUT ? B3G_E_TIMEOUT : B3G_E_CAPACITY,
			"world query: tree walk stopped (stack or step limit)");
	return B3G_OK;
}

} // namespace

extern "C" int b3g_query_aabb(b3g_ctx* c, uint32_t n, const float* boxes, const uint32_t* worlds, uint32_t* out,
	uint32_t capacity)
{
	if (!c || (n && (!boxes || (!out && capacity))))
		return c ? qfail(c, B3G_E_INVALID, "b3g_query_aabb: null argument") : B3G_E_INVALID;
	if (n == 0)
		return 0;
	QueryCtx q;
	char* base;
	const uint32_t* dWorlds;
	const void* dIn;
	const size_t cntBytes = ((4 * (size_t)n + 4 + 255) & ~(size_t)255);
	const size_t outBytes = 8 * (size_t)capacity;
	int rc = q_begin(c, n, boxes, 24 * (size_t)n, worlds, q, cntBytes + outBytes + 256, base, dWorlds, dIn);
	if (rc)
		return rc;
	uint32_t* counts = (uint32_t*)base;
	uint2* dOut = (uint2*)(base + cntBytes);
	cudaStream_t s = c->stream;
	cudaMemsetAsync(c->buf.counters + CTR_SCRATCH, 0, 4, s);
	const uint32_t blocks = (n + 127) / 128;
	k_query_aabb<0><<<blocks, 128, 0, s>>>(q, (const float*)dIn, dWorlds, n, counts, dOut, capacity);
	scan_exclusive(counts, n, c->buf.scanAux, counts + n, c->buf.counters + CTR_STATUS, s);
	k_query_aabb<1><<<blocks, 128, 0, s>>>(q, (const float*)dIn, dWorlds, n, counts, dOut, capacity);
	uint32_t total = 0;
	if (cudaMemcpyAsync(&total, counts + n, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "b3g_query_aabb: copy");
	rc = q_status(c);
	if (rc)
		return rc;
	uint32_t m = total < capacity ? total : capacity;
	if (m && cudaMemcpy(out, dOut, 8 * (size_t)m, cudaMemcpyDeviceToHost) != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "b3g_query_aabb: copy");
	return (int)total;
}

extern "C" int b3g_ray_cast(b3g_ctx* c, uint32_t n, const float* rays, const uint32_t* worlds, uint32_t* index,
	float* hits, uint32_t capacity)
{
	if (!c || (n && (!rays || ((!index || !hits) && capacity))))
		return c ? qfail(c, B3G_E_INVALID, "b3g_ray_cast: null argument") : B3G_E_INVALID;
	if (n == 0)
		return 0;
	QueryCtx q;
	char* base;
	const uint32_t* dWorlds;
	const void* dIn;
	const size_t cntBytes = ((4 * (size_t)n + 4 + 255) & ~(size_t)255);
	const size_t idxBytes = ((8 * (size_t)capacity + 255) & ~(size_t)255);
	int rc = q_begin(c, n, rays, 24 * (size_t)n, worlds, q, cntBytes + idxBytes + 28 * (size_t)capacity + 256, base,
		dWorlds, dIn);
	if (rc)
		return rc;
	uint32_t* counts = (uint32_t*)base;
	uint2* dIdx = (uint2*)(base + cntBytes);
	float* dHit = (float*)(base + cntBytes + idxBytes);
	cudaStream_t s = c->stream;
	cudaMemsetAsync(c->buf.counters + CTR_SCRATCH, 0, 4, s);
	const uint32_t blocks = (n + 127) / 128;
	k_ray_cast<0><<<blocks, 128, 0, s>>>(q, (const float*)dIn, dWorlds, n, counts, dIdx, dHit, capacity, nullptr);
	scan_exclusive(counts, n, c->buf.scanAux, counts + n, c->buf.counters + CTR_STATUS, s);
	k_ray_cast<1><<<blocks, 128, 0, s>>>(q, (const float*)dIn, dWorlds, n, counts, dIdx, dHit, capacity, nullptr);
	uint32_t total = 0;
	if (cudaMemcpyAsync(&total, counts + n, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "b3g_ray_cast: copy");
	rc = q_status(c);
	if (rc)
		return rc;
	uint32_t m = total < capacity ? total : capacity;
	if (m && (cudaMemcpy(index, dIdx, 8 * (size_t)m, cudaMemcpyDeviceToHost) != cudaSuccess ||
				 cudaMemcpy(hits, dHit, 28 * (size_t)m, cudaMemcpyDeviceToHost) != cudaSuccess))
		return qfail(c, B3G_E_CUDA, "b3g_ray_cast: copy");
	return (int)total;
}

extern "C" int b3g_ray_cast_single(b3g_ctx* c, uint32_t n, const float* rays, const uint32_t* worlds,
	uint32_t* fixture, float* hit)
{
	if (!c || (n && (!rays || !fixture || !hit)))
		return c ? qfail(c, B3G_E_INVALID, "b3g_ray_cast_single: null argument") : B3G_E_INVALID;
	if (n == 0)
		return 0;
	QueryCtx q;
	char* base;
	const uint32_t* dWorlds;
	const void* dIn;
	const size_t fixBytes = ((4 * (size_t)n + 255) & ~(size_t)255);
	int rc = q_begin(c, n, rays, 24 * (size_t)n, worlds, q, fixBytes + 28 * (size_t)n + 256, base, dWorlds, dIn);
	if (rc)
		return rc;
	uint32_t* dFix = (uint32_t*)base;
	float* dHit = (float*)(base + fixBytes);
	cudaStream_t s = c->stream;
	cudaMemsetAsync(c->buf.counters + CTR_SCRATCH, 0, 4, s);
	k_ray_cast<2><<<(n + 127) / 128, 128, 0, s>>>(q, (const float*)dIn, dWorlds, n, nullptr, nullptr, dHit, n, dFix);
	rc = q_status(c);
	if (rc)
		return rc;
	if (cudaMemcpy(fixture, dFix, 4 * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess ||
		cudaMemcpy(hit, dHit, 28 * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "b3g_ray_cast_single: copy");
	int hits = 0;
	for (uint32_t i = 0; i < n; ++i)
		hits += fixture[i] != B3G_NULL ? 1 : 0;
	return hits;
}

extern "C" int b3g_ray_cast_single_device(b3g_ctx* c, uint32_t n, const float* rays, const uint32_t* worlds,
	uint32_t* fixture, float* hit, void* stream)
{
	if (!c || (n && (!rays || !fixture || !hit)))
		return c ? qfail(c, B3G_E_INVALID, "b3g_ray_cast_single_device: null argument") : B3G_E_INVALID;
	if (!c->havePass || c->treeLeaves == 0)
		return qfail(c, B3G_E_STATE, "world query: no collision pass yet");
	if (n == 0)
		return B3G_OK;
	QueryCtx q;
	q.S = c->scene;
	q.nodeLo = c->buf.nodeLo;
	q.nodeHi = c->buf.nodeHi;
	q.fatLo = c->buf.fatLo;
	q.fatHi = c->buf.fatHi;
	q.leaves = c->treeLeaves;
	q.status = c->buf.counters + CTR_SCRATCH;
	cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
	k_ray_cast<2><<<(n + 127) / 128, 128, 0, s>>>(q, rays, worlds, n, nullptr, nullptr, hit, n, fixture);
	if (cudaGetLastError() != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "b3g_ray_cast_single_device: launch");
	return B3G_OK;
}

// Host check of the casts: the shape types a cast may have and their hulls.
static_assert(sizeof(b3g_shape_cast_input) == 112, "b3g_shape_cast_input: 28 words");

// Scratch bytes of cast_order for n casts.
static size_t cast_order_bytes(uint32_t n)
{
	auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
	return 2 * al(8 * (size_t)n) + 2 * al(4 * (size_t)n) + al(4 * (size_t)radix_sort_scratch_words(n, 48));
}

// The casts' processing order (sorted by world and Morton key) in scratch
// at p; returns the order array.
static const uint32_t* cast_order(b3g_ctx* c, const float* dCasts, uint32_t n, char* p, uint32_t worldBits,
	cudaStream_t s)
{
	auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
	unsigned long long* keys = (unsigned long long*)p;
	p += al(8 * (size_t)n);
	unsigned long long* keysTmp = (unsigned long long*)p;
	p += al(8 * (size_t)n);
	uint32_t* vals = (uint32_t*)p;
	p += al(4 * (size_t)n);
	uint32_t* valsTmp = (uint32_t*)p;
	p += al(4 * (size_t)n);
	uint32_t* scratch = (uint32_t*)p;
	k_cast_keys<<<(n + 255) / 256, 256, 0, s>>>(dCasts, n, c->buf.nodeLo, c->buf.nodeHi, keys, vals);
	bool swapped = radix_sort_pairs(keys, vals, keysTmp, valsTmp, n, 30 + (int)worldBits, scratch,
		c->buf.counters + CTR_SCRATCH, s);
	return swapped ? valsTmp : vals;
}

static uint32_t world_bits(const b3g_ctx* c)
{
	uint32_t b = 0;
	while (b < 18 && (1u << b) < c->nWorlds)
		++b;
	return b;
}

static int cast_check(b3g_ctx* c, uint32_t n, const b3g_shape_cast_input* casts)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		const uint32_t t = casts[i].shape_type;
		if (t > B3G_SHAPE_MESH)
			return qfail(c, B3G_E_INVALID, "shape cast: unknown shape type");
		if (t == B3G_SHAPE_HULL && casts[i].hull >= c->nHulls)
			return qfail(c, B3G_E_INVALID, "shape cast: hull out of range");
	}
	return B3G_OK;
}

extern "C" int b3g_shape_cast(b3g_ctx* c, uint32_t n, const b3g_shape_cast_input* casts, uint32_t* index,
	float* hits, uint32_t capacity)
{
	if (!c || (n && (!casts || ((!index || !hits) && capacity))))
		return c ? qfail(c, B3G_E_INVALID, "b3g_shape_cast: null argument") : B3G_E_INVALID;
	if (n == 0)
		return 0;
	int rc = cast_check(c, n, casts);
	if (rc)
		return rc;
	QueryCtx q;
	char* base;
	const uint32_t* dWorlds;
	const void* dIn;
	const size_t cntBytes = ((4 * (size_t)n + 4 + 255) & ~(size_t)255);
	const size_t idxBytes = ((12 * (size_t)capacity + 255) & ~(size_t)255);
	const size_t hitBytes = ((28 * (size_t)capacity + 255) & ~(size_t)255);
	rc = q_begin(c, n, casts, sizeof(b3g_shape_cast_input) * (size_t)n, nullptr, q,
		cntBytes + idxBytes + hitBytes + cast_order_bytes(n) + 256, base, dWorlds, dIn);
	if (rc)
		return rc;
	uint32_t* counts = (uint32_t*)base;
	uint32_t* dIdx = (uint32_t*)(base + cntBytes);
	float* dHit = (float*)(base + cntBytes + idxBytes);
	cudaStream_t s = c->stream;
	cudaMemsetAsync(c->buf.counters + CTR_SCRATCH, 0, 4, s);
	const uint32_t* order =
		cast_order(c, (const float*)dIn, n, base + cntBytes + idxBytes + hitBytes, world_bits(c), s);
	const uint32_t blocks = (n + 127) / 128;
	k_shape_cast<0><<<blocks, 128, 0, s>>>(q, (const float*)dIn, order, n, counts, dIdx, dHit, capacity, nullptr);
	scan_exclusive(counts, n, c->buf.scanAux, counts + n, c->buf.counters + CTR_STATUS, s);
	k_shape_cast<1><<<blocks, 128, 0, s>>>(q, (const float*)dIn, order, n, counts, dIdx, dHit, capacity, nullptr);
	uint32_t total = 0;
	if (cudaMemcpyAsync(&total, counts + n, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "b3g_shape_cast: copy");
	rc = q_status(c);
	if (rc)
		return rc;
	uint32_t m = total < capacity ? total : capacity;
	if (m && (cudaMemcpy(index, dIdx, 12 * (size_t)m, cudaMemcpyDeviceToHost) != cudaSuccess ||
				 cudaMemcpy(hits, dHit, 28 * (size_t)m, cudaMemcpyDeviceToHost) != cudaSuccess))
		return qfail(c, B3G_E_CUDA, "b3g_shape_cast: copy");
	return (int)total;
}

extern "C" int b3g_shape_cast_single(b3g_ctx* c, uint32_t n, const b3g_shape_cast_input* casts, uint32_t* fixture,
	float* hit)
{
	if (!c || (n && (!casts || !fixture || !hit)))
		return c ? qfail(c, B3G_E_INVALID, "b3g_shape_cast_single: null argument") : B3G_E_INVALID;
	if (n == 0)
		return 0;
	int rc = cast_check(c, n, casts);
	if (rc)
		return rc;
	QueryCtx q;
	char* base;
	const uint32_t* dWorlds;
	const void* dIn;
	const size_t fixBytes = ((8 * (size_t)n + 255) & ~(size_t)255);
	const size_t hitBytes = ((28 * (size_t)n + 255) & ~(size_t)255);
	rc = q_begin(c, n, casts, sizeof(b3g_shape_cast_input) * (size_t)n, nullptr, q,
		fixBytes + hitBytes + cast_order_bytes(n) + 256, base, dWorlds, dIn);
	if (rc)
		return rc;
	uint32_t* dFix = (uint32_t*)base;
	float* dHit = (float*)(base + fixBytes);
	cudaStream_t s = c->stream;
	cudaMemsetAsync(c->buf.counters + CTR_SCRATCH, 0, 4, s);
	const uint32_t* order = cast_order(c, (const float*)dIn, n, base + fixBytes + hitBytes, world_bits(c), s);
	k_shape_cast<2><<<(n + 127) / 128, 128, 0, s>>>(q, (const float*)dIn, order, n, nullptr, nullptr, dHit, n, dFix);
	rc = q_status(c);
	if (rc)
		return rc;
	if (cudaMemcpy(fixture, dFix, 8 * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess ||
		cudaMemcpy(hit, dHit, 28 * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "b3g_shape_cast_single: copy");
	int hits = 0;
	for (uint32_t i = 0; i < n; ++i)
		hits += fixture[2 * i] != B3G_NULL ? 1 : 0;
	return hits;
}

extern "C" int b3g_shape_cast_single_device(b3g_ctx* c, uint32_t n, const b3g_shape_cast_input* casts,
	uint32_t* fixture, float* hit, void* stream)
{
	if (!c || (n && (!casts || !fixture || !hit)))
		return c ? qfail(c, B3G_E_INVALID, "b3g_shape_cast_single_device: null argument") : B3G_E_INVALID;
	if (!c->havePass || c->treeLeaves == 0)
		return qfail(c, B3G_E_STATE, "world query: no collision pass yet");
	if (n == 0)
		return B3G_OK;
	QueryCtx q;
	q.S = c->scene;
	q.nodeLo = c->buf.nodeLo;
	q.nodeHi = c->buf.nodeHi;
	q.fatLo = c->buf.fatLo;
	q.fatHi = c->buf.fatHi;
	q.leaves = c->treeLeaves;
	q.status = c->buf.counters + CTR_SCRATCH;
	cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
	if (n > std::max(c->cfg.max_proxies, c->cfg.max_contacts))
		return qfail(c, B3G_E_CAPACITY, "world query: more queries than max(max_proxies, max_contacts) per call");
	if (!q_reserve(c, cast_order_bytes(n)))
		return qfail(c, B3G_E_CUDA, "world query: device allocation failed");
	const uint32_t* order = cast_order(c, (const float*)casts, n, (char*)c->qScratch, world_bits(c), s);
	k_shape_cast<2><<<(n + 127) / 128, 128, 0, s>>>(q, (const float*)casts, order, n, nullptr, nullptr, hit, n,
		fixture);
	if (cudaGetLastError() != cudaSuccess)
		return qfail(c, B3G_E_CUDA, "b3g_shape_cast_single_device: launch");
	return B3G_OK;
}

void free_queries(b3g_ctx* c)
{
	if (c->qScratch)
		cudaFree(c->qScratch);
	c->qScratch = nullptr;
	c->qScratchBytes = 0;
}

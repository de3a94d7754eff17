// Time of impact and GJK shape cast as batched device functions, one thread
// per query, with the reference's arithmetic:
//   b3TimeOfImpact(const b3TOIInput&)   time_of_impact.cpp:26-660 (the local
//       separating axis method on two sweeps: b3SeparationFunction, the
//       secant / bisection root finder, b3GJK with its simplex cache)
//   b3TimeOfImpact(aabb1, d1, aabb2, d2) time_of_impact.cpp:782-902
//   b3ShapeCast                          gjk.cpp:938-1102 (GJK ray cast)
// with b3GetFeaturePair (gjk_feature_pair.cpp:21-236) and
// b3Sweep::GetTransform (sweep.h:43-63).
#include "collide_common.cuh"

static_assert(sizeof(b3g_toi_input) == 272, "b3g_toi_input: 68 words");
static_assert(sizeof(b3g_gjk_cast_input) == 192, "b3g_gjk_cast_input: 48 words");

namespace {

// b3Sweep in the b3g_toi_input layout: localCenter, orientation0,
// worldCenter0, t0, orientation, worldCenter (sweep.h:28-41).
struct Sweep
{
	V3 lc;
	Q4 q0;
	V3 c0;
	Q4 q;
	V3 c;
};

__device__ __forceinline__ Sweep load_sweep(const float* s)
{
	Sweep w;
	w.lc = V3{s[0], s[1], s[2]};
	w.q0 = Q4{V3{s[3], s[4], s[5]}, s[6]};
	w.c0 = V3{s[7], s[8], s[9]};
	w.q = Q4{V3{s[11], s[12], s[13]}, s[14]};
	w.c = V3{s[15], s[16], s[17]};
	return w;
}

// b3Sweep::GetTransform (sweep.h:43-63). Kept out of line (as are the
// separation function's methods): the time of impact calls them from many
// places, and inlined copies overflow the instruction cache.
__device__ __noinline__ XF sweep_at(const Sweep& w, float t)
{
	const V3 c = (1.0f - t) * w.c0 + t * w.c;
	Q4 q1 = w.q0;
	const Q4 q2 = w.q;
	if (qdot(q1, q2) < 0.0f)
		q1 = qneg(q1);
	const float u = 1.0f - t;
	Q4 q = Q4{u * q1.v + t * q2.v, u * q1.s + t * q2.s};
	qnormalize_inplace(q);
	XF xf;
	xf.p = c - rot(q, w.lc);
	xf.q = q;
	return xf;
}

// b3UniqueCount (math.h:84-104).
__device__ __forceinline__ uint32_t unique3(const uint32_t* v, uint32_t n)
{
	uint32_t count = 0;
	for (uint32_t i = 0; i < n; ++i)
	{
		uint32_t j = 0;
		while (j < n && v[i] != v[j])
			++j;
		count += i == j ? 1u : 0u;
	}
	return count;
}

struct FeaturePair
{
	uint32_t index1[3], count1, index2[3], count2;
};

// b3GetFeaturePair (gjk_feature_pair.cpp:21-236); counts 0 for the
// combinations the reference asserts never happen.
__device__ FeaturePair feature_pair(const GJKCache& cache)
{
	FeaturePair p;
	p.count1 = p.count2 = 0;
	for (int k = 0; k < 3; ++k)
		p.index1[k] = p.index2[k] = 0;
	const uint32_t n = cache.count;
	if (n == 0 || n > 3)
		return p;
	const uint32_t u1 = unique3(cache.index1, n), u2 = unique3(cache.index2, n);
	auto second = [](const uint32_t* v) { return v[0] == v[1] ? v[2] : v[1]; };
	if (n == 1)
	{
		p.count1 = p.count2 = 1;
		p.index1[0] = cache.index1[0];
		p.index2[0] = cache.index2[0];
		return p;
	}
	if (n == 2)
	{
		if (u1 == 2 && u2 == 2)
		{
			p.count1 = p.count2 = 2;
			p.index1[0] = cache.index1[0];
			p.index1[1] = cache.index1[1];
			p.index2[0] = cache.index2[0];
			p.index2[1] = cache.index2[1];
		}
		else if (u1 == 1)
		{
			p.count1 = 1;
			p.count2 = 2;
			p.index1[0] = cache.index1[0];
			p.index2[0] = cache.index2[0];
			p.index2[1] = cache.index2[1];
		}
		else if (u2 == 1)
		{
			p.count1 = 2;
			p.count2 = 1;
			p.index1[0] = cache.index1[0];
			p.index1[1] = cache.index1[1];
			p.index2[0] = cache.index2[0];
		}
		return p;
	}
	if (u1 == 1 && u2 == 3)
	{
		p.count1 = 1;
		p.count2 = 3;
		p.index1[0] = cache.index1[0];
		for (int k = 0; k < 3; ++k)
			p.index2[k] = cache.index2[k];
	}
	else if (u1 == 3 && u2 == 1)
	{
		p.count1 = 3;
		p.count2 = 1;
		for (int k = 0; k < 3; ++k)
			p.index1[k] = cache.index1[k];
		p.index2[0] = cache.index2[0];
	}
	else if (u1 == 2 && u2 == 2)
	{
		p.count1 = p.count2 = 2;
		p.index1[0] = cache.index1[0];
		p.index1[1] = second(cache.index1);
		p.index2[0] = cache.index2[0];
		p.index2[1] = second(cache.index2);
	}
	else if (u1 == 2 && u2 == 3)
	{
		p.count1 = 2;
		p.count2 = 3;
		p.index1[0] = cache.index1[0];
		p.index1[1] = second(cache.index1);
		for (int k = 0; k < 3; ++k)
			p.index2[k] = cache.index2[k];
	}
	else if (u1 == 3 && u2 == 2)
	{
		p.count1 = 3;
		p.count2 = 2;
		for (int k = 0; k < 3; ++k)
			p.index1[k] = cache.index1[k];
		p.index2[0] = cache.index2[0];
		p.index2[1] = second(cache.index2);
	}
	else if (u1 == 3 && u2 == 3)
	{
		p.count1 = p.count2 = 3;
		for (int k = 0; k < 3; ++k)
		{
			p.index1[k] = cache.index1[k];
			p.index2[k] = cache.index2[k];
		}
	}
	return p;
}

enum : uint32_t
{
	SEP_POINTS = 0,
	SEP_EDGE_A,
	SEP_FACE_A,
	SEP_EDGE_B,
	SEP_FACE_B,
	SEP_EDGES,
	SEP_NONE
};

// b3SeparationFunction (time_of_impact.cpp:26-461).
struct Separation
{
	const GProxy* pA;
	const GProxy* pB;
	const Sweep* sA;
	const Sweep* sB;
	uint32_t type;
	V3 localPoint, axis;
	bool parallel;

	__device__ __noinline__ void init(const GJKCache& cache, float t1)
	{
		const XF xfA = sweep_at(*sA, t1), xfB = sweep_at(*sB, t1);
		const FeaturePair fp = feature_pair(cache);
		const uint32_t countA = fp.count1, countB = fp.count2;
		parallel = false;
		localPoint = V3{0.0f, 0.0f, 0.0f};
		type = SEP_NONE;
		if (countA == 1 && countB == 1)
		{
			type = SEP_POINTS;
			const V3 A = xmul(xfA, gp_vertex(*pA, fp.index1[0]));
			const V3 B = xmul(xfB, gp_vertex(*pB, fp.index2[0]));
			axis = B - A;
			normalize_inplace(axis);
		}
		else if (countA == 2 && countB == 1)
		{
			type = SEP_EDGE_A;
			const V3 A = gp_vertex(*pA, fp.index1[0]);
			const V3 B = gp_vertex(*pA, fp.index1[1]);
			const V3 C = xmult(xfA, xmul(xfB, gp_vertex(*pB, fp.index2[0])));
			const V3 AB = B - A, AC = C - A;
			const V3 PC = cross(cross(AB, AC), AB);
			axis = rot(xfA.q, PC);
			normalize_inplace(axis);
		}
		else if (countA == 3)
		{
			type = SEP_FACE_A;
			const V3 A = gp_vertex(*pA, fp.index1[0]);
			const V3 B = gp_vertex(*pA, fp.index1[1]);
			const V3 C = gp_vertex(*pA, fp.index1[2]);
			const V3 D = xmult(xfA, xmul(xfB, gp_vertex(*pB, fp.index2[0])));
			V3 N = -cross(B - A, C - A);
			if (dot(D - A, N) < 0.0f)
				N = -N;
			axis = N;
			normalize_inplace(axis);
			localPoint = A;
		}
		else if (countB == 2 && countA == 1)
		{
			type = SEP_EDGE_B;
			const V3 A = gp_vertex(*pB, fp.index2[0]);
			const V3 B = gp_vertex(*pB, fp.index2[1]);
			const V3 C = xmult(xfB, xmul(xfA, gp_vertex(*pA, fp.index1[0])));
			const V3 AB = B - A, AC = C - A;
			const V3 PC = cross(cross(AB, AC), AB);
			axis = rot(xfB.q, PC);
			normalize_inplace(axis);
		}
		else if (countB == 3)
		{
			type = SEP_FACE_B;
			const V3 A = gp_vertex(*pB, fp.index2[0]);
			const V3 B = gp_vertex(*pB, fp.index2[1]);
			const V3 C = gp_vertex(*pB, fp.index2[2]);
			const V3 D = xmult(xfB, xmul(xfA, gp_vertex(*pA, fp.index1[0])));
			V3 N = -cross(B - A, C - A);
			if (dot(D - A, N) < 0.0f)
				N = -N;
			axis = N;
			normalize_inplace(axis);
			localPoint = A;
		}
		else if (countA == 2 && countB == 2)
		{
			type = SEP_EDGES;
			const V3 A = gp_vertex(*pA, fp.index1[0]);
			const V3 B = gp_vertex(*pA, fp.index1[1]);
			const V3 C = xmult(xfA, xmul(xfB, gp_vertex(*pB, fp.index2[0])));
			const V3 D = xmult(xfA, xmul(xfB, gp_vertex(*pB, fp.index2[1])));
			const V3 E1 = B - A, E2 = D - C;
			const float L1 = len(E1), L2 = len(E2);
			const float kTol = 0.005f;
			const V3 E1_x_E2 = cross(E1, E2);
			const float L = len(E1_x_E2);
			if (L < (kTol * L1) * L2)
			{
				// Parallel edges: the closest points of the segments.
				V3 C1, C2;
				closest_on_segments(C1, C2, A, B, C, D);
				C1 = xmul(xfA, C1);
				C2 = xmul(xfA, C2);
				axis = C2 - C1;
				normalize_inplace(axis);
				parallel = true;
				return;
			}
			const V3 C1 = 0.5f * (A + B);
			const V3 C2 = 0.5f * (C + D);
			V3 N = (1.0f / L) * E1_x_E2;
			if (dot(N, C2 - C1) < 0.0f)
				N = -N;
			axis = N;
			localPoint = C1;
		}
	}

	__device__ __noinline__ float find_min(uint32_t& indexA, uint32_t& indexB, float t) const
	{
		const XF xfA = sweep_at(*sA, t), xfB = sweep_at(*sB, t);
		switch (type)
		{
		case SEP_POINTS:
		case SEP_EDGE_A:
		{
			indexA = gp_support(*pA, rotc(xfA.q, axis));
			indexB = gp_support(*pB, rotc(xfB.q, -axis));
			const V3 A = xmul(xfA, gp_vertex(*pA, indexA));
			const V3 B = xmul(xfB, gp_vertex(*pB, indexB));
			return dot(B - A, axis);
		}
		case SEP_FACE_A:
		{
			const V3 N = rot(xfA.q, axis);
			const V3 A = xmul(xfA, localPoint);
			indexA = B3G_NULL;
			indexB = gp_support(*pB, rotc(xfB.q, -N));
			const V3 B = xmul(xfB, gp_vertex(*pB, indexB));
			return dot(B - A, N);
		}
		case SEP_EDGE_B:
		{
			indexA = gp_support(*pA, rotc(xfA.q, -axis));
			indexB = gp_support(*pB, rotc(xfB.q, axis));
			const V3 A = xmul(xfA, gp_vertex(*pA, indexA));
			const V3 B = xmul(xfB, gp_vertex(*pB, indexB));
			return dot(A - B, axis);
		}
		case SEP_FACE_B:
		{
			const V3 N = rot(xfB.q, axis);
			const V3 B = xmul(xfB, localPoint);
			indexA = gp_support(*pA, rotc(xfA.q, -N));
			indexB = B3G_NULL;
			const V3 A = xmul(xfA, gp_vertex(*pA, indexA));
			return dot(A - B, N);
		}
		case SEP_EDGES:
		{
			if (parallel)
			{
				indexA = gp_support(*pA, rotc(xfA.q, axis));
				indexB = gp_support(*pB, rotc(xfB.q, -axis));
				const V3 A = xmul(xfA, gp_vertex(*pA, indexA));
				const V3 B = xmul(xfB, gp_vertex(*pB, indexB));
				return dot(B - A, axis);
			}
			const V3 N = rot(xfA.q, axis);
			const V3 A = xmul(xfA, localPoint);
			indexA = B3G_NULL;
			indexB = gp_support(*pB, rotc(xfB.q, -N));
			const V3 B = xmul(xfB, gp_vertex(*pB, indexB));
			return dot(B - A, N);
		}
		default:
			indexA = indexB = B3G_NULL;
			return -B3G_MAX_SCALAR;
		}
	}

	__device__ __noinline__ float evaluate(uint32_t indexA, uint32_t indexB, float t) const
	{
		const XF xfA = sweep_at(*sA, t), xfB = sweep_at(*sB, t);
		switch (type)
		{
		case SEP_POINTS:
		case SEP_EDGE_A:
			return dot(xmul(xfB, gp_vertex(*pB, indexB)) - xmul(xfA, gp_vertex(*pA, indexA)), axis);
		case SEP_FACE_A:
		{
			const V3 N = rot(xfA.q, axis);
			const V3 A = xmul(xfA, localPoint);
			return dot(xmul(xfB, gp_vertex(*pB, indexB)) - A, N);
		}
		case SEP_EDGE_B:
			return dot(xmul(xfA, gp_vertex(*pA, indexA)) - xmul(xfB, gp_vertex(*pB, indexB)), axis);
		case SEP_FACE_B:
		{
			const V3 N = rot(xfB.q, axis);
			const V3 B = xmul(xfB, localPoint);
			return dot(xmul(xfA, gp_vertex(*pA, indexA)) - B, N);
		}
		case SEP_EDGES:
		{
			if (parallel)
				return dot(xmul(xfB, gp_vertex(*pB, indexB)) - xmul(xfA, gp_vertex(*pA, indexA)), axis);
			const V3 N = rot(xfA.q, axis);
			const V3 A = xmul(xfA, localPoint);
			return dot(xmul(xfB, gp_vertex(*pB, indexB)) - A, N);
		}
		default:
			return 0.0f;
		}
	}
};

// b3TOIOutput::State (time_of_impact.h:40-47).
enum : uint32_t
{
	ST_UNKNOWN = 0,
	ST_FAILED,
	ST_OVERLAPPED,
	ST_TOUCHING,
	ST_SEPARATED
};

// b3TimeOfImpact(const b3TOIInput&) (time_of_impact.cpp:465-660). A feature
// pair the reference asserts never happens ends the query as failed.
__device__ void toi_sweeps(const GProxy& pA, const Sweep& sA, const GProxy& pB, const Sweep& sB, float tMax,
	uint32_t& state, float& tOut, uint32_t& iterations)
{
	state = ST_UNKNOWN;
	tOut = tMax;
	const float totalRadius = pA.radius + pB.radius;
	const float target = fmaxr(B3G_LINEAR_SLOP, totalRadius - 3.0f * B3G_LINEAR_SLOP);
	const float tolerance = 0.25f * B3G_LINEAR_SLOP;
	float t1 = 0.0f;
	const uint32_t kMaxIterations = 20;
	uint32_t iteration = 0;
	GJKCache cache;
	cache.count = 0;
	cache.metric = 0.0f;
	for (int k = 0; k < 4; ++k)
		cache.index1[k] = cache.index2[k] = 0u;
	for (;;)
	{
		const XF xfA = sweep_at(sA, t1), xfB = sweep_at(sB, t1);
		const GJKOut g = gjk_cached(xfA, pA, xfB, pB, cache);
		if (g.distance == 0.0f)
		{
			state = ST_OVERLAPPED;
			tOut = 0.0f;
			break;
		}
		if (g.distance < target + tolerance)
		{
			state = ST_TOUCHING;
			tOut = t1;
			break;
		}
		Separation fcn;
		fcn.pA = &pA;
		fcn.pB = &pB;
		fcn.sA = &sA;
		fcn.sB = &sB;
		fcn.init(cache, t1);
		if (fcn.type == SEP_NONE)
		{
			state = ST_FAILED;
			tOut = t1;
			break;
		}
		bool done = false;
		float t2 = tMax;
		uint32_t pushBackIter = 0;
		for (;;)
		{
			uint32_t indexA, indexB;
			float s2 = fcn.find_min(indexA, indexB, t2);
			if (s2 > target + tolerance)
			{
				state = ST_SEPARATED;
				tOut = tMax;
				done = true;
				break;
			}
			if (s2 > target - tolerance)
			{
				t1 = t2;
				break;
			}
			float s1 = fcn.evaluate(indexA, indexB, t1);
			if (s1 < target - tolerance)
			{
				state = ST_FAILED;
				tOut = t1;
				done = true;
				break;
			}
			if (s1 <= target + tolerance)
			{
				state = ST_TOUCHING;
				tOut = t1;
				done = true;
				break;
			}
			uint32_t rootIteration = 0;
			float a1 = t1, a2 = t2;
			for (;;)
			{
				float t;
				if (rootIteration & 1u)
					t = a1 + (target - s1) * (a2 - a1) / (s2 - s1);
				else
					t = 0.5f * (a1 + a2);
				++rootIteration;
				const float s = fcn.evaluate(indexA, indexB, t);
				if (fabsr(s - target) < tolerance)
				{
					t2 = t;
					break;
				}
				if (s > target)
				{
					a1 = t;
					s1 = s;
				}
				else
				{
					a2 = t;
					s2 = s;
				}
				if (rootIteration == 50u)
					break;
			}
			++pushBackIter;
			if (pushBackIter == 64u)
				break;
		}
		++iteration;
		if (done)
			break;
		if (iteration == kMaxIterations)
		{
			state = ST_FAILED;
			tOut = t1;
			break;
		}
	}
	iterations = iteration;
}

// b3TimeOfImpact(aabb1, d1, aabb2, d2) (time_of_impact.cpp:782-902).
__device__ void toi_aabbs(const float* in, uint32_t& state, float& tOut)
{
	const float aLo[3] = {in[0], in[1], in[2]}, aHi[3] = {in[3], in[4], in[5]};
	const float d1[3] = {in[6], in[7], in[8]};
	const float bLo[3] = {in[9], in[10], in[11]}, bHi[3] = {in[12], in[13], in[14]};
	const float d2[3] = {in[15], in[16], in[17]};
	AABB A, B;
	A.lo = V3{aLo[0], aLo[1], aLo[2]};
	A.hi = V3{aHi[0], aHi[1], aHi[2]};
	B.lo = V3{bLo[0], bLo[1], bLo[2]};
	B.hi = V3{bHi[0], bHi[1], bHi[2]};
	if (aabb_overlap(A, B))
	{
		state = ST_OVERLAPPED;
		tOut = 0.0f;
		return;
	}
	float t1[3] = {0.0f, 0.0f, 0.0f}, t2[3] = {1.0f, 1.0f, 1.0f};
	for (int i = 0; i < 3; ++i)
	{
		const float d = d2[i] - d1[i];
		if (d == 0.0f && (aLo[i] > bHi[i] || aHi[i] < bLo[i]))
		{
			state = ST_SEPARATED;
			tOut = 1.0f;
			return;
		}
		if (d < 0.0f)
		{
			if (bHi[i] < aLo[i])
			{
				state = ST_SEPARATED;
				tOut = 1.0f;
				return;
			}
			t2[i] = (aLo[i] - bHi[i]) / d;
			if (bLo[i] > aHi[i])
			{
				t1[i] = (aHi[i] - bLo[i]) / d;
				if (t1[i] >= 1.0f)
				{
					state = ST_SEPARATED;
					tOut = 1.0f;
					return;
				}
			}
		}
		if (d > 0.0f)
		{
			if (bLo[i] > aHi[i])
			{
				state = ST_SEPARATED;
				tOut = 1.0f;
				return;
			}
			t2[i] = (aHi[i] - bLo[i]) / d;
			if (bHi[i] < aLo[i])
			{
				t1[i] = (aLo[i] - bHi[i]) / d;
				if (t1[i] >= 1.0f)
				{
					state = ST_SEPARATED;
					tOut = 1.0f;
					return;
				}
			}
		}
	}
	const float t1max = fmaxr(t1[0], fmaxr(t1[1], t1[2]));
	const float t2min = fminr(t2[0], fminr(t2[1], t2[2]));
	if (t1max > t2min)
	{
		state = ST_SEPARATED;
		tOut = 0.0f;
		return;
	}
	state = ST_TOUCHING;
	tOut = t1max;
}

// b3ShapeCast (gjk.cpp:938-1102): GJK ray cast of proxy 2 along r against
// proxy 1 (radii included). Returns false when they do not meet within r.
__device__ bool gjk_ray_cast(const XF& xf1, const GProxy& p1, const XF& xf2, const GProxy& p2, V3 r, float& tOut,
	V3& point, V3& normalOut, uint32_t& iterations)
{
	const float r1 = p1.radius, r2 = p2.radius;
	const float radius = r1 + r2;
	float t = 0.0f;
	V3 n = V3{0.0f, 0.0f, 0.0f};
	uint32_t index1 = gp_support(p1, rotc(xf1.q, -r));
	uint32_t index2 = gp_support(p2, rotc(xf2.q, r));
	V3 w1 = xmul(xf1, gp_vertex(p1, index1));
	V3 w2 = xmul(xf2, gp_vertex(p2, index2));
	V3 v = w1 - w2;
	Simplex sx;
	sx.count = 0;
	for (int i = 0; i < 4; ++i)
	{
		sx.v[i].point1 = sx.v[i].point2 = sx.v[i].point = V3{0.0f, 0.0f, 0.0f};
		sx.v[i].weight = 0.0f;
		sx.v[i].index1 = sx.v[i].index2 = 0u;
	}
	uint32_t save1[4], save2[4];
	uint32_t saveCount = 0;
	const uint32_t kMaxIters = 20;
	const float kTolerance = 10.0f * B3G_EPSILON;
	float maxTolerance = 1.0f;
	uint32_t iter = 0;
	while (iter < kMaxIters && fabsr(len2(v) - radius * radius) > kTolerance * maxTolerance)
	{
		index1 = gp_support(p1, rotc(xf1.q, -v));
		index2 = gp_support(p2, rotc(xf2.q, v));
		w1 = xmul(xf1, gp_vertex(p1, index1));
		w2 = xmul(xf2, gp_vertex(p2, index2));
		const V3 p = w1 - w2;
		const float vp = dot(v, p);
		const float vr = dot(v, r);
		if (vp - radius > t * vr)
		{
			if (vr > 0.0f)
			{
				t = (vp - radius) / vr;
				if (t > 1.0f)
				{
					iterations = iter;
					return false;
				}
				n = -v;
				sx.count = 0;
				saveCount = 0;
			}
			else
			{
				iterations = iter;
				return false;
			}
		}
		const V3 s = t * r;
		SVert vx;
		vx.index1 = index1;
		vx.point1 = w1;
		vx.index2 = index2;
		vx.point2 = w2;
		vx.point = p - s;
		vx.weight = 0.0f;
		bool duplicate = false;
		for (uint32_t i = 0; i < 4; ++i)
			if (i < saveCount && vx.index1 == save1[i] && vx.index2 == save2[i])
				duplicate = true;
		if (duplicate)
			break;
		if (sx.count == 0)
			sx.v[0] = vx;
		else if (sx.count == 1)
			sx.v[1] = vx;
		else if (sx.count == 2)
			sx.v[2] = vx;
		else
			sx.v[3] = vx;
		++sx.count;
		maxTolerance = -B3G_EPSILON;
#pragma unroll
		for (int i = 0; i < 4; ++i)
			if ((uint32_t)i < sx.count)
				maxTolerance = fmaxr(maxTolerance, len2(sx.v[i].point));
		saveCount = sx.count;
#pragma unroll
		for (int i = 0; i < 4; ++i)
		{
			save1[i] = sx.v[i].index1;
			save2[i] = sx.v[i].index2;
		}
		if (sx.count == 2)
			sx.solve2();
		else if (sx.count == 3)
			sx.solve3();
		else if (sx.count == 4)
			sx.solve4();
		if (sx.count == 4)
			break;
		v = sx.closest();
		++iter;
	}
	V3 point1, point2;
	sx.closest_points(point1, point2);
	if (len2(v) > B3G_EPSILON * B3G_EPSILON)
		n = -v;
	normalize_inplace(n);
	tOut = t;
	point = point1 + r1 * n;
	normalOut = n;
	iterations = iter;
	return true;
}

__device__ __forceinline__ GProxy input_proxy(const DevScene& S, const float* w, uint32_t type, uint32_t hull)
{
	return convex_proxy(S, type, make_float4(w[0], w[1], w[2], w[3]), make_float4(w[4], w[5], w[6], w[7]),
		make_float4(w[8], w[9], w[10], w[11]), hull);
}

__global__ void k_toi_sweeps(DevScene S, const float* in, uint32_t n, uint32_t* out)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const float* r = in + 68 * (size_t)i;
	const uint32_t typeA = __float_as_uint(r[0]), hullA = __float_as_uint(r[1]);
	const uint32_t typeB = __float_as_uint(r[2]), hullB = __float_as_uint(r[3]);
	const GProxy pA = input_proxy(S, r + 4, typeA, hullA);
	const GProxy pB = input_proxy(S, r + 16, typeB, hullB);
	const Sweep sA = load_sweep(r + 28), sB = load_sweep(r + 46);
	uint32_t state, iterations;
	float t;
	toi_sweeps(pA, sA, pB, sB, r[64], state, t, iterations);
	out[4 * (size_t)i] = state;
	out[4 * (size_t)i + 1] = __float_as_uint(t);
	out[4 * (size_t)i + 2] = iterations;
	out[4 * (size_t)i + 3] = 0;
}

__global__ void k_toi_aabbs(const float* in, uint32_t n, uint32_t* out)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	uint32_t state;
	float t;
	toi_aabbs(in + 18 * (size_t)i, state, t);
	out[4 * (size_t)i] = state;
	out[4 * (size_t)i + 1] = __float_as_uint(t);
	out[4 * (size_t)i + 2] = 0;
	out[4 * (size_t)i + 3] = 0;
}

__global__ void k_gjk_ray_cast(DevScene S, const float* in, uint32_t n, float* out)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const float* r = in + 48 * (size_t)i;
	const uint32_t typeA = __float_as_uint(r[0]), hullA = __float_as_uint(r[1]);
	const uint32_t typeB = __float_as_uint(r[2]), hullB = __float_as_uint(r[3]);
	const GProxy pA = input_proxy(S, r + 4, typeA, hullA);
	const GProxy pB = input_proxy(S, r + 16, typeB, hullB);
	XF xfA, xfB;
	xfA.p = V3{r[28], r[29], r[30]};
	xfA.q = Q4{V3{r[31], r[32], r[33]}, r[34]};
	xfB.p = V3{r[35], r[36], r[37]};
	xfB.q = Q4{V3{r[38], r[39], r[40]}, r[41]};
	const V3 tr = V3{r[42], r[43], r[44]};
	float t = 0.0f;
	V3 point = V3{0.0f, 0.0f, 0.0f}, normal = V3{0.0f, 0.0f, 0.0f};
	uint32_t iterations = 0;
	const bool hit = gjk_ray_cast(xfA, pA, xfB, pB, tr, t, point, normal, iterations);
	float* o = out + 9 * (size_t)i;
	o[0] = __uint_as_float(hit ? 1u : 0u);
	o[1] = hit ? t : 0.0f;
	o[2] = hit ? point.x : 0.0f;
	o[3] = hit ? point.y : 0.0f;
	o[4] = hit ? point.z : 0.0f;
	o[5] = hit ? normal.x : 0.0f;
	o[6] = hit ? normal.y : 0.0f;
	o[7] = hit ? normal.z : 0.0f;
	o[8] = __uint_as_float(iterations);
}

int tfail(b3g_ctx* c, int code, const char* msg)
{
	c->err = msg;
	return code;
}

// Copies n records of `bytes` each in, runs the launch, copies `outBytes`
// per record out (synchronous, on the context's stream). The device copies
// live in the context's scratch, grown on demand.
template <class Launch>
int run_batch(b3g_ctx* c, uint32_t n, const void* in, size_t bytes, void* out, size_t outBytes, Launch&& launch)
{
	if (n == 0)
		return 0;
	if (cudaSetDevice(c->device) != cudaSuccess)
		return tfail(c, B3G_E_CUDA, "time of impact: device");
	const size_t inBytes = (bytes * n + 255) & ~(size_t)255;
	const size_t need = inBytes + outBytes * n;
	if (c->toiScratchBytes < need)
	{
		if (c->toiScratch && cudaFree(c->toiScratch) != cudaSuccess)
			return tfail(c, B3G_E_CUDA, "time of impact: device free failed");
		c->toiScratch = nullptr;
		c->toiScratchBytes = 0;
		if (cudaMalloc(&c->toiScratch, need) != cudaSuccess)
			return tfail(c, B3G_E_CUDA, "time of impact: device allocation failed");
		c->toiScratchBytes = need;
	}
	void* dIn = c->toiScratch;
	void* dOut = (char*)c->toiScratch + inBytes;
	if (cudaMemcpyAsync(dIn, in, bytes * n, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
		return tfail(c, B3G_E_CUDA, "time of impact: copy");
	launch((const float*)dIn, dOut, c->stream);
	if (cudaGetLastError() != cudaSuccess ||
		cudaMemcpyAsync(out, dOut, outBytes * n, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
		cudaStreamSynchronize(c->stream) != cudaSuccess)
		return tfail(c, B3G_E_CUDA, "time of impact: kernel or copy failed");
	return (int)n;
}

// Shape types and hulls of a query's two proxies: convex types only.
bool proxies_ok(const b3g_ctx* c, uint32_t typeA, uint32_t hullA, uint32_t typeB, uint32_t hullB)
{
	auto ok = [&](uint32_t t, uint32_t h) { return t < B3G_SHAPE_MESH && (t != B3G_SHAPE_HULL || h < c->nHulls); };
	return ok(typeA, hullA) && ok(typeB, hullB);
}

} // namespace

extern "C" int b3g_time_of_impact(b3g_ctx* c, uint32_t n, const b3g_toi_input* in, uint32_t* out)
{
	if (!c || (n && (!in || !out)))
		return c ? tfail(c, B3G_E_INVALID, "b3g_time_of_impact: null argument") : B3G_E_INVALID;
	for (uint32_t i = 0; i < n; ++i)
		if (!proxies_ok(c, in[i].type_a, in[i].hull_a, in[i].type_b, in[i].hull_b))
			return tfail(c, B3G_E_INVALID, "b3g_time_of_impact: shape type or hull out of range");
	const DevScene S = c->scene;
	return run_batch(c, n, in, sizeof(b3g_toi_input), out, 16, [&](const float* dIn, void* dOut, cudaStream_t s) {
		k_toi_sweeps<<<(n + 127) / 128, 128, 0, s>>>(S, dIn, n, (uint32_t*)dOut);
	});
}

extern "C" int b3g_time_of_impact_device(b3g_ctx* c, uint32_t n, const b3g_toi_input* in, uint32_t* out,
	void* stream)
{
	if (!c || (n && (!in || !out)))
		return c ? tfail(c, B3G_E_INVALID, "b3g_time_of_impact_device: null argument") : B3G_E_INVALID;
	if (n == 0)
		return B3G_OK;
	if (cudaSetDevice(c->device) != cudaSuccess)
		return tfail(c, B3G_E_CUDA, "time of impact: device");
	cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
	k_toi_sweeps<<<(n + 127) / 128, 128, 0, s>>>(c->scene, (const float*)in, n, out);
	if (cudaGetLastError() != cudaSuccess)
		return tfail(c, B3G_E_CUDA, "b3g_time_of_impact_device: launch");
	return B3G_OK;
}

extern "C" int b3g_time_of_impact_aabb(b3g_ctx* c, uint32_t n, const float* in, uint32_t* out)
{
	if (!c || (n && (!in || !out)))
		return c ? tfail(c, B3G_E_INVALID, "b3g_time_of_impact_aabb: null argument") : B3G_E_INVALID;
	return run_batch(c, n, in, 18 * sizeof(float), out, 16, [&](const float* dIn, void* dOut, cudaStream_t s) {
		k_toi_aabbs<<<(n + 127) / 128, 128, 0, s>>>(dIn, n, (uint32_t*)dOut);
	});
}

extern "C" int b3g_gjk_shape_cast(b3g_ctx* c, uint32_t n, const b3g_gjk_cast_input* in, float* out)
{
	if (!c || (n && (!in || !out)))
		return c ? tfail(c, B3G_E_INVALID, "b3g_gjk_shape_cast: null argument") : B3G_E_INVALID;
	for (uint32_t i = 0; i < n; ++i)
		if (!proxies_ok(c, in[i].type_a, in[i].hull_a, in[i].type_b, in[i].hull_b))
			return tfail(c, B3G_E_INVALID, "b3g_gjk_shape_cast: shape type or hull out of range");
	const DevScene S = c->scene;
	return run_batch(c, n, in, sizeof(b3g_gjk_cast_input), out, 36, [&](const float* dIn, void* dOut, cudaStream_t s) {
		k_gjk_ray_cast<<<(n + 127) / 128, 128, 0, s>>>(S, dIn, n, (float*)dOut);
	});
}

// Device GJK distance (Voronoi regions + barycentric coordinates), the
// algorithm of src/bounce/collision/gjk/gjk.cpp:276-812 evaluated with the
// same operation order: Solve2 / Solve3 / Solve4 region tests, the search
// direction of each simplex size, at most 20 support iterations, the
// duplicate-support exit, and the optional radius application. The simplex
// cache is always empty on the narrowphase paths (b3GJK(..., applyRadius) at
// gjk.cpp:1104-1110), so only the arbitrary one-vertex start is needed.
#pragma once

#include "b3g_math.cuh"

struct GProxy
{
	const float4* gv; // global vertices (hulls) or nullptr
	V3 lv[3];         // local vertices (sphere, capsule, triangle)
	uint32_t count;
	float radius;
};

__device__ __forceinline__ V3 gp_vertex(const GProxy& p, uint32_t i)
{
	if (p.gv)
	{
		float4 w = p.gv[i];
		return V3{w.x, w.y, w.z};
	}
	return i == 0 ? p.lv[0] : (i == 1 ? p.lv[1] : p.lv[2]);
}

// b3GJKProxy::GetSupportIndex (gjk_proxy.h:72-86): first maximum.
__device__ __forceinline__ uint32_t gp_support(const GProxy& p, V3 d)
{
	uint32_t maxIndex = 0;
	float maxProj = dot(d, gp_vertex(p, 0));
	for (uint32_t i = 1; i < p.count; ++i)
	{
		float proj = dot(d, gp_vertex(p, i));
		if (proj > maxProj)
		{
			maxIndex = i;
			maxProj = proj;
		}
	}
	return maxIndex;
}

struct SVert
{
	V3 point1, point2, point;
	float weight;
	uint32_t index1, index2;
};

struct GJKOut
{
	V3 point1, point2;
	float distance;
	uint32_t iterations;
};

// The final simplex's support indices (b3Simplex::WriteCache, gjk.cpp:870-878).
struct GJKSimplexOut
{
	uint32_t count;
	uint32_t index1[4], index2[4];
};

// b3Barycentric (gjk.cpp:99-113): divisor = u + v.
__device__ __forceinline__ void bary2(float out[3], V3 A, V3 B, V3 Q)
{
	V3 AB = B - A;
	V3 QA = A - Q;
	V3 QB = B - Q;
	out[0] = dot(QB, AB);
	out[1] = -dot(QA, AB);
	out[2] = out[0] + out[1];
}

// (gjk.cpp:115-139): divisor = u + v + w.
__device__ __forceinline__ void bary3(float out[4], V3 A, V3 B, V3 C, V3 Q)
{
	V3 AB = B - A;
	V3 AC = C - A;
	V3 QA = A - Q;
	V3 QB = B - Q;
	V3 QC = C - Q;
	V3 QB_x_QC = cross(QB, QC);
	V3 QC_x_QA = cross(QC, QA);
	V3 QA_x_QB = cross(QA, QB);
	V3 AB_x_AC = cross(AB, AC);
	out[0] = dot(QB_x_QC, AB_x_AC);
	out[1] = dot(QC_x_QA, AB_x_AC);
	out[2] = dot(QA_x_QB, AB_x_AC);
	out[3] = (out[0] + out[1]) + out[2];
}

__device__ __forceinline__ float det3(V3 a, V3 b, V3 c) { return dot(a, cross(b, c)); }
__device__ __forceinline__ float signf_(float x) { return (float)(0.0f < x) - (float)(x < 0.0f); }

// (gjk.cpp:141-166).
__device__ __forceinline__ void bary4(float out[5], V3 A, V3 B, V3 C, V3 D, V3 Q)
{
	V3 AB = B - A;
	V3 AC = C - A;
	V3 AD = D - A;
	V3 QA = A - Q;
	V3 QB = B - Q;
	V3 QC = C - Q;
	V3 QD = D - Q;
	float divisor = det3(AB, AC, AD);
	float sign = signf_(divisor);
	out[0] = sign * det3(QB, QC, QD);
	out[1] = sign * det3(QA, QD, QC);
	out[2] = sign * det3(QA, QB, QD);
	out[3] = sign * det3(QA, QC, QB);
	out[4] = sign * divisor;
}

struct Simplex
{
	SVert v[4];
	uint32_t count;

	__device__ V3 search_dir() const
	{
		// Q = origin.
		const V3 Q = V3{0.0f, 0.0f, 0.0f};
		if (count == 1)
			return Q - v[0].point;
		if (count == 2)
		{
			V3 A = v[0].point, B = v[1].point;
			V3 AB = B - A;
			V3 AQ = Q - A;
			V3 AB_x_AQ = cross(AB, AQ);
			return cross(AB_x_AQ, AB);
		}
		if (count == 3)
		{
			V3 A = v[0].point, B = v[1].point, C = v[2].point;
			V3 AB = B - A;
			V3 AC = C - A;
			V3 AQ = Q - A;
			V3 AB_x_AC = cross(AB, AC);
			float sign = dot(AB_x_AC, AQ);
			if (sign > 0.0f)
				return AB_x_AC;
			return -AB_x_AC;
		}
		return V3{0.0f, 0.0f, 0.0f};
	}

	__device__ V3 closest() const
	{
		if (count == 1)
			return v[0].point;
		if (count == 2)
			return v[0].weight * v[0].point + v[1].weight * v[1].point;
		if (count == 3)
			return (v[0].weight * v[0].point + v[1].weight * v[1].point) + v[2].weight * v[2].point;
		return V3{0.0f, 0.0f, 0.0f};
	}

	__device__ void closest_points(V3& p1, V3& p2) const
	{
		if (count == 1)
		{
			p1 = v[0].point1;
			p2 = v[0].point2;
		}
		else if (count == 2)
		{
			p1 = v[0].weight * v[0].point1 + v[1].weight * v[1].point1;
			p2 = v[0].weight * v[0].point2 + v[1].weight * v[1].point2;
		}
		else if (count == 3)
		{
			p1 = (v[0].weight * v[0].point1 + v[1].weight * v[1].point1) + v[2].weight * v[2].point1;
			p2 = (v[0].weight * v[0].point2 + v[1].weight * v[1].point2) + v[2].weight * v[2].point2;
		}
		else if (count == 4)
		{
			p1 = ((v[0].weight * v[0].point1 + v[1].weight * v[1].point1) + v[2].weight * v[2].point1) +
				v[3].weight * v[3].point1;
			p2 = p1;
		}
	}

	// closest_points with the witness points recomputed from the support
	// indices, by the same expressions that made them when each vertex
	// joined the simplex (the same bits): the simplex then carries no
	// witness points through the loop, and the registers they would hold
	// stay free.
	__device__ void closest_points_from(const XF& xf1, const GProxy& p1, const XF& xf2, const GProxy& p2, V3& P1,
		V3& P2) const;

	__device__ void set1(const SVert& a)
	{
		count = 1;
		v[0] = a;
		v[0].weight = 1.0f;
	}
	__device__ void set2(const SVert& a, float wa, const SVert& b, float wb)
	{
		count = 2;
		v[0] = a;
		v[0].weight = wa;
		v[1] = b;
		v[1].weight = wb;
	}
	__device__ void set3(const SVert& a, float wa, const SVert& b, float wb, const SVert& c, float wc)
	{
		count = 3;
		v[0] = a;
		v[0].weight = wa;
		v[1] = b;
		v[1].weight = wb;
		v[2] = c;
		v[2].weight = wc;
	}

	// (gjk.cpp:276-308)
	__device__ void solve2()
	{
		const V3 Q = V3{0.0f, 0.0f, 0.0f};
		SVert A = v[0], B = v[1];
		float wAB[3];
		bary2(wAB, A.point, B.point, Q);
		if (wAB[1] <= 0.0f)
		{
			set1(A);
			return;
		}
		if (wAB[0] <= 0.0f)
		{
			set1(B);
			return;
		}
		float s = 1.0f / wAB[2];
		set2(A, s * wAB[0], B, s * wAB[1]);
	}

	// (gjk.cpp:312-412)
	__device__ void solve3()
	{
		const V3 Q = V3{0.0f, 0.0f, 0.0f};
		SVert A = v[0], B = v[1], C = v[2];
		float wAB[3], wBC[3], wCA[3];
		bary2(wAB, A.point, B.point, Q);
		bary2(wBC, B.point, C.point, Q);
		bary2(wCA, C.point, A.point, Q);
		if (wAB[1] <= 0.0f && wCA[0] <= 0.0f)
		{
			set1(A);
			return;
		}
		if (wAB[0] <= 0.0f && wBC[1] <= 0.0f)
		{
			set1(B);
			return;
		}
		if (wBC[0] <= 0.0f && wCA[1] <= 0.0f)
		{
			set1(C);
			return;
		}
		float wABC[4];
		bary3(wABC, A.point, B.point, C.point, Q);
		float area = wABC[3];
		if (wAB[0] > 0.0f && wAB[1] > 0.0f && area * wABC[2] <= 0.0f)
		{
			float s = 1.0f / wAB[2];
			set2(A, s * wAB[0], B, s * wAB[1]);
			return;
		}
		if (wBC[0] > 0.0f && wBC[1] > 0.0f && area * wABC[0] <= 0.0f)
		{
			float s = 1.0f / wBC[2];
			set2(B, s * wBC[0], C, s * wBC[1]);
			return;
		}
		if (wCA[0] > 0.0f && wCA[1] > 0.0f && area * wABC[1] <= 0.0f)
		{
			float s = 1.0f / wCA[2];
			set2(C, s * wCA[0], A, s * wCA[1]);
			return;
		}
		float divisor = wABC[3];
		if (divisor <= 0.0f)
			return;
		float s = 1.0f / divisor;
		set3(A, s * wABC[0], B, s * wABC[1], C, s * wABC[2]);
	}

	// (gjk.cpp:416-650)
	__device__ void solve4()
	{
		const V3 Q = V3{0.0f, 0.0f, 0.0f};
		SVert A = v[0], B = v[1], C = v[2], D = v[3];
		float wAB[3], wAC[3], wAD[3], wBC[3], wCD[3], wDB[3];
		bary2(wAB, A.point, B.point, Q);
		bary2(wBC, B.point, C.point, Q);
		bary2(wAC, A.point, C.point, Q);
		bary2(wAD, A.point, D.point, Q);
		bary2(wCD, C.point, D.point, Q);
		bary2(wDB, D.point, B.point, Q);
		if (wAB[1] <= 0.0f && wAC[1] <= 0.0f && wAD[1] <= 0.0f)
		{
			set1(A);
			return;
		}
		if (wAB[0] <= 0.0f && wDB[0] <= 0.0f && wBC[1] <= 0.0f)
		{
			set1(B);
			return;
		}
		if (wAC[0] <= 0.0f && wBC[0] <= 0.0f && wCD[1] <= 0.0f)
		{
			set1(C);
			return;
		}
		if (wAD[0] <= 0.0f && wCD[0] <= 0.0f && wDB[1] <= 0.0f)
		{
			set1(D);
			return;
		}
		float wACB[4], wABD[4], wADC[4], wBCD[4];
		bary3(wACB, A.point, C.point, B.point, Q);
		bary3(wABD, A.point, B.point, D.point, Q);
		bary3(wADC, A.point, D.point, C.point, Q);
		bary3(wBCD, B.point, C.point, D.point, Q);
		if (wABD[2] <= 0.0f && wACB[1] <= 0.0f && wAB[0] > 0.0f && wAB[1] > 0.0f)
		{
			float s = 1.0f / wAB[2];
			set2(A, s * wAB[0], B, s * wAB[1]);
			return;
		}
		if (wACB[2] <= 0.0f && wADC[1] <= 0.0f && wAC[0] > 0.0f && wAC[1] > 0.0f)
		{
			float s = 1.0f / wAC[2];
			set2(A, s * wAC[0], C, s * wAC[1]);
			return;
		}
		if (wADC[2] <= 0.0f && wABD[1] <= 0.0f && wAD[0] > 0.0f && wAD[1] > 0.0f)
		{
			float s = 1.0f / wAD[2];
			set2(A, s * wAD[0], D, s * wAD[1]);
			return;
		}
		if (wACB[0] <= 0.0f && wBCD[2] <= 0.0f && wBC[0] > 0.0f && wBC[1] > 0.0f)
		{
			float s = 1.0f / wBC[2];
			set2(B, s * wBC[0], C, s * wBC[1]);
			return;
		}
		if (wADC[0] <= 0.0f && wBCD[0] <= 0.0f && wCD[0] > 0.0f && wCD[1] > 0.0f)
		{
			float s = 1.0f / wCD[2];
			set2(C, s * wCD[0], D, s * wCD[1]);
			return;
		}
		if (wABD[0] <= 0.0f && wBCD[1] <= 0.0f && wDB[0] > 0.0f && wDB[1] > 0.0f)
		{
			float s = 1.0f / wDB[2];
			set2(D, s * wDB[0], B, s * wDB[1]);
			return;
		}
		float wABCD[5];
		bary4(wABCD, A.point, B.point, C.point, D.point, Q);
		if (wABCD[3] <= 0.0f && wACB[0] > 0.0f && wACB[1] > 0.0f && wACB[2] > 0.0f)
		{
			float s = 1.0f / ((wACB[0] + wACB[1]) + wACB[2]);
			set3(A, s * wACB[0], C, s * wACB[1], B, s * wACB[2]);
			return;
		}
		if (wABCD[2] <= 0.0f && wABD[0] > 0.0f && wABD[1] > 0.0f && wABD[2] > 0.0f)
		{
			float s = 1.0f / ((wABD[0] + wABD[1]) + wABD[2]);
			set3(A, s * wABD[0], B, s * wABD[1], D, s * wABD[2]);
			return;
		}
		if (wABCD[1] <= 0.0f && wADC[0] > 0.0f && wADC[1] > 0.0f && wADC[2] > 0.0f)
		{
			float s = 1.0f / ((wADC[0] + wADC[1]) + wADC[2]);
			set3(A, s * wADC[0], D, s * wADC[1], C, s * wADC[2]);
			return;
		}
		if (wABCD[0] <= 0.0f && wBCD[0] > 0.0f && wBCD[1] > 0.0f && wBCD[2] > 0.0f)
		{
			float s = 1.0f / ((wBCD[0] + wBCD[1]) + wBCD[2]);
			set3(B, s * wBCD[0], C, s * wBCD[1], D, s * wBCD[2]);
			return;
		}
		float divisor = ((wABCD[0] + wABCD[1]) + wABCD[2]) + wABCD[3];
		if (divisor <= 0.0f)
			return;
		float s = 1.0f / divisor;
		count = 4;
		v[0].weight = s * wABCD[0];
		v[1].weight = s * wABCD[1];
		v[2].weight = s * wABCD[2];
		v[3].weight = s * wABCD[3];
	}
};

__device__ __forceinline__ void Simplex::closest_points_from(const XF& xf1, const GProxy& p1, const XF& xf2,
	const GProxy& p2, V3& P1, V3& P2) const
{
	V3 a1[4], a2[4];
#pragma unroll
	for (int i = 0; i < 4; ++i)
	{
		if ((uint32_t)i < count)
		{
			a1[i] = xmul(xf1, gp_vertex(p1, v[i].index1));
			a2[i] = xmul(xf2, gp_vertex(p2, v[i].index2));
		}
		else
		{
			a1[i] = V3{0.0f, 0.0f, 0.0f};
			a2[i] = V3{0.0f, 0.0f, 0.0f};
		}
	}
	if (count == 1)
	{
		P1 = a1[0];
		P2 = a2[0];
	}
	else if (count == 2)
	{
		P1 = v[0].weight * a1[0] + v[1].weight * a1[1];
		P2 = v[0].weight * a2[0] + v[1].weight * a2[1];
	}
	else if (count == 3)
	{
		P1 = (v[0].weight * a1[0] + v[1].weight * a1[1]) + v[2].weight * a1[2];
		P2 = (v[0].weight * a2[0] + v[1].weight * a2[1]) + v[2].weight * a2[2];
	}
	else if (count == 4)
	{
		P1 = ((v[0].weight * a1[0] + v[1].weight * a1[1]) + v[2].weight * a1[2]) + v[3].weight * a1[3];
		P2 = P1;
	}
}

// The main loop of b3GJK (gjk.cpp:683-768) on an initialised simplex;
// returns the support iterations.
__device__ __forceinline__ uint32_t gjk_loop(Simplex& sx, const XF& xf1, const GProxy& p1, const XF& xf2,
	const GProxy& p2)
{
	uint32_t save1[4], save2[4];
	uint32_t saveCount = 0;
	const uint32_t kMaxIters = 20;
	uint32_t iter = 0;
	while (iter < kMaxIters)
	{
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
		V3 d = sx.search_dir();
		if (dot(d, d) < B3G_EPSILON * B3G_EPSILON)
			break;
		SVert vx;
		vx.index1 = gp_support(p1, rotc(xf1.q, -d));
		vx.point1 = xmul(xf1, gp_vertex(p1, vx.index1));
		vx.index2 = gp_support(p2, rotc(xf2.q, d));
		vx.point2 = xmul(xf2, gp_vertex(p2, vx.index2));
		vx.point = vx.point2 - vx.point1;
		vx.weight = 0.0f;
		++iter;
		bool duplicate = false;
#pragma unroll
		for (int i = 0; i < 4; ++i)
			if ((uint32_t)i < saveCount && vx.index1 == save1[i] && vx.index2 == save2[i])
				duplicate = true;
		if (duplicate)
			break;
		if (sx.count == 1)
			sx.v[1] = vx;
		else if (sx.count == 2)
			sx.v[2] = vx;
		else
			sx.v[3] = vx;
		++sx.count;
	}
	return iter;
}

// b3Simplex's arbitrary first vertex (gjk.cpp:855-867).
__device__ __forceinline__ void simplex_first(Simplex& sx, const XF& xf1, const GProxy& p1, const XF& xf2,
	const GProxy& p2)
{
	SVert& v = sx.v[0];
	v.point1 = xmul(xf1, gp_vertex(p1, 0));
	v.point2 = xmul(xf2, gp_vertex(p2, 0));
	v.point = v.point2 - v.point1;
	v.weight = 1.0f;
	v.index1 = 0;
	v.index2 = 0;
	sx.count = 1;
	// The simplex is indexed with constants only (unrolled loops, explicit
	// slot selection) so it stays in registers.
	for (int i = 1; i < 4; ++i)
		sx.v[i] = sx.v[0];
}

// b3GJK with an empty simplex cache (gjk.cpp:654-812 via :1104-1110).
__device__ inline GJKOut gjk(const XF& xf1, const GProxy& p1, const XF& xf2, const GProxy& p2, bool applyRadius,
	GJKSimplexOut* simplexOut = nullptr)
{
	Simplex sx;
	simplex_first(sx, xf1, p1, xf2, p2);
	uint32_t iter = gjk_loop(sx, xf1, p1, xf2, p2);
	if (simplexOut)
	{
		simplexOut->count = sx.count;
#pragma unroll
		for (int i = 0; i < 4; ++i)
		{
			simplexOut->index1[i] = sx.v[i].index1;
			simplexOut->index2[i] = sx.v[i].index2;
		}
	}
	GJKOut out;
	sx.closest_points_from(xf1, p1, xf2, p2, out.point1, out.point2);
	out.distance = len(out.point1 - out.point2);
	out.iterations = iter;
	if (applyRadius)
	{
		float r1 = p1.radius, r2 = p2.radius;
		if (out.distance > r1 + r2 && out.distance > B3G_EPSILON)
		{
			out.distance -= r1 + r2;
			V3 dd = out.point2 - out.point1;
			V3 normal = normalized(dd);
			out.point1 = out.point1 + r1 * normal;
			out.point2 = out.point2 - r2 * normal;
		}
		else
		{
			V3 p = 0.5f * (out.point1 + out.point2);
			out.point1 = p;
			out.point2 = p;
			out.distance = 0.0f;
		}
	}
	return out;
}

// b3SimplexCache (gjk.h): the support indices of the last simplex and its
// metric.
struct GJKCache
{
	uint32_t count;
	uint32_t index1[4], index2[4];
	float metric;
};

// b3Simplex::GetMetric (gjk.cpp:881-912).
__device__ __forceinline__ float simplex_metric(const Simplex& sx)
{
	if (sx.count == 2)
		return len(sx.v[0].point - sx.v[1].point);
	if (sx.count == 3)
		return len(cross(sx.v[1].point - sx.v[0].point, sx.v[2].point - sx.v[0].point));
	if (sx.count == 4)
	{
		V3 E1 = sx.v[1].point - sx.v[0].point;
		V3 E2 = sx.v[2].point - sx.v[0].point;
		V3 E3 = sx.v[3].point - sx.v[0].point;
		float det = det3(E1, E2, E3);
		return signf_(det) * det;
	}
	return 0.0f;
}

// b3GJK(xf1, proxy1, xf2, proxy2, false, &cache) (gjk.cpp:654-812): the
// simplex starts from the cache (b3Simplex::ReadCache, gjk.cpp:820-868: the
// cached support points with zero weights, flushed to the arbitrary vertex
// when their metric changed by more than a factor of two or vanished) and is
// written back to it (WriteCache, gjk.cpp:870-879). No radius is applied.
__device__ inline GJKOut gjk_cached(const XF& xf1, const GProxy& p1, const XF& xf2, const GProxy& p2, GJKCache& cache)
{
	Simplex sx;
	sx.count = cache.count;
	// Only the cached entries are read (their indices are support indices of
	// these proxies); the slots past them repeat slot 0.
#pragma unroll
	for (int i = 0; i < 4; ++i)
	{
		SVert& v = sx.v[i];
		if ((uint32_t)i < cache.count)
		{
			v.index1 = cache.index1[i];
			v.index2 = cache.index2[i];
			v.point1 = xmul(xf1, gp_vertex(p1, v.index1));
			v.point2 = xmul(xf2, gp_vertex(p2, v.index2));
			v.point = v.point2 - v.point1;
			v.weight = 0.0f;
		}
		else if (i > 0)
		{
			v = sx.v[0];
		}
	}
	if (sx.count > 1)
	{
		const float metric1 = cache.metric;
		const float metric2 = simplex_metric(sx);
		if (metric2 < 0.5f * metric1 || 2.0f * metric1 < metric2 || metric2 < B3G_EPSILON)
			sx.count = 0;
	}
	if (sx.count == 0)
		simplex_first(sx, xf1, p1, xf2, p2);
	GJKOut out;
	out.iterations = gjk_loop(sx, xf1, p1, xf2, p2);
	sx.closest_points_from(xf1, p1, xf2, p2, out.point1, out.point2);
	out.distance = len(out.point1 - out.point2);
	cache.metric = simplex_metric(sx);
	cache.count = sx.count;
#pragma unroll
	for (int i = 0; i < 4; ++i)
	{
		cache.index1[i] = sx.v[i].index1;
		cache.index2[i] = sx.v[i].index2;
	}
	return out;
}

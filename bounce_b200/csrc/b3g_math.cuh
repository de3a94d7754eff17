// Device math with the reference's exact single-precision operation order.
//
// Every routine here evaluates the same IEEE operations, in the same order,
// as the inline functions of include/bounce/common/math/{vec3,quat,transform,
// sweep}.h, include/bounce/collision/geometry/{aabb,plane}.h. The library is
// compiled with -fmad=false (no FMA contraction) and IEEE-rounded division
// and square root, so a routine given the same inputs returns the same bits
// as the reference built without FMA. Left-to-right evaluation of a + b + c
// in the reference is spelled out with explicit parentheses.
#pragma once

#include <cstdint>

#define B3G_EPSILON 1.1920928955078125e-07f /* FLT_EPSILON, B3_EPSILON (common.h:57) */
#define B3G_MAX_SCALAR 3.402823466e+38f     /* FLT_MAX, B3_MAX_SCALAR (common.h:56) */
#define B3G_LINEAR_SLOP 0.005f              /* B3_LINEAR_SLOP (common.h:81) */
#define B3G_AABB_EXTENSION 0.2f             /* B3_AABB_EXTENSION (common.h:73) */
#define B3G_AABB_MULTIPLIER 2.0f            /* B3_AABB_MULTIPLIER (common.h:78) */
#define B3G_NULL 0xFFFFFFFFu

#define B3G_HD __host__ __device__ __forceinline__

struct V3
{
	float x, y, z;
};

struct Q4
{
	V3 v;
	float s;
};

struct XF
{
	V3 p;
	Q4 q;
};

struct AABB
{
	V3 lo, hi;
};

struct PL
{
	V3 n;
	float d;
};

B3G_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
B3G_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
B3G_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
B3G_HD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
B3G_HD V3 operator*(float s, V3 v) { return V3{s * v.x, s * v.y, s * v.z}; }
// operator/(v, s): component-wise true division (vec3.h:178-181).
B3G_HD V3 operator/(V3 v, float s) { return V3{v.x / s, v.y / s, v.z / s}; }
B3G_HD float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
B3G_HD V3 cross(V3 a, V3 b)
{
	return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
B3G_HD float len(V3 v) { return sqrtf((v.x * v.x + v.y * v.y) + v.z * v.z); }
// b3Mul(vec, vec): component-wise product (scaling).
B3G_HD V3 vmul(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
B3G_HD float len2(V3 v) { return (v.x * v.x + v.y * v.y) + v.z * v.z; }
B3G_HD float fminr(float a, float b) { return a < b ? a : b; } // b3Min (math.h:45-48)
B3G_HD float fmaxr(float a, float b) { return a > b ? a : b; } // b3Max (math.h:51-54)
B3G_HD V3 vmin(V3 a, V3 b) { return V3{fminr(a.x, b.x), fminr(a.y, b.y), fminr(a.z, b.z)}; }
B3G_HD V3 vmax(V3 a, V3 b) { return V3{fmaxr(a.x, b.x), fmaxr(a.y, b.y), fmaxr(a.z, b.z)}; }
B3G_HD float fabsr(float x) { return fabsf(x); } // b3Abs = std::abs (math.h:39-42)

// b3Vec3::Normalize (vec3.h:92-103): scale by the reciprocal.
B3G_HD float normalize_inplace(V3& v)
{
	float l = sqrtf((v.x * v.x + v.y * v.y) + v.z * v.z);
	if (l > B3G_EPSILON)
	{
		float s = 1.0f / l;
		v.x *= s;
		v.y *= s;
		v.z *= s;
	}
	return l;
}

// b3Normalize(v) (vec3.h:210-219).
B3G_HD V3 normalized(V3 v)
{
	float l = len(v);
	if (l > B3G_EPSILON)
	{
		float s = 1.0f / l;
		return s * v;
	}
	return v;
}

// Quaternions (quat.h).
B3G_HD Q4 conj(Q4 q) { return Q4{-q.v, q.s}; }
B3G_HD Q4 qneg(Q4 q) { return Q4{-q.v, -q.s}; }
B3G_HD float qdot(Q4 a, Q4 b) { return dot(a.v, b.v) + a.s * b.s; }
// b3Mul(Quat, Quat) (quat.h:232-238).
B3G_HD Q4 qmul(Q4 a, Q4 b)
{
	Q4 r;
	r.v = (cross(a.v, b.v) + a.s * b.v) + b.s * a.v;
	r.s = a.s * b.s - dot(a.v, b.v);
	return r;
}
// b3Quat::Normalize (quat.h:50-59): v /= len scales by 1/len, s /= len divides.
B3G_HD void qnormalize_inplace(Q4& q)
{
	float l = sqrtf(dot(q.v, q.v) + q.s * q.s);
	if (l > B3G_EPSILON)
	{
		float s = 1.0f / l;
		q.v.x *= s;
		q.v.y *= s;
		q.v.z *= s;
		q.s /= l;
	}
}
// Rotate (quat.h:270-274): v + s*t + q.v x t with t = 2 (q.v x v).
B3G_HD V3 rot(Q4 q, V3 v)
{
	V3 t = 2.0f * cross(q.v, v);
	return (v + q.s * t) + cross(q.v, t);
}
B3G_HD V3 rotc(Q4 q, V3 v) { return rot(conj(q), v); }

// Transforms (transform.h:66-102).
B3G_HD V3 xmul(const XF& T, V3 v) { return rot(T.q, v) + T.p; }
B3G_HD V3 xmult(const XF& T, V3 v) { return rotc(T.q, v - T.p); }
// b3MulT(A, B) = A^-1 * B (transform.h:82-90).
B3G_HD XF xmult(const XF& A, const XF& B)
{
	XF C;
	C.q = qmul(conj(A.q), B.q);
	C.p = rotc(A.q, B.p - A.p);
	return C;
}

// Planes (plane.h:55-80).
B3G_HD PL pmul(const XF& T, PL p)
{
	V3 n = rot(T.q, p.n);
	return PL{n, p.d + dot(n, T.p)};
}
B3G_HD float pdist(V3 P, PL p) { return dot(p.n, P) - p.d; }
B3G_HD V3 pclosest(V3 P, PL p)
{
	float f = pdist(P, p);
	return P - f * p.n;
}

// AABBs (aabb.h).
B3G_HD V3 aabb_center(const AABB& a) { return 0.5f * (a.lo + a.hi); }
B3G_HD bool aabb_contains(const AABB& a, const AABB& b)
{
	bool r = true;
	r = r && a.lo.x <= b.lo.x;
	r = r && a.lo.y <= b.lo.y;
	r = r && a.lo.z <= b.lo.z;
	r = r && b.hi.x <= a.hi.x;
	r = r && b.hi.y <= a.hi.y;
	r = r && b.hi.z <= a.hi.z;
	return r;
}
// b3TestOverlap (aabb.h:347-367): closed intervals.
B3G_HD bool aabb_overlap(const AABB& a, const AABB& b)
{
	if (a.hi.x < b.lo.x || a.lo.x > b.hi.x)
		return false;
	if (a.hi.y < b.lo.y || a.lo.y > b.hi.y)
		return false;
	if (a.hi.z < b.lo.z || a.lo.z > b.hi.z)
		return false;
	return true;
}
B3G_HD void aabb_extend(AABB& a, float s)
{
	a.lo.x -= s;
	a.lo.y -= s;
	a.lo.z -= s;
	a.hi.x += s;
	a.hi.y += s;
	a.hi.z += s;
}

// Segment helpers (collision.cpp:139-215).
B3G_HD V3 closest_on_segment(V3 Q, V3 A, V3 B)
{
	V3 AB = B - A;
	float u = dot(B - Q, AB);
	float v = dot(Q - A, AB);
	if (v <= 0.0f)
		return A;
	if (u <= 0.0f)
		return B;
	float den = dot(AB, AB);
	if (den < B3G_LINEAR_SLOP * B3G_LINEAR_SLOP)
		return A;
	return (u * A + v * B) / den;
}

B3G_HD void closest_on_segments(V3& C1, V3& C2, V3 P1, V3 Q1, V3 P2, V3 Q2)
{
	V3 E1 = Q1 - P1;
	float L1 = len(E1);
	V3 E2 = Q2 - P2;
	float L2 = len(E2);
	if (L1 < B3G_LINEAR_SLOP && L2 < B3G_LINEAR_SLOP)
	{
		C1 = P1;
		C2 = P2;
		return;
	}
	if (L1 < B3G_LINEAR_SLOP)
	{
		C1 = P1;
		C2 = closest_on_segment(P1, P2, Q2);
		return;
	}
	if (L2 < B3G_LINEAR_SLOP)
	{
		C1 = closest_on_segment(P2, P1, Q1);
		C2 = P2;
		return;
	}
	V3 N1 = E1 / L1;
	V3 N2 = E2 / L2;
	float b = dot(N1, N2);
	float den = 1.0f - b * b;
	if (den != 0.0f)
	{
		float inv_den = 1.0f / den;
		V3 E3 = P1 - P2;
		float d = dot(N1, E3);
		float e = dot(N2, E3);
		float s = inv_den * (b * e - d);
		float t = inv_den * (e - b * d);
		C1 = P1 + s * N1;
		C2 = P2 + t * N2;
	}
	else
	{
		C1 = P1;
		C2 = P2;
	}
	C1 = closest_on_segment(C1, P1, Q1);
	C2 = closest_on_segment(C1, P2, Q2);
	C1 = closest_on_segment(C2, P1, Q1);
}

// b3BarycentricCoordinates for a segment (geometry.h:27-40).
B3G_HD void barycentric_segment(float out[3], V3 A, V3 B, V3 Q)
{
	V3 AB = B - A;
	V3 QA = A - Q;
	V3 QB = B - Q;
	float divisor = dot(AB, AB);
	out[0] = dot(QB, AB);
	out[1] = -dot(QA, AB);
	out[2] = divisor;
}

// b3BarycentricCoordinates for a triangle (geometry.h:45-68): u, v, w and
// the divisor.
B3G_HD void barycentric_triangle(float out[4], V3 A, V3 B, V3 C, V3 Q)
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
	out[3] = dot(AB_x_AC, AB_x_AC);
}

// b3Perp (vec3.h:247-262).
B3G_HD V3 perp(V3 v)
{
	const float sqrt_inv3 = 0.57735025882720947265625f; // sqrtf(1.0f / 3.0f)
	V3 u;
	if (fabsr(v.x) >= sqrt_inv3)
		u = V3{v.y, -v.x, 0.0f};
	else
		u = V3{0.0f, v.z, -v.y};
	normalize_inplace(u);
	return u;
}

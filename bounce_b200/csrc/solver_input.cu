// Solver input on the GPU: b3ContactSolver's constructor and
// InitializeVelocityConstraints (src/bounce/dynamics/contacts/contact_solver.cpp:28-149,
// :177-305) evaluated on the manifolds of the last collision pass, with the
// world manifold of b3WorldManifold::Initialize (src/bounce/collision/collision.cpp:63-101).
//
// The reference builds the constraints island by island from b3Position /
// b3Velocity arrays (island.cpp:130-152) and heap records per contact,
// manifold and point. Here one pass over the selected contacts writes two
// fixed-size record arrays (include/b3g.h: b3g_contact_constraint,
// b3g_manifold_constraint), the manifolds of consecutive constraints stored
// consecutively.
//
// Three launches, no per-contact scratch: k_ci_tiles reduces each tile of
// 256 items to (constraints, manifolds) packed in one u64, k_ci_scan_tiles
// scans the tile sums in one block and publishes the totals, and k_ci_build
// recomputes its items' counts, scans them inside the block and writes the
// records. Every expression below keeps the reference's operand order (the
// library is built with -fmad=false), so the records are the reference's bit
// for bit.
#include "collide_common.cuh"

static_assert(sizeof(b3g_solver_body) == 112, "b3g_solver_body: 7 float4");
static_assert(sizeof(b3g_contact_constraint) == 128, "b3g_contact_constraint: 8 float4");
static_assert(sizeof(b3g_manifold_constraint) == 464, "b3g_manifold_constraint: 29 float4");

namespace {

constexpr int CI_BLOCK = 256;

struct CIArgs
{
	const uint32_t* pairA;
	const uint32_t* pairB;
	const uint32_t* cstate;
	const DevManifold* man;
	const DevManifold* extra; // manifolds 1 and 2 of mesh contacts, or null
	const uint32_t* nContacts; // device: contacts of the last pass
	uint32_t maxContacts;
	const uint32_t* list;     // contacts to solve, or null: every touching non-sensor contact
	uint32_t listCount;
	const uint32_t* fixBody;
	const uint32_t* fixType;
	const uint32_t* fixFlags;
	const float4* fixParams;
	const float2* material;   // per fixture: friction, restitution
	const float4* bodies;     // b3g_solver_body records (7 float4 each)
	float dtRatio;
	int warm;
	unsigned long long* tiles;
	uint32_t* counts;         // device: constraints, manifolds
	float4* cOut;             // b3g_contact_constraint records (8 float4 each)
	uint32_t cCap;
	float4* mOut;             // b3g_manifold_constraint records (29 float4 each)
	uint32_t mCap;
};

// The items: the list entries, or the contacts of the last pass.
__device__ __forceinline__ uint32_t item_count(const CIArgs& a)
{
	return a.list ? a.listCount : min(*a.nContacts, a.maxContacts);
}

// Item i: its contact, whether it gets a constraint and its manifold count.
// A listed contact always gets one (the reference solves what its island
// holds; an index past the contact list gets a record without manifolds);
// by default a contact gets one when it is touching and neither fixture is a
// sensor (the island filter of b3World::Solve, world.cpp:336-348).
__device__ __forceinline__ void item_counts(const CIArgs& a, uint32_t i, uint32_t n, uint32_t& c, uint32_t& flag,
	uint32_t& mc)
{
	flag = 0;
	mc = 0;
	c = 0xFFFFFFFFu;
	if (i >= n)
		return;
	if (a.list)
	{
		c = a.list[i];
		flag = 1;
		if (c < min(*a.nContacts, a.maxContacts))
			mc = min((a.cstate[c] >> 8) & 0xFFu, 3u);
		else
			c = 0xFFFFFFFFu;
		return;
	}
	c = i;
	uint32_t st = a.cstate[c];
	if ((st & 1u) == 0)
		return;
	if (((a.fixFlags[a.pairA[c]] | a.fixFlags[a.pairB[c]]) & B3G_FIXTURE_SENSOR) != 0)
		return;
	flag = 1;
	mc = min((st >> 8) & 0xFFu, 3u);
}

__device__ __forceinline__ unsigned long long pack2(uint32_t flag, uint32_t mc)
{
	return ((unsigned long long)flag << 32) | mc;
}

// Block-wide exclusive scan of one u64 per thread; returns the thread's
// exclusive prefix and leaves the block total in *total.
__device__ __forceinline__ unsigned long long block_scan(unsigned long long v, unsigned long long* total)
{
	__shared__ unsigned long long warpSum[CI_BLOCK / 32];
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	unsigned long long x = v;
	for (int off = 1; off < 32; off <<= 1)
	{
		unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, off);
		if (lane >= (uint32_t)off)
			x += y;
	}
	if (lane == 31)
		warpSum[warp] = x;
	__syncthreads();
	if (warp == 0)
	{
		unsigned long long w = lane < CI_BLOCK / 32 ? warpSum[lane] : 0ull;
		for (int off = 1; off < 32; off <<= 1)
		{
			unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, w, off);
			if (lane >= (uint32_t)off)
				w += y;
		}
		if (lane < CI_BLOCK / 32)
			warpSum[lane] = w;
	}
	__syncthreads();
	unsigned long long before = warp ? warpSum[warp - 1] : 0ull;
	*total = warpSum[CI_BLOCK / 32 - 1];
	return before + x - v;
}

__global__ void __launch_bounds__(CI_BLOCK) k_ci_tiles(CIArgs a)
{
	const uint32_t n = item_count(a);
	if (blockIdx.x * CI_BLOCK >= n)
	{
		if (threadIdx.x == 0)
			a.tiles[blockIdx.x] = 0;
		return;
	}
	uint32_t c, flag, mc;
	item_counts(a, blockIdx.x * CI_BLOCK + threadIdx.x, n, c, flag, mc);
	unsigned long long total;
	block_scan(pack2(flag, mc), &total);
	if (threadIdx.x == 0)
		a.tiles[blockIdx.x] = total;
}

// Exclusive scan of the tile sums (one block); the totals go to counts.
__global__ void __launch_bounds__(1024) k_ci_scan_tiles(CIArgs a, uint32_t tiles)
{
	__shared__ unsigned long long part[1024];
	const uint32_t per = (tiles + 1023) / 1024;
	const uint32_t beg = threadIdx.x * per, end = min(beg + per, tiles);
	unsigned long long sum = 0;
	for (uint32_t i = beg; i < end; ++i)
		sum += a.tiles[i];
	part[threadIdx.x] = sum;
	__syncthreads();
	for (uint32_t off = 1; off < 1024; off <<= 1)
	{
		unsigned long long v = threadIdx.x >= off ? part[threadIdx.x - off] : 0ull;
		__syncthreads();
		part[threadIdx.x] += v;
		__syncthreads();
	}
	unsigned long long run = part[threadIdx.x] - sum;
	for (uint32_t i = beg; i < end; ++i)
	{
		unsigned long long t = a.tiles[i];
		a.tiles[i] = run;
		run += t;
	}
	if (threadIdx.x == 1023)
	{
		a.counts[0] = (uint32_t)(part[1023] >> 32);
		a.counts[1] = (uint32_t)(part[1023] & 0xFFFFFFFFull);
	}
}

// b3g_solver_body: x[3] q[4] v[3] w[3] invMass localCenter[3] invI[9] pad[2].
struct SBody
{
	V3 x;
	Q4 q;
	V3 v, w;
	float invMass;
	V3 lc;
	V3 I[3]; // columns of b3Position::I
};

__device__ __forceinline__ SBody load_body(const float4* bodies, uint32_t b)
{
	float r[28];
	const float4* p = bodies + 7 * (size_t)b;
#pragma unroll
	for (int k = 0; k < 7; ++k)
	{
		float4 t = __ldg(p + k);
		r[4 * k] = t.x;
		r[4 * k + 1] = t.y;
		r[4 * k + 2] = t.z;
		r[4 * k + 3] = t.w;
	}
	SBody s;
	s.x = v3(r[0], r[1], r[2]);
	s.q = Q4{v3(r[3], r[4], r[5]), r[6]};
	s.v = v3(r[7], r[8], r[9]);
	s.w = v3(r[10], r[11], r[12]);
	s.invMass = r[13];
	s.lc = v3(r[14], r[15], r[16]);
	s.I[0] = v3(r[17], r[18], r[19]);
	s.I[1] = v3(r[20], r[21], r[22]);
	s.I[2] = v3(r[23], r[24], r[25]);
	return s;
}

// b3Mat33 * b3Vec3 (mat33.h:129-132): v.x * A.x + v.y * A.y + v.z * A.z.
__device__ __forceinline__ V3 mat_mul(const V3 A[3], V3 v)
{
	return (v.x * A[0] + v.y * A[1]) + v.z * A[2];
}

// b3Shape::m_radius: sphere and capsule radius, B3_HULL_RADIUS (0) for hulls,
// triangles and meshes unless the fixture's parameters say otherwise
// (hull_shape.cpp:28, triangle_shape.cpp:27, mesh_shape.cpp:27).
__device__ __forceinline__ float shape_radius(const CIArgs& a, uint32_t f)
{
	const float4 p0 = a.fixParams[3 * f], p1 = a.fixParams[3 * f + 1], p2 = a.fixParams[3 * f + 2];
	switch (a.fixType[f])
	{
	case B3G_SHAPE_SPHERE:
		return p0.w;
	case B3G_SHAPE_CAPSULE:
		return p1.z;
	case B3G_SHAPE_TRIANGLE:
		return p2.y;
	case B3G_SHAPE_HULL:
		return p0.x;
	default:
		return p0.w;
	}
}

__device__ __forceinline__ float4 f4(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
__device__ __forceinline__ float u2f(uint32_t u) { return __uint_as_float(u); }

// One manifold of one constraint: the velocity-constraint manifold of the
// constructor (contact_solver.cpp:87-147) completed by
// InitializeVelocityConstraints (:214-302), and the position-constraint points.
__device__ void build_manifold(const CIArgs& a, const DevManifold& m, uint32_t k, const SBody& A, const SBody& B,
	const XF& xfA, const XF& xfB, float radiusA, float radiusB, float rest, float4* out)
{
	const uint32_t pc = min(m.pointCount, 4u);
	V3 point[4], nrm[4];
	// b3WorldManifold::Initialize (collision.cpp:78-101) with
	// b3WorldManifoldPoint::Initialize (:63-76).
	V3 center = v3(0.0f, 0.0f, 0.0f), normal = v3(0.0f, 0.0f, 0.0f);
#pragma unroll
	for (uint32_t q = 0; q < 4; ++q)
	{
		if (q >= pc)
			break;
		const DevPoint& p = m.points[q];
		V3 nA = rot(xfA.q, v3(p.n[0], p.n[1], p.n[2]));
		V3 cA = xmul(xfA, v3(p.p1[0], p.p1[1], p.p1[2]));
		V3 cB = xmul(xfB, v3(p.p2[0], p.p2[1], p.p2[2]));
		V3 pA = cA + radiusA * nA;
		V3 pB = cB - radiusB * nA;
		point[q] = 0.5f * (pA + pB);
		nrm[q] = nA;
		center = center + point[q];
		normal = normal + nA;
	}
	V3 t1 = v3(0.0f, 0.0f, 0.0f), t2 = v3(0.0f, 0.0f, 0.0f);
	V3 mrA = v3(0.0f, 0.0f, 0.0f), mrB = v3(0.0f, 0.0f, 0.0f);
	float tm[4] = {0.0f, 0.0f, 0.0f, 0.0f};
	float motorMass = 0.0f;
	const float mA = A.invMass, mB = B.invMass;
	if (pc > 0)
	{
		// center /= pointCount (vec3.h:70-76: scale by the reciprocal)
		const float s = 1.0f / (float)pc;
		center = v3(center.x * s, center.y * s, center.z * s);
		normalize_inplace(normal);
		t1 = perp(normal);
		t2 = cross(t1, normal);
		// Friction (contact_solver.cpp:267-292).
		mrA = center - A.x;
		mrB = center - B.x;
		V3 rn1A = cross(mrA, t1), rn1B = cross(mrB, t1);
		V3 rn2A = cross(mrA, t2), rn2B = cross(mrB, t2);
		float k11 = ((mA + mB) + dot(mat_mul(A.I, rn1A), rn1A)) + dot(mat_mul(B.I, rn1B), rn1B);
		float k12 = dot(mat_mul(A.I, rn1A), rn2A) + dot(mat_mul(B.I, rn1B), rn2B);
		float k22 = ((mA + mB) + dot(mat_mul(A.I, rn2A), rn2A)) + dot(mat_mul(B.I, rn2B), rn2B);
		// b3Inverse(b3Mat22) (math.cpp:89-97): det * b3Adjugate(K), K = [(k11, k12), (k12, k22)].
		float det = k11 * k22 - k12 * k12;
		if (det != 0.0f)
			det = 1.0f / det;
		tm[0] = det * k22;
		tm[1] = det * -k12;
		tm[2] = det * -k12;
		tm[3] = det * k11;
		// Twist (:295-299): dot(normal, (iA + iB) * normal).
		V3 S[3] = {A.I[0] + B.I[0], A.I[1] + B.I[1], A.I[2] + B.I[2]};
		float mass = dot(normal, mat_mul(S, normal));
		motorMass = mass > 0.0f ? 1.0f / mass : 0.0f;
	}
	const float ti0 = a.warm ? a.dtRatio * m.tangentImpulse[0] : 0.0f;
	const float ti1 = a.warm ? a.dtRatio * m.tangentImpulse[1] : 0.0f;
	const float mi = a.warm ? a.dtRatio * m.motorImpulse : 0.0f;
	out[0] = f4(mrA.x, mrA.y, mrA.z, mrB.x);
	out[1] = f4(mrB.y, mrB.z, normal.x, normal.y);
	out[2] = f4(normal.z, t1.x, t1.y, t1.z);
	out[3] = f4(t2.x, t2.y, t2.z, m.tangentSpeed1);
	out[4] = f4(m.tangentSpeed2, tm[0], tm[1], tm[2]);
	out[5] = f4(tm[3], ti0, ti1, mi);
	out[6] = f4(motorMass, m.motorSpeed, u2f(pc), u2f(k));
	out[7] = f4(0.0f, 0.0f, 0.0f, 0.0f);
	// Velocity-constraint points (:225-264).
	const V3 vA = A.v, wA = A.w, vB = B.v, wB = B.w;
#pragma unroll
	for (uint32_t q = 0; q < 4; ++q)
	{
		float4* o = out + 8 + 3 * q;
		if (q >= pc)
		{
			o[0] = o[1] = o[2] = f4(0.0f, 0.0f, 0.0f, 0.0f);
			continue;
		}
		const V3 n = nrm[q];
		const V3 rA = point[q] - A.x;
		const V3 rB = point[q] - B.x;
		V3 rnA = cross(rA, n), rnB = cross(rB, n);
		float K = ((mA + mB) + dot(mat_mul(A.I, rnA), rnA)) + dot(mat_mul(B.I, rnB), rnB);
		float normalMass = K > 0.0f ? 1.0f / K : 0.0f;
		V3 dv = ((vB + cross(wB, rB)) - vA) - cross(wA, rA);
		float vn = dot(n, dv);
		float bias = 0.0f;
		if (vn < -1.0f) // B3_VELOCITY_THRESHOLD (common.h:120)
			bias = -rest * vn;
		float ni = a.warm ? a.dtRatio * m.points[q].normalImpulse : 0.0f;
		o[0] = f4(rA.x, rA.y, rA.z, rB.x);
		o[1] = f4(rB.y, rB.z, n.x, n.y);
		o[2] = f4(n.z, normalMass, ni, bias);
	}
	// Position-constraint points (:127-130): the manifold's local frames.
	float pp[36];
#pragma unroll
	for (uint32_t q = 0; q < 4; ++q)
	{
		const DevPoint& p = m.points[q];
		const bool on = q < pc;
#pragma unroll
		for (int e = 0; e < 3; ++e)
		{
			pp[9 * q + e] = on ? p.n[e] : 0.0f;
			pp[9 * q + 3 + e] = on ? p.p1[e] : 0.0f;
			pp[9 * q + 6 + e] = on ? p.p2[e] : 0.0f;
		}
	}
#pragma unroll
	for (int e = 0; e < 9; ++e)
		out[20 + e] = f4(pp[4 * e], pp[4 * e + 1], pp[4 * e + 2], pp[4 * e + 3]);
}

__global__ void __launch_bounds__(CI_BLOCK) k_ci_build(CIArgs a)
{
	const uint32_t n = item_count(a);
	if (blockIdx.x * CI_BLOCK >= n)
		return;
	const uint32_t i = blockIdx.x * CI_BLOCK + threadIdx.x;
	uint32_t c, flag, mc;
	item_counts(a, i, n, c, flag, mc);
	unsigned long long total;
	unsigned long long pre = a.tiles[blockIdx.x] + block_scan(pack2(flag, mc), &total);
	if (!flag)
		return;
	const uint32_t k = (uint32_t)(pre >> 32);
	const uint32_t ms = (uint32_t)(pre & 0xFFFFFFFFull);
	if (c == 0xFFFFFFFFu)
	{
		if (k < a.cCap)
		{
			float4* o = a.cOut + 8 * (size_t)k;
			o[0] = f4(u2f(0xFFFFFFFFu), u2f(0xFFFFFFFFu), u2f(ms), u2f(0u));
			for (int e = 1; e < 7; ++e)
				o[e] = f4(0.0f, 0.0f, 0.0f, 0.0f);
			o[7] = f4(u2f(c), 0.0f, 0.0f, 0.0f);
		}
		return;
	}
	const uint32_t fa = a.pairA[c], fb = a.pairB[c];
	const uint32_t ba = a.fixBody[fa], bb = a.fixBody[fb];
	const SBody A = load_body(a.bodies, ba);
	const SBody B = load_body(a.bodies, bb);
	const float radiusA = shape_radius(a, fa), radiusB = shape_radius(a, fb);
	const float2 matA = a.material[fa], matB = a.material[fb];
	// b3MixFriction, b3MixRestitution (contact.h:33-43).
	const float friction = sqrtf(matA.x * matB.x);
	const float rest = fmaxr(matA.y, matB.y);
	if (k < a.cCap)
	{
		float4* o = a.cOut + 8 * (size_t)k;
		o[0] = f4(u2f(ba), u2f(bb), u2f(ms), u2f(mc));
		o[1] = f4(A.invMass, B.invMass, friction, rest);
		o[2] = f4(A.I[0].x, A.I[0].y, A.I[0].z, A.I[1].x);
		o[3] = f4(A.I[1].y, A.I[1].z, A.I[2].x, A.I[2].y);
		o[4] = f4(A.I[2].z, B.I[0].x, B.I[0].y, B.I[0].z);
		o[5] = f4(B.I[1].x, B.I[1].y, B.I[1].z, B.I[2].x);
		o[6] = f4(B.I[2].y, B.I[2].z, radiusA, radiusB);
		o[7] = f4(u2f(c), 0.0f, 0.0f, 0.0f);
	}
	// b3ContactSolver::InitializeVelocityConstraints (contact_solver.cpp:211-217):
	// the body frames from the centre of mass.
	XF xfA, xfB;
	xfA.q = A.q;
	xfA.p = A.x - rot(A.q, A.lc);
	xfB.q = B.q;
	xfB.p = B.x - rot(B.q, B.lc);
	for (uint32_t j = 0; j < mc; ++j)
	{
		if (ms + j >= a.mCap)
			break;
		const DevManifold& m = j == 0 ? a.man[c] : a.extra[2 * (size_t)c + j - 1];
		build_manifold(a, m, k, A, B, xfA, xfB, radiusA, radiusB, rest, a.mOut + 29 * (size_t)(ms + j));
	}
}

} // namespace

uint32_t contact_constraint_tiles(uint32_t items) { return (items + CI_BLOCK - 1) / CI_BLOCK; }

// Enqueues the three launches on s. items: the grid's item capacity (the
// list length, or max_contacts for the default selection).
void launch_contact_constraints(b3g_ctx* c, const ConstraintCall& q, cudaStream_t s)
{
	Buffers& B = c->buf;
	CIArgs a;
	a.pairA = B.pairA[c->cur];
	a.pairB = B.pairB[c->cur];
	a.cstate = B.cstate[c->cur];
	a.man = B.man[c->cur];
	a.extra = B.extraMan[c->cur];
	a.nContacts = B.counters + CTR_PAIRS;
	a.maxContacts = c->cfg.max_contacts;
	a.list = q.list;
	a.listCount = q.listCount;
	a.fixBody = c->scene.fixBody;
	a.fixType = c->scene.fixType;
	a.fixFlags = c->scene.fixFlags;
	a.fixParams = c->scene.fixParams;
	a.material = q.material;
	a.bodies = reinterpret_cast<const float4*>(q.bodies);
	a.dtRatio = q.dtRatio;
	a.warm = q.warm;
	a.tiles = q.tiles;
	a.counts = q.counts;
	a.cOut = reinterpret_cast<float4*>(q.constraints);
	a.cCap = q.constraints ? q.constraintCap : 0;
	a.mOut = reinterpret_cast<float4*>(q.manifolds);
	a.mCap = q.manifolds ? q.manifoldCap : 0;
	const uint32_t items = q.list ? q.listCount : c->cfg.max_contacts;
	const uint32_t tiles = std::max(contact_constraint_tiles(items), 1u);
	k_ci_tiles<<<tiles, CI_BLOCK, 0, s>>>(a);
	k_ci_scan_tiles<<<1, 1024, 0, s>>>(a, tiles);
	k_ci_build<<<tiles, CI_BLOCK, 0, s>>>(a);
}

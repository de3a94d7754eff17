// Solver input on the GPU: b3ContactSolver's constructor and
// InitializeVelocityConstraints (src/bounce/dynamics/contacts/contact_solver.cpp:28-149,
// :177-305) evaluated on the manifolds of the last collision pass, with the
// world manifold of b3WorldManifold::Initialize (src/bounce/collision/collision.cpp:63-101).
//
// The reference builds the constraints island by island from b3Position /
// b3Velocity arrays (island.cpp:130-152) and heap records per contact,
// manifold and point. Here one launch over the selected contacts writes two
// fixed-size record arrays (include/b3g.h: b3g_contact_constraint,
// b3g_manifold_constraint), the manifolds of consecutive constraints stored
// consecutively.
//
// One kernel of resident blocks. Each block takes tiles of 1,024 items
// (contacts of the list, or the caller's list entries) in order through a
// counter until none is left, counts the constraints and manifolds its items
// produce, and finds the counts of the tiles before it by decoupled look-back (Merrill & Garland: publish the
// tile's own count, add the published counts of earlier tiles until one that
// holds its inclusive prefix, 32 tiles per probe; bounded waits). The tile's
// selected items are compacted in shared memory in constraint order and
// handed out to quads: the four lanes of a quad build one constraint, lane q
// taking manifold point q, so consecutive quads write consecutive records.
// Every expression keeps the reference's operand order (the library is built
// with -fmad=false), so the records are the reference's bit for bit.
#include "collide_common.cuh"

static_assert(sizeof(b3g_solver_body) == 112, "b3g_solver_body: 7 float4");
static_assert(sizeof(b3g_contact_constraint) == 128, "b3g_contact_constraint: 8 float4");
static_assert(sizeof(b3g_manifold_constraint) == 464, "b3g_manifold_constraint: 29 float4");

namespace {

constexpr int CI_BLOCK = 256;
constexpr int CI_ITEMS = 4;
constexpr uint32_t CI_TILE = CI_BLOCK * CI_ITEMS;
// Tile status words: state in bits 62-63, (constraints << 32 | manifolds) below.
constexpr unsigned long long CI_AGG = 1ull << 62;
constexpr unsigned long long CI_INC = 2ull << 62;
constexpr unsigned long long CI_VAL = CI_AGG - 1ull;
constexpr uint32_t CI_SPIN = 1u << 22;

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
	unsigned long long* tileState; // [0]: tile counter, [1 + t]: status of tile t (zeroed per call)
	uint32_t* counts;         // device: constraints, manifolds (zeroed per call)
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
// sensor (the island filter of b3World::Solve, world.cpp:336-348). A selected
// contact's fixtures and bodies are looked up here, four items per thread in
// flight, rather than at the head of its quad's dependent loads.
struct Item
{
	uint32_t c, flag, mc, fa, fb, ba, bb;
};

__device__ __forceinline__ Item item_counts(const CIArgs& a, uint32_t i, uint32_t n)
{
	Item it{0xFFFFFFFFu, 0u, 0u, 0u, 0u, 0u, 0u};
	if (i >= n)
		return it;
	const uint32_t nc = min(*a.nContacts, a.maxContacts);
	uint32_t c;
	if (a.list)
	{
		c = a.list[i];
		it.flag = 1;
		if (c >= nc)
			return it;
	}
	else
	{
		c = i;
	}
	const uint32_t st = a.cstate[c];
	if (!a.list && (st & 1u) == 0)
		return it;
	it.fa = a.pairA[c];
	it.fb = a.pairB[c];
	if (!a.list && ((a.fixFlags[it.fa] | a.fixFlags[it.fb]) & B3G_FIXTURE_SENSOR) != 0)
		return it;
	it.c = c;
	it.flag = 1;
	it.mc = min((st >> 8) & 0xFFu, 3u);
	it.ba = a.fixBody[it.fa];
	it.bb = a.fixBody[it.fb];
	return it;
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

// b3g_solver_body as 7 float4: (x, q0) (q1 q2 q3, v0) (v1 v2, w0 w1)
// (w2, invMass, lc0 lc1) (lc2, I0 I1 I2) (I3..I6) (I7 I8, pad); B points at
// a body's record.

// b3Mat33 * b3Vec3 (mat33.h:129-132): v.x * A.x + v.y * A.y + v.z * A.z,
// the matrix as its 9 column-major words.
__device__ __forceinline__ V3 mat_mul(const float* I, V3 v)
{
	return (v.x * v3(I[0], I[1], I[2]) + v.y * v3(I[3], I[4], I[5])) + v.z * v3(I[6], I[7], I[8]);
}

__device__ __forceinline__ void load_inertia(const float4* B, float* I)
{
	const float4 f4 = B[4], f5 = B[5], f6 = B[6];
	I[0] = f4.y;
	I[1] = f4.z;
	I[2] = f4.w;
	I[3] = f5.x;
	I[4] = f5.y;
	I[5] = f5.z;
	I[6] = f5.w;
	I[7] = f6.x;
	I[8] = f6.y;
}

// b3ContactSolver::InitializeVelocityConstraints (contact_solver.cpp:211-217):
// the body frame from the centre of mass, x - q * localCenter.
__device__ __forceinline__ XF body_frame(const float4* B)
{
	const float4 f0 = B[0], f1 = B[1], f3 = B[3], f4 = B[4];
	XF xf;
	xf.q = Q4{v3(f0.w, f1.x, f1.y), f1.z};
	xf.p = v3(f0.x, f0.y, f0.z) - rot(xf.q, v3(f3.z, f3.w, f4.x));
	return xf;
}

// b3Shape::m_radius: sphere and capsule radius, B3_HULL_RADIUS (0) for hulls,
// triangles and meshes unless the fixture's parameters say otherwise
// (hull_shape.cpp:28, triangle_shape.cpp:27, mesh_shape.cpp:27).
__device__ __forceinline__ float shape_radius(const CIArgs& a, uint32_t f)
{
	switch (a.fixType[f])
	{
	case B3G_SHAPE_SPHERE:
		return a.fixParams[3 * f].w;
	case B3G_SHAPE_CAPSULE:
		return a.fixParams[3 * f + 1].z;
	case B3G_SHAPE_TRIANGLE:
		return a.fixParams[3 * f + 2].y;
	case B3G_SHAPE_HULL:
		return a.fixParams[3 * f].x;
	default:
		return a.fixParams[3 * f].w;
	}
}

__device__ __forceinline__ float4 f4(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
__device__ __forceinline__ float u2f(uint32_t u) { return __uint_as_float(u); }

// One manifold, built by the four lanes of a quad (lane `sub` = point sub):
// the velocity-constraint manifold of the constructor (contact_solver.cpp:87-147)
// completed by InitializeVelocityConstraints (:219-302), and the
// position-constraint points (:127-130). Every lane of the quad calls this.
__device__ void quad_manifold(const CIArgs& a, const DevManifold* m, uint32_t k, const float4* BA, const float4* BB,
	float radiusA, float radiusB, float rest, uint32_t sub, uint32_t mask, float4* out)
{
	const uint32_t pc = min(m->pointCount, 4u);
	const bool has = sub < pc;
	const DevPoint* p = m->points + sub;
	const V3 ln = v3(p->n[0], p->n[1], p->n[2]);
	const V3 lp1 = v3(p->p1[0], p->p1[1], p->p1[2]);
	const V3 lp2 = v3(p->p2[0], p->p2[1], p->p2[2]);
	const float lni = p->normalImpulse;
	// b3WorldManifoldPoint::Initialize (collision.cpp:63-76) for this lane's point.
	V3 point = v3(0.0f, 0.0f, 0.0f), nA = v3(0.0f, 0.0f, 0.0f);
	if (has)
	{
		const XF xfA = body_frame(BA), xfB = body_frame(BB);
		nA = rot(xfA.q, ln);
		V3 cA = xmul(xfA, lp1);
		V3 cB = xmul(xfB, lp2);
		V3 pA = cA + radiusA * nA;
		V3 pB = cB - radiusB * nA;
		point = 0.5f * (pA + pB);
	}
	// b3WorldManifold::Initialize (:78-101): the sums in point order, in
	// every lane.
	V3 center = v3(0.0f, 0.0f, 0.0f), normal = v3(0.0f, 0.0f, 0.0f);
#pragma unroll
	for (int r = 0; r < 4; ++r)
	{
		V3 pr, nr;
		pr.x = __shfl_sync(mask, point.x, r, 4);
		pr.y = __shfl_sync(mask, point.y, r, 4);
		pr.z = __shfl_sync(mask, point.z, r, 4);
		nr.x = __shfl_sync(mask, nA.x, r, 4);
		nr.y = __shfl_sync(mask, nA.y, r, 4);
		nr.z = __shfl_sync(mask, nA.z, r, 4);
		if ((uint32_t)r < pc)
		{
			center = center + pr;
			normal = normal + nr;
		}
	}
	const float4 b0A = BA[0], b0B = BB[0];
	const V3 xA = v3(b0A.x, b0A.y, b0A.z), xB = v3(b0B.x, b0B.y, b0B.z);
	const float mA = BA[3].y, mB = BB[3].y;
	float IA[9], IB[9];
	load_inertia(BA, IA);
	load_inertia(BB, IB);
	// Velocity-constraint point (:225-264) of this lane.
	{
		float4* o = out + 8 + 3 * sub;
		float* op = reinterpret_cast<float*>(out) + 80 + 9 * sub;
		if (has)
		{
			const float4 b1A = BA[1], b2A = BA[2], b3A = BA[3];
			const float4 b1B = BB[1], b2B = BB[2], b3B = BB[3];
			const V3 vA = v3(b1A.w, b2A.x, b2A.y), wA = v3(b2A.z, b2A.w, b3A.x);
			const V3 vB = v3(b1B.w, b2B.x, b2B.y), wB = v3(b2B.z, b2B.w, b3B.x);
			const V3 rA = point - xA;
			const V3 rB = point - xB;
			V3 rnA = cross(rA, nA), rnB = cross(rB, nA);
			float K = ((mA + mB) + dot(mat_mul(IA, rnA), rnA)) + dot(mat_mul(IB, rnB), rnB);
			float normalMass = K > 0.0f ? 1.0f / K : 0.0f;
			V3 dv = ((vB + cross(wB, rB)) - vA) - cross(wA, rA);
			float vn = dot(nA, dv);
			float bias = 0.0f;
			if (vn < -1.0f) // B3_VELOCITY_THRESHOLD (common.h:120)
				bias = -rest * vn;
			float ni = a.warm ? a.dtRatio * lni : 0.0f;
			o[0] = f4(rA.x, rA.y, rA.z, rB.x);
			o[1] = f4(rB.y, rB.z, nA.x, nA.y);
			o[2] = f4(nA.z, normalMass, ni, bias);
			op[0] = ln.x;
			op[1] = ln.y;
			op[2] = ln.z;
			op[3] = lp1.x;
			op[4] = lp1.y;
			op[5] = lp1.z;
			op[6] = lp2.x;
			op[7] = lp2.y;
			op[8] = lp2.z;
		}
		else
		{
			o[0] = o[1] = o[2] = f4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
			for (int e = 0; e < 9; ++e)
				op[e] = 0.0f;
		}
	}
	// The manifold's own terms (:219-222, :267-299), in every lane; lane sub
	// writes header float4s 2 sub and 2 sub + 1.
	V3 t1 = v3(0.0f, 0.0f, 0.0f), t2 = v3(0.0f, 0.0f, 0.0f);
	V3 mrA = v3(0.0f, 0.0f, 0.0f), mrB = v3(0.0f, 0.0f, 0.0f);
	float tm0 = 0.0f, tm1 = 0.0f, tm3 = 0.0f, motorMass = 0.0f;
	if (pc > 0)
	{
		// center /= pointCount (vec3.h:70-76: scale by the reciprocal)
		const float s = 1.0f / (float)pc;
		center = v3(center.x * s, center.y * s, center.z * s);
		normalize_inplace(normal);
		t1 = perp(normal);
		t2 = cross(t1, normal);
		mrA = center - xA;
		mrB = center - xB;
		V3 rn1A = cross(mrA, t1), rn1B = cross(mrB, t1);
		V3 rn2A = cross(mrA, t2), rn2B = cross(mrB, t2);
		float k11 = ((mA + mB) + dot(mat_mul(IA, rn1A), rn1A)) + dot(mat_mul(IB, rn1B), rn1B);
		float k12 = dot(mat_mul(IA, rn1A), rn2A) + dot(mat_mul(IB, rn1B), rn2B);
		float k22 = ((mA + mB) + dot(mat_mul(IA, rn2A), rn2A)) + dot(mat_mul(IB, rn2B), rn2B);
		// b3Inverse(b3Mat22) (math.cpp:89-97): det * b3Adjugate(K), K = [(k11, k12), (k12, k22)].
		float det = k11 * k22 - k12 * k12;
		if (det != 0.0f)
			det = 1.0f / det;
		tm0 = det * k22;
		tm1 = det * -k12;
		tm3 = det * k11;
		// Twist (:295-299): dot(normal, (iA + iB) * normal).
		float S[9];
#pragma unroll
		for (int e = 0; e < 9; ++e)
			S[e] = IA[e] + IB[e];
		float mass = dot(normal, mat_mul(S, normal));
		motorMass = mass > 0.0f ? 1.0f / mass : 0.0f;
	}
	float4 w0, w1;
	switch (sub)
	{
	case 0:
		w0 = f4(mrA.x, mrA.y, mrA.z, mrB.x);
		w1 = f4(mrB.y, mrB.z, normal.x, normal.y);
		break;
	case 1:
		w0 = f4(normal.z, t1.x, t1.y, t1.z);
		w1 = f4(t2.x, t2.y, t2.z, m->tangentSpeed1);
		break;
	case 2:
	{
		const float ti0 = a.warm ? a.dtRatio * m->tangentImpulse[0] : 0.0f;
		const float ti1 = a.warm ? a.dtRatio * m->tangentImpulse[1] : 0.0f;
		const float mi = a.warm ? a.dtRatio * m->motorImpulse : 0.0f;
		w0 = f4(m->tangentSpeed2, tm0, tm1, tm1);
		w1 = f4(tm3, ti0, ti1, mi);
		break;
	}
	default:
		w0 = f4(motorMass, m->motorSpeed, u2f(pc), u2f(k));
		w1 = f4(0.0f, 0.0f, 0.0f, 0.0f);
		break;
	}
	out[2 * sub] = w0;
	out[2 * sub + 1] = w1;
}

// One constraint, built by a quad (every lane calls this with the same item).
__device__ void quad_contact(const CIArgs& a, uint32_t c, uint32_t k, uint32_t ms, uint32_t mc, uint32_t fa,
	uint32_t fb, uint32_t ba, uint32_t bb, uint32_t sub, uint32_t mask)
{
	if (c == 0xFFFFFFFFu)
	{
		if (k < a.cCap)
		{
			float4* o = a.cOut + 8 * (size_t)k;
			float4 w0 = f4(0.0f, 0.0f, 0.0f, 0.0f), w1 = w0;
			if (sub == 0)
				w0 = f4(u2f(0xFFFFFFFFu), u2f(0xFFFFFFFFu), u2f(ms), u2f(0u));
			if (sub == 3)
				w1 = f4(u2f(c), 0.0f, 0.0f, 0.0f);
			o[2 * sub] = w0;
			o[2 * sub + 1] = w1;
		}
		return;
	}
	const float4* BA = a.bodies + 7 * (size_t)ba;
	const float4* BB = a.bodies + 7 * (size_t)bb;
	const float radiusA = shape_radius(a, fa), radiusB = shape_radius(a, fb);
	const float2 matA = a.material[fa], matB = a.material[fb];
	// b3MixRestitution (contact.h:40-43).
	const float rest = fmaxr(matA.y, matB.y);
	if (k < a.cCap)
	{
		float4 w0, w1;
		switch (sub)
		{
		case 0:
			// b3MixFriction (contact.h:33-36).
			w0 = f4(u2f(ba), u2f(bb), u2f(ms), u2f(mc));
			w1 = f4(BA[3].y, BB[3].y, sqrtf(matA.x * matB.x), rest);
			break;
		case 1:
			w0 = f4(BA[4].y, BA[4].z, BA[4].w, BA[5].x);
			w1 = f4(BA[5].y, BA[5].z, BA[5].w, BA[6].x);
			break;
		case 2:
			w0 = f4(BA[6].y, BB[4].y, BB[4].z, BB[4].w);
			w1 = BB[5];
			break;
		default:
			w0 = f4(BB[6].x, BB[6].y, radiusA, radiusB);
			w1 = f4(u2f(c), 0.0f, 0.0f, 0.0f);
			break;
		}
		float4* o = a.cOut + 8 * (size_t)k;
		o[2 * sub] = w0;
		o[2 * sub + 1] = w1;
	}
	for (uint32_t j = 0; j < mc; ++j)
	{
		if (ms + j >= a.mCap)
			break;
		const DevManifold* m = j == 0 ? a.man + c : a.extra + 2 * (size_t)c + j - 1;
		quad_manifold(a, m, k, BA, BB, radiusA, radiusB, rest, sub, mask, a.mOut + 29 * (size_t)(ms + j));
	}
}

__global__ void __launch_bounds__(CI_BLOCK) k_contact_constraints(CIArgs a)
{
	__shared__ uint32_t sTile;
	__shared__ unsigned long long sPrefix;
	__shared__ uint32_t sItem[7][CI_TILE]; // per selected item: c, ms, mc, fa, fb, ba, bb
	const uint32_t t = threadIdx.x, lane = t & 31u;
	const uint32_t n = item_count(a);
	const uint32_t tiles = max((n + CI_TILE - 1) / CI_TILE, 1u);
	const uint32_t sub = lane & 3u, mask = 0xFu << (lane & ~3u);
	for (;;)
	{
		if (t == 0)
			sTile = (uint32_t)atomicAdd(a.tileState, 1ull);
		__syncthreads();
		const uint32_t tile = sTile;
		if (tile >= tiles)
			break;
		// Thread t holds items 4t .. 4t + 3 of the tile.
		Item it[CI_ITEMS];
		unsigned long long sum = 0;
#pragma unroll
		for (int r = 0; r < CI_ITEMS; ++r)
		{
			it[r] = item_counts(a, tile * CI_TILE + CI_ITEMS * t + r, n);
			sum += ((unsigned long long)it[r].flag << 32) | it[r].mc;
		}
		unsigned long long total;
		unsigned long long run = block_scan(sum, &total);
		if (t < 32)
		{
			// Publish the tile's counts, then look back 32 tiles at a time:
			// the counts of the tiles up to the nearest one holding its
			// inclusive prefix (tiles before the first count as such a tile
			// holding 0).
			volatile unsigned long long* st = a.tileState + 1;
			unsigned long long prefix = 0;
			bool timedOut = false;
			if (tile == 0)
			{
				if (lane == 0)
					st[0] = CI_INC | total;
			}
			else
			{
				if (lane == 0)
					st[tile] = CI_AGG | total;
				int32_t hi = (int32_t)tile - 1;
				uint32_t spins = 0;
				while (true)
				{
					const int32_t idx = hi - (int32_t)lane;
					const unsigned long long v = idx >= 0 ? (unsigned long long)st[idx] : (unsigned long long)CI_INC;
					const uint32_t notReady = __ballot_sync(0xFFFFFFFFu, (v & ~CI_VAL) == 0ull);
					const uint32_t inc = __ballot_sync(0xFFFFFFFFu, (v & CI_INC) != 0ull);
					const uint32_t last = inc ? (uint32_t)__ffs(inc) - 1u : 31u;
					const uint32_t need = last == 31u ? 0xFFFFFFFFu : (2u << last) - 1u;
					if (notReady & need)
					{
						if (++spins > CI_SPIN)
						{
							timedOut = true;
							break;
						}
						continue;
					}
					unsigned long long part = lane <= last ? (v & CI_VAL) : 0ull;
					for (int off = 16; off > 0; off >>= 1)
						part += __shfl_xor_sync(0xFFFFFFFFu, part, off);
					prefix += part;
					if (inc)
						break;
					hi -= 32;
				}
				if (lane == 0)
				{
					__threadfence();
					st[tile] = CI_INC | (prefix + total);
				}
			}
			if (lane == 0)
			{
				sPrefix = prefix;
				if (timedOut)
				{
					atomicMax(a.counts, 0xFFFFFFFFu);
					atomicMax(a.counts + 1, 0xFFFFFFFFu);
				}
				if (tile == tiles - 1)
				{
					const unsigned long long all = prefix + total;
					atomicMax(a.counts, (uint32_t)(all >> 32));
					atomicMax(a.counts + 1, (uint32_t)(all & 0xFFFFFFFFull));
				}
			}
		}
		// The tile's selected items in constraint order.
#pragma unroll
		for (int r = 0; r < CI_ITEMS; ++r)
		{
			if (it[r].flag)
			{
				const uint32_t kl = (uint32_t)(run >> 32);
				sItem[0][kl] = it[r].c;
				sItem[1][kl] = (uint32_t)(run & 0xFFFFFFFFull);
				sItem[2][kl] = it[r].mc;
				sItem[3][kl] = it[r].fa;
				sItem[4][kl] = it[r].fb;
				sItem[5][kl] = it[r].ba;
				sItem[6][kl] = it[r].bb;
			}
			run += ((unsigned long long)it[r].flag << 32) | it[r].mc;
		}
		__syncthreads();
		const uint32_t k0 = (uint32_t)(sPrefix >> 32), ms0 = (uint32_t)(sPrefix & 0xFFFFFFFFull);
		const uint32_t count = (uint32_t)(total >> 32);
		for (uint32_t e = t >> 2; e < count; e += CI_BLOCK / 4)
			quad_contact(a, sItem[0][e], k0 + e, ms0 + sItem[1][e], sItem[2][e], sItem[3][e], sItem[4][e],
				sItem[5][e], sItem[6][e], sub, mask);
		__syncthreads();
	}
}

} // namespace

uint32_t contact_constraint_tiles(uint32_t items) { return std::max((items + CI_TILE - 1) / CI_TILE, 1u); }

// Zeroes the tile states and the counts, then launches the kernel on s over
// the tiles of the item capacity (the list length, or max_contacts for the
// default selection).
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
	a.tileState = q.tiles;
	a.counts = q.counts;
	a.cOut = reinterpret_cast<float4*>(q.constraints);
	a.cCap = q.constraints ? q.constraintCap : 0;
	a.mOut = reinterpret_cast<float4*>(q.manifolds);
	a.mCap = q.manifolds ? q.manifoldCap : 0;
	const uint32_t tiles = contact_constraint_tiles(q.list ? q.listCount : c->cfg.max_contacts);
	// Persistent blocks (as many as are resident at once) take the tiles in
	// order through the counter until they run out.
	static int perSM = 0;
	if (perSM == 0 &&
		(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_contact_constraints, CI_BLOCK, 0) != cudaSuccess ||
			perSM < 1))
		perSM = 1;
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
	const uint32_t blocks = std::min<uint32_t>(tiles, (uint32_t)(perSM * sms));
	cudaMemsetAsync(q.tiles, 0, sizeof(unsigned long long) * ((size_t)tiles + 1), s);
	cudaMemsetAsync(q.counts, 0, 2 * sizeof(uint32_t), s);
	k_contact_constraints<<<blocks, CI_BLOCK, 0, s>>>(a);
}

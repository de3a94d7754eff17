// Fat-AABB update and broadphase of one collision pass.
//
//  k_sync        per proxy: swept AABB of the fixture over [xf0, xf1] and the
//                b3DynamicTree::MoveProxy keep-or-reinsert rule
//                (fixture.cpp:120-132, dynamic_tree.cpp:139-207), or the
//                CreateProxy fattening on a creation pass (dynamic_tree.cpp:108-128)
//  k_bounds / k_morton / radix sort
//                world-major 64-bit keys: world index << 32 | 30-bit Morton code
//                of the fat-AABB centre, sorted by an LSD radix sort
//  k_build       Karras (2012) radix tree over the sorted keys, with ropes
//                (the next node in depth-first order after a subtree)
//  k_refit       bottom-up node AABBs
//  k_traverse    stackless rope traversal from each leaf's own rope, which
//                visits exactly the leaves after it in sorted order, so each
//                overlapping pair is met once; the AddPair filters
//                (contact_manager.cpp:98-160) and the b3Contact::Create A/B
//                order (contact.cpp:290-322) are applied per pair
//
// The overlap set found this way is the set of pairs the reference has a
// contact for after FindNewContacts (pairs are created when either proxy
// moves); order.cu turns it into the contact list, which also keeps the
// contacts UpdateContacts skips because neither body is active.

#include <cuda/atomic>

#include "collide_common.cuh"

namespace {

constexpr uint32_t SENT = 0xFFFFFFFFu;


// Lanes per fixture in k_sync: a hull's vertex loop is split across them.
constexpr uint32_t SYNC_LANES = 8;

__device__ __forceinline__ V3 shfl_xor3(uint32_t mask, V3 v, int o)
{
	return V3{__shfl_xor_sync(mask, v.x, o), __shfl_xor_sync(mask, v.y, o), __shfl_xor_sync(mask, v.z, o)};
}

// b3Shape::ComputeAABB at two transforms for the lanes of one group, from
// the fixture's preloaded type and params (compute_aabbs's arithmetic): a
// hull's vertices are strided over the lanes and the boxes combined by min /
// max, which are exact, so the result is the serial loop's
// (b3HullShape::ComputeAABB, hull_shape.cpp:160-164). Every lane of the
// group ends with the same boxes.
__device__ __forceinline__ void group_aabbs(const DevScene& S, uint32_t type, float4 p0, float4 p1, float4 p2,
	uint32_t hullIndex, const XF& xa, const XF& xb, bool two, AABB& a, AABB& b, uint32_t lane, uint32_t mask)
{
	if (type == B3G_SHAPE_SPHERE)
	{
		V3 c = V3{p0.x, p0.y, p0.z};
		V3 rv = V3{p0.w, p0.w, p0.w};
		V3 ca = xmul(xa, c);
		a.lo = ca - rv;
		a.hi = ca + rv;
		V3 cb = two ? xmul(xb, c) : ca;
		b.lo = cb - rv;
		b.hi = cb + rv;
		return;
	}
	if (type == B3G_SHAPE_CAPSULE)
	{
		V3 v1 = V3{p0.x, p0.y, p0.z};
		V3 v2 = V3{p0.w, p1.x, p1.y};
		V3 rv = V3{p1.z, p1.z, p1.z};
		V3 c1 = xmul(xa, v1), c2 = xmul(xa, v2);
		a.lo = vmin(c1, c2) - rv;
		a.hi = vmax(c1, c2) + rv;
		if (two)
		{
			c1 = xmul(xb, v1);
			c2 = xmul(xb, v2);
		}
		b.lo = vmin(c1, c2) - rv;
		b.hi = vmax(c1, c2) + rv;
		return;
	}
	if (type == B3G_SHAPE_TRIANGLE)
	{
		// The reference ignores the transform here (triangle_shape.cpp:59-67).
		V3 v1 = V3{p0.x, p0.y, p0.z};
		V3 v2 = V3{p0.w, p1.x, p1.y};
		V3 v3_ = V3{p1.z, p1.w, p2.x};
		V3 rv = V3{p2.y, p2.y, p2.y};
		a.lo = vmin(v1, vmin(v2, v3_)) - rv;
		a.hi = vmax(v1, vmax(v2, v3_)) + rv;
		b = a;
		return;
	}
	const HullDesc h = S.hulls[hullIndex];
	const float4* hv = S.hverts + h.vOff;
	float4 w = hv[0];
	V3 v0 = V3{w.x, w.y, w.z};
	V3 ta = xmul(xa, v0), tb = two ? xmul(xb, v0) : ta;
	a.lo = a.hi = ta;
	b.lo = b.hi = tb;
	for (uint32_t k = 1 + lane; k < h.vCnt; k += SYNC_LANES)
	{
		w = hv[k];
		V3 v = V3{w.x, w.y, w.z};
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
	for (int o = SYNC_LANES / 2; o > 0; o >>= 1)
	{
		a.lo = vmin(a.lo, shfl_xor3(mask, a.lo, o));
		a.hi = vmax(a.hi, shfl_xor3(mask, a.hi, o));
		if (two)
		{
			b.lo = vmin(b.lo, shfl_xor3(mask, b.lo, o));
			b.hi = vmax(b.hi, shfl_xor3(mask, b.hi, o));
		}
	}
	float r = p0.x;
	aabb_extend(a, r);
	if (two)
		aabb_extend(b, r);
}

// Atomic min / max of IEEE floats (no NaN): non-negative floats order like
// their bits as signed integers, negative ones in reverse as unsigned.
__device__ __forceinline__ void atomic_min_float(float* a, float v)
{
	if (v >= 0.0f)
		atomicMin(reinterpret_cast<int*>(a), __float_as_int(v));
	else
		atomicMax(reinterpret_cast<unsigned int*>(a), __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_float(float* a, float v)
{
	if (v >= 0.0f)
		atomicMax(reinterpret_cast<int*>(a), __float_as_int(v));
	else
		atomicMin(reinterpret_cast<unsigned int*>(a), __float_as_uint(v));
}

// Refit of a reused tree (the passes between rebuilds): only the proxies
// whose fat AABB was re-inserted (moved) changed, and a walk needs every
// node to contain its leaves, not to be tight. k_sync writes a moved proxy's
// new box into its leaf and grows the leaf's ancestors by it (atomic min /
// max per coordinate), stopping at the first that already contains it (every
// node above contains that one). Nodes only grow until the next rebuild makes
// them tight again; an unmoved leaf's box is contained already.
__device__ __forceinline__ void grow_leaf(Buffers& B, uint32_t nLeaves, uint32_t proxy, V3 lo, V3 hi)
{
	const uint32_t leaf = nLeaves - 1u + B.leafOf[proxy];
	float* llo = reinterpret_cast<float*>(&B.nodeLo[leaf]);
	float* lhi = reinterpret_cast<float*>(&B.nodeHi[leaf]);
	llo[0] = lo.x;
	llo[1] = lo.y;
	llo[2] = lo.z;
	lhi[0] = hi.x;
	lhi[1] = hi.y;
	lhi[2] = hi.z;
	if (nLeaves < 2)
		return;
	uint32_t p = B.nodeParent[leaf];
	while (true)
	{
		const float4 cl = __ldcg(&B.nodeLo[p]), ch = __ldcg(&B.nodeHi[p]);
		if (cl.x <= lo.x && cl.y <= lo.y && cl.z <= lo.z && ch.x >= hi.x && ch.y >= hi.y && ch.z >= hi.z)
			return;
		float* plo = reinterpret_cast<float*>(&B.nodeLo[p]);
		float* phi = reinterpret_cast<float*>(&B.nodeHi[p]);
		atomic_min_float(plo + 0, lo.x);
		atomic_min_float(plo + 1, lo.y);
		atomic_min_float(plo + 2, lo.z);
		atomic_max_float(phi + 0, hi.x);
		atomic_max_float(phi + 1, hi.y);
		atomic_max_float(phi + 2, hi.z);
		if (p == 0)
			return;
		p = B.nodeParent[p];
	}
}

// One group of SYNC_LANES lanes per fixture; lane 0 writes. All lanes of a
// group take the same branches, so the group mask is exact for the shuffles.
// The per-body transforms of the pass (m_xf and b3Sweep::GetTransform(0),
// sweep.h:43-63, two float4 each, read by the later stages) are written by
// lane 1 of group b for body b. The fixture's records are loaded before any
// branch so that their loads overlap.
__global__ void k_sync(DevScene S, Buffers B, uint32_t nf, uint32_t nb, int creation, int grow)
{
	const uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) / SYNC_LANES;
	const uint32_t lane = threadIdx.x % SYNC_LANES;
	const uint32_t mask = ((1u << SYNC_LANES) - 1u) << ((threadIdx.x & 31u) & ~(SYNC_LANES - 1u));
	if (lane == 1 && g < nb)
	{
		pack_xf(S.bodyXf, g, load_xf(S.bodyState + 17 * (size_t)g));
		pack_xf(S.bodyXf0, g, sweep_xf0(S, g));
	}
	if (g >= nf)
		return;
	const uint32_t i = g;
	const bool w0 = lane == 0;
	const uint8_t life = S.fixLife[i];
	const uint32_t type = S.fixType[i];
	const uint32_t body = S.fixBody[i];
	const uint32_t hullIndex = S.fixHull[i];
	const float4 p0 = S.fixParams[3 * i + 0], p1 = S.fixParams[3 * i + 1], p2 = S.fixParams[3 * i + 2];
	const float4 tl = B.fatLo[i], th = B.fatHi[i];
	const float* st = S.bodyState + 17 * (size_t)body;
	float sv[17];
#pragma unroll
	for (int k = 0; k < 17; ++k)
		sv[k] = st[k];
	const uint32_t btype = S.bodyType[body];
	// The walk's filter reads one word per proxy (pair_filter).
	if (w0)
		B.proxyInfo[i] = (body & 0x0FFFFFFFu) | (btype == B3G_BODY_DYNAMIC ? 1u << 28 : 0u) | (type << 29);
	if (life == FIX_DEAD)
	{
		// No proxy: an empty box (lower > upper) that overlaps nothing.
		if (w0)
		{
			B.fatLo[i] = make_float4(B3G_MAX_SCALAR, B3G_MAX_SCALAR, B3G_MAX_SCALAR, 0.0f);
			B.fatHi[i] = make_float4(-B3G_MAX_SCALAR, -B3G_MAX_SCALAR, -B3G_MAX_SCALAR, 0.0f);
			B.moved[i] = 0;
		}
		return;
	}
	if (type == B3G_SHAPE_MESH)
	{
		// Meshes sit on static bodies: their proxy is created once (k_mesh_fat
		// on a creation pass) and never moves.
		if (w0)
			B.moved[i] = 0;
		return;
	}
	XF xf1 = load_xf(sv);
	if (creation || life == FIX_FRESH)
	{
		// b3DynamicTree::CreateProxy (dynamic_tree.cpp:108-128).
		AABB a, unused;
		group_aabbs(S, type, p0, p1, p2, hullIndex, xf1, xf1, false, a, unused, lane, mask);
		if (w0)
		{
			V3 r = V3{B3G_AABB_EXTENSION, B3G_AABB_EXTENSION, B3G_AABB_EXTENSION};
			V3 lo = a.lo - r, hi = a.hi + r;
			B.fatLo[i] = make_float4(lo.x, lo.y, lo.z, 0.0f);
			B.fatHi[i] = make_float4(hi.x, hi.y, hi.z, 0.0f);
			B.moved[i] = 1;
		}
		return;
	}
	// Every non-static body is synchronised, whatever its awake flag:
	// b3World::Solve synchronises each body of a solved island
	// (world.cpp:424-449), including those the island put to sleep in that
	// step (island.cpp:297-305). A body asleep since its last move keeps its
	// sweep, so synchronising it again finds its AABB inside the fat AABB it
	// got then and moves nothing: the result is the reference's, which skips it.
	if (btype == B3G_BODY_STATIC)
	{
		if (w0)
			B.moved[i] = 0;
		return;
	}
	// b3Body::SynchronizeFixtures (body.cpp:216-229): xf0 from the sweep start.
	XF xf0;
	xf0.q = Q4{V3{sv[10], sv[11], sv[12]}, sv[13]};
	V3 c0 = V3{sv[7], sv[8], sv[9]};
	V3 lc = V3{sv[14], sv[15], sv[16]};
	xf0.p = c0 - rot(xf0.q, lc);

	// b3Fixture::Synchronize (fixture.cpp:120-132).
	AABB a1, a2;
	group_aabbs(S, type, p0, p1, p2, hullIndex, xf0, xf1, true, a1, a2, lane, mask);
	if (!w0)
		return;
	AABB aabb;
	aabb.lo = vmin(a1.lo, a2.lo);
	aabb.hi = vmax(a1.hi, a2.hi);
	V3 disp = aabb_center(a2) - aabb_center(a1);

	// b3DynamicTree::MoveProxy (dynamic_tree.cpp:139-207).
	AABB fat = aabb;
	aabb_extend(fat, B3G_AABB_EXTENSION);
	V3 d = B3G_AABB_MULTIPLIER * disp;
	if (d.x < 0.0f)
		fat.lo.x += d.x;
	else
		fat.hi.x += d.x;
	if (d.y < 0.0f)
		fat.lo.y += d.y;
	else
		fat.hi.y += d.y;
	if (d.z < 0.0f)
		fat.lo.z += d.z;
	else
		fat.hi.z += d.z;

	AABB tree;
	tree.lo = V3{tl.x, tl.y, tl.z};
	tree.hi = V3{th.x, th.y, th.z};
	if (aabb_contains(tree, aabb))
	{
		AABB huge = fat;
		aabb_extend(huge, 4.0f * B3G_AABB_EXTENSION);
		if (aabb_contains(huge, tree))
		{
			B.moved[i] = 0;
			return;
		}
	}
	B.fatLo[i] = make_float4(fat.lo.x, fat.lo.y, fat.lo.z, 0.0f);
	B.fatHi[i] = make_float4(fat.hi.x, fat.hi.y, fat.hi.z, 0.0f);
	B.moved[i] = 1;
	if (grow)
		grow_leaf(B, nf, i, fat.lo, fat.hi);
}

// ---------------------------------------------------------------------------
// Scene bounds of the fat-AABB centres (for Morton quantisation).

__device__ __forceinline__ int f2o(float f)
{
	int i = __float_as_int(f);
	return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float o2f(int i)
{
	return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF);
}

__global__ void k_bounds_init(int* bnd)
{
	if (threadIdx.x < 3)
		bnd[threadIdx.x] = 0x7FFFFFFF;
	else if (threadIdx.x < 6)
		bnd[threadIdx.x] = (int)0x80000000;
}

__global__ void k_bounds(DevScene S, Buffers B, uint32_t n, int* bnd)
{
	__shared__ int s[6][8];
	float mn[3] = {B3G_MAX_SCALAR, B3G_MAX_SCALAR, B3G_MAX_SCALAR};
	float mx[3] = {-B3G_MAX_SCALAR, -B3G_MAX_SCALAR, -B3G_MAX_SCALAR};
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		if (S.fixLife[i] == FIX_DEAD)
			continue;
		float4 lo = B.fatLo[i], hi = B.fatHi[i];
		float c[3] = {0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z)};
		for (int k = 0; k < 3; ++k)
		{
			mn[k] = fminf(mn[k], c[k]);
			mx[k] = fmaxf(mx[k], c[k]);
		}
	}
	for (int k = 0; k < 3; ++k)
	{
		for (int o = 16; o > 0; o >>= 1)
		{
			mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
			mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
		}
	}
	int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (lane == 0)
	{
		for (int k = 0; k < 3; ++k)
		{
			s[k][warp] = f2o(mn[k]);
			s[3 + k][warp] = f2o(mx[k]);
		}
	}
	__syncthreads();
	if (threadIdx.x < 6)
	{
		int nw = blockDim.x >> 5;
		int v = s[threadIdx.x][0];
		for (int w = 1; w < nw; ++w)
			v = threadIdx.x < 3 ? min(v, s[threadIdx.x][w]) : max(v, s[threadIdx.x][w]);
		if (threadIdx.x < 3)
			atomicMin(bnd + threadIdx.x, v);
		else
			atomicMax(bnd + threadIdx.x, v);
	}
}

__device__ __forceinline__ uint32_t expand10(uint32_t v)
{
	v = (v * 0x00010001u) & 0xFF0000FFu;
	v = (v * 0x00000101u) & 0x0F00F00Fu;
	v = (v * 0x00000011u) & 0xC30C30C3u;
	v = (v * 0x00000005u) & 0x49249249u;
	return v;
}

__global__ void k_morton(DevScene S, Buffers B, uint32_t n, const int* bnd)
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	float lo[3] = {o2f(bnd[0]), o2f(bnd[1]), o2f(bnd[2])};
	float hi[3] = {o2f(bnd[3]), o2f(bnd[4]), o2f(bnd[5])};
	float4 a = B.fatLo[i], b = B.fatHi[i];
	float c[3] = {0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z)};
	uint32_t q[3];
	for (int k = 0; k < 3; ++k)
	{
		float ext = hi[k] - lo[k];
		float t = ext > 0.0f ? (c[k] - lo[k]) / ext : 0.0f;
		t = fminf(fmaxf(t, 0.0f), 1.0f);
		q[k] = min((uint32_t)(t * 1024.0f), 1023u);
	}
	uint32_t code = (expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]);
	// A proxy wider than a quarter of the scene along some axis (a ground
	// box, a mesh) sorts after the other proxies of its world: its pairs are
	// then found by the many short walks of the leaves before it instead of
	// by one long walk of its own. Only the traversal order changes.
	float e[3] = {b.x - a.x, b.y - a.y, b.z - a.z};
	for (int k = 0; k < 3; ++k)
		if (hi[k] > lo[k] && e[k] > 0.25f * (hi[k] - lo[k]))
			code = 0xFFFFFFFEu;
	uint32_t world = S.bodyWorld[S.fixBody[i]];
	// Dead proxies sort after every live one.
	B.keysA[i] = S.fixLife[i] == FIX_DEAD ? ~0ull : ((unsigned long long)world << 32) | code;
	B.valsA[i] = i;
}

// ---------------------------------------------------------------------------
// Scans.

// One-sweep LSD radix sort (Merrill & Garland's decoupled look-back): one
// histogram kernel for every digit pass up front, then one kernel per pass.
// A block ranks its tile's keys per digit in shared memory (stable: element
// order within the tile), publishes the tile's digit counts, adds up the
// counts of the tiles before it (walking back until a tile that already
// published an inclusive prefix) and scatters. Tiles are taken in launch
// order through a counter, so a tile only waits for tiles of blocks that
// started before it; the waits are bounded all the same.
constexpr int OS_THREADS = 256;
constexpr int OS_ITEMS = 4;
constexpr uint32_t OS_TILE = OS_THREADS * OS_ITEMS;
constexpr uint32_t OS_AGG = 1u << 30;     // the tile's own count is published
constexpr uint32_t OS_INC = 2u << 30;     // the count through this tile is published
constexpr uint32_t OS_MASK = OS_AGG - 1u; // counts below 2^30
constexpr uint32_t OS_SPIN = 1u << 22;

struct SortShifts
{
	int s[8];
	int n;
};

__global__ void k_os_hist(const unsigned long long* keys, uint32_t n, SortShifts sh, uint32_t* ghist)
{
	__shared__ uint32_t h[8][256];
	for (int p = 0; p < sh.n; ++p)
		h[p][threadIdx.x] = 0;
	__syncthreads();
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		unsigned long long k = keys[i];
		for (int p = 0; p < sh.n; ++p)
			atomicAdd(&h[p][(uint32_t)(k >> sh.s[p]) & 0xFFu], 1u);
	}
	__syncthreads();
	for (int p = 0; p < sh.n; ++p)
		if (h[p][threadIdx.x])
			atomicAdd(&ghist[p * 256 + threadIdx.x], h[p][threadIdx.x]);
}

// Exclusive scan of each pass's 256 digit counts (one block of 256 per pass).
__global__ void k_os_scan(uint32_t* ghist)
{
	__shared__ uint32_t v[256];
	uint32_t* g = ghist + blockIdx.x * 256;
	uint32_t x = g[threadIdx.x];
	v[threadIdx.x] = x;
	__syncthreads();
	for (uint32_t off = 1; off < 256; off <<= 1)
	{
		uint32_t y = threadIdx.x >= off ? v[threadIdx.x - off] : 0u;
		__syncthreads();
		v[threadIdx.x] += y;
		__syncthreads();
	}
	g[threadIdx.x] = v[threadIdx.x] - x;
}

__global__ void __launch_bounds__(OS_THREADS) k_onesweep(const unsigned long long* kin, const uint32_t* vin,
	unsigned long long* kout, uint32_t* vout, uint32_t n, int shift, const uint32_t* gOffset, uint32_t* status,
	uint32_t* tileCounter, uint32_t* err)
{
	__shared__ uint32_t sTile;
	__shared__ uint32_t run[256];
	__shared__ uint32_t wc[OS_THREADS / 32][256];
	__shared__ uint32_t base[256];
	const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
	if (t == 0)
		sTile = atomicAdd(tileCounter, 1u);
	run[t] = 0;
	for (int w = 0; w < OS_THREADS / 32; ++w)
		wc[w][t] = 0;
	__syncthreads();
	const uint32_t tile = sTile;
	const uint32_t lt = (1u << lane) - 1u;
	unsigned long long key[OS_ITEMS];
	uint32_t val[OS_ITEMS], dig[OS_ITEMS], rank[OS_ITEMS];
	for (int r = 0; r < OS_ITEMS; ++r)
	{
		uint32_t idx = tile * OS_TILE + r * OS_THREADS + t;
		bool valid = idx < n;
		key[r] = valid ? kin[idx] : 0ull;
		val[r] = valid ? vin[idx] : 0u;
		uint32_t d = valid ? ((uint32_t)(key[r] >> shift) & 0xFFu) : 0x100u;
		dig[r] = d;
		uint32_t peers = __match_any_sync(0xffffffffu, d);
		uint32_t pr = __popc(peers & lt);
		if (valid && pr == 0)
			wc[warp][d] = __popc(peers);
		__syncthreads();
		{
			uint32_t sum = run[t];
			for (int w = 0; w < OS_THREADS / 32; ++w)
			{
				uint32_t cnt = wc[w][t];
				wc[w][t] = sum;
				sum += cnt;
			}
			run[t] = sum;
		}
		__syncthreads();
		rank[r] = valid ? wc[warp][d] + pr : 0u;
		__syncthreads();
		for (int w = 0; w < OS_THREADS / 32; ++w)
			wc[w][t] = 0;
		__syncthreads();
	}
	// Thread t owns digit t: publish, look back, publish the inclusive prefix.
	{
		const uint32_t mine = run[t];
		volatile uint32_t* st = status;
		if (tile == 0)
			st[t] = OS_INC | mine;
		else
		{
			st[(size_t)tile * 256 + t] = OS_AGG | mine;
			uint32_t prefix = 0;
			int32_t look = (int32_t)tile - 1;
			uint32_t spins = 0;
			while (look >= 0)
			{
				uint32_t v = st[(size_t)look * 256 + t];
				if ((v & ~OS_MASK) == 0u)
				{
					if (++spins > OS_SPIN)
					{
						atomicOr(err, B3G_ST_WAIT_TIMEOUT);
						break;
					}
					continue;
				}
				prefix += v & OS_MASK;
				if (v & OS_INC)
					break;
				--look;
			}
			__threadfence();
			st[(size_t)tile * 256 + t] = OS_INC | (prefix + mine);
			base[t] = gOffset[t] + prefix;
		}
		if (tile == 0)
			base[t] = gOffset[t];
	}
	__syncthreads();
	for (int r = 0; r < OS_ITEMS; ++r)
	{
		if (dig[r] > 0xFFu)
			continue;
		uint32_t pos = base[dig[r]] + rank[r];
		if (pos < n)
		{
			kout[pos] = key[r];
			vout[pos] = val[r];
		}
	}
}

// ---------------------------------------------------------------------------
// Karras radix tree.

__device__ __forceinline__ int delta(const unsigned long long* k, int n, int i, int j)
{
	if (j < 0 || j >= n)
		return -1;
	unsigned long long a = k[i], b = k[j];
	if (a == b)
		return 64 + __clz((uint32_t)i ^ (uint32_t)j);
	return __clzll(a ^ b);
}

__global__ void k_build(Buffers B, int n)
{
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n - 1)
		return;
	const unsigned long long* k = B.keysA;
	int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
	int dmin = delta(k, n, i, i - d);
	int lmax = 2;
	while (delta(k, n, i, i + lmax * d) > dmin)
		lmax <<= 1;
	int l = 0;
	for (int t = lmax >> 1; t >= 1; t >>= 1)
		if (delta(k, n, i, i + (l + t) * d) > dmin)
			l += t;
	int j = i + l * d;
	int dnode = delta(k, n, i, j);
	int s = 0;
	int t = l;
	do
	{
		t = (t + 1) >> 1;
		if (delta(k, n, i, i + (s + t) * d) > dnode)
			s += t;
	} while (t > 1);
	int gamma = i + s * d + min(d, 0);
	int first = min(i, j), last = max(i, j);
	uint32_t left = (first == gamma) ? (uint32_t)(n - 1 + gamma) : (uint32_t)gamma;
	uint32_t right = (last == gamma + 1) ? (uint32_t)(n - 1 + gamma + 1) : (uint32_t)(gamma + 1);
	B.nodeLeft[i] = left;
	B.nodeRight[i] = right;
	B.nodeParent[left] = i;
	B.nodeParent[right] = i;
	B.nodeFirst[i] = first;
	B.nodeEnd[i] = last;
	B.splitRight[gamma] = right;
}

__global__ void k_leaves(DevScene S, Buffers B, int n)
{
	int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= n)
		return;
	uint32_t node = n - 1 + j;
	uint32_t proxy = B.valsA[j];
	uint32_t rope = (j == n - 1) ? SENT : B.splitRight[j];
	B.nodeLeft[node] = proxy;
	B.nodeFirst[node] = j;
	B.leafOf[proxy] = j;
	// Traversal reads a node as two float4: (lower, left child or proxy) and
	// (upper, rope).
	float4 lo = B.fatLo[proxy], hi = B.fatHi[proxy];
	B.nodeLo[node] = make_float4(lo.x, lo.y, lo.z, __uint_as_float(proxy));
	B.nodeHi[node] = make_float4(hi.x, hi.y, hi.z, __uint_as_float(rope));
	B.nodeRope[node] = rope;
	// What the walk's filter and contact order need of the proxy, addressed
	// by the leaf's position so it loads beside the node.
	B.leafData[j] = make_uint2(B.proxyInfo[proxy], S.fixKey[proxy]);
	if (j < n - 1)
	{
		B.nodeRope[j] = (B.nodeEnd[j] == (uint32_t)(n - 1)) ? SENT : B.splitRight[B.nodeEnd[j]];
		B.refitFlag[j] = 0;
	}
	// Last sorted leaf of each world (dead proxies, sorted last, belong to none).
	if (S.fixLife[proxy] != FIX_DEAD)
	{
		uint32_t w = S.bodyWorld[S.fixBody[proxy]];
		uint32_t nx = j == n - 1 ? SENT : B.valsA[j + 1];
		if (nx == SENT || S.fixLife[nx] == FIX_DEAD || S.bodyWorld[S.fixBody[nx]] != w)
			B.worldEnd[w] = j;
	}
}

__global__ void k_refit(Buffers B, int n)
{
	int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= n || n < 2)
		return;
	uint32_t node = n - 1 + j;
	uint32_t p = B.nodeParent[node];
	while (true)
	{
		// Release this child's box, acquire the sibling's: one acq_rel atomic
		// per level instead of two full fences.
		cuda::atomic_ref<uint32_t, cuda::thread_scope_device> flag(B.refitFlag[p]);
		uint32_t old = flag.fetch_add(1u, cuda::memory_order_acq_rel);
		if (old == 0)
			return;
		uint32_t l = B.nodeLeft[p], r = B.nodeRight[p];
		float4 al = __ldcg(&B.nodeLo[l]), ah = __ldcg(&B.nodeHi[l]);
		float4 bl = __ldcg(&B.nodeLo[r]), bh = __ldcg(&B.nodeHi[r]);
		B.nodeLo[p] = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), __uint_as_float(l));
		B.nodeHi[p] = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z),
			__uint_as_float(B.nodeRope[p]));
		if (p == 0)
			return;
		p = B.nodeParent[p];
	}
}

// ---------------------------------------------------------------------------
// Pair search.

// b3Contact::s_registers (contact.cpp:253-288): registered type pairs, and
// whether (t1, t2) is the primary order (fixture A keeps type t1).
__device__ __forceinline__ bool registered(uint32_t a, uint32_t b)
{
	// bit (a * 5 + b)
	const uint32_t mask =
		(1u << (0 * 5 + 0)) | (1u << (1 * 5 + 0)) | (1u << (0 * 5 + 1)) | (1u << (1 * 5 + 1)) |
		(1u << (2 * 5 + 0)) | (1u << (0 * 5 + 2)) | (1u << (2 * 5 + 1)) | (1u << (1 * 5 + 2)) |
		(1u << (3 * 5 + 0)) | (1u << (0 * 5 + 3)) | (1u << (3 * 5 + 1)) | (1u << (1 * 5 + 3)) |
		(1u << (3 * 5 + 2)) | (1u << (2 * 5 + 3)) | (1u << (3 * 5 + 3)) |
		(1u << (3 * 5 + 4)) | (1u << (4 * 5 + 3)) | (1u << (4 * 5 + 0)) | (1u << (0 * 5 + 4)) |
		(1u << (4 * 5 + 1)) | (1u << (1 * 5 + 4));
	return (mask >> (a * 5 + b)) & 1u;
}
__device__ __forceinline__ bool primary(uint32_t a, uint32_t b)
{
	const uint32_t mask = (1u << (0 * 5 + 0)) | (1u << (1 * 5 + 0)) | (1u << (1 * 5 + 1)) |
		(1u << (2 * 5 + 0)) | (1u << (2 * 5 + 1)) | (1u << (3 * 5 + 0)) | (1u << (3 * 5 + 1)) |
		(1u << (3 * 5 + 2)) | (1u << (3 * 5 + 3)) | (1u << (3 * 5 + 4)) | (1u << (4 * 5 + 0)) |
		(1u << (4 * 5 + 1));
	return (mask >> (a * 5 + b)) & 1u;
}

// AddPair filters: same body (contact_manager.cpp:104-108), b3Body::ShouldCollide
// (at least one dynamic body, body.cpp:240-246) and a registered shape pair
// (b3Contact::Create returns nullptr otherwise, contact.cpp:318-321).
__device__ __forceinline__ bool pair_filter(uint32_t infoA, uint32_t infoB)
{
	if (((infoA ^ infoB) & 0x0FFFFFFFu) == 0u)
		return false;
	if (((infoA | infoB) & (1u << 28)) == 0u)
		return false;
	return registered(infoA >> 29, infoB >> 29);
}

// The contact record of overlapping proxies pa, pb (keys keyA, keyB, shape
// types typeA, typeB): the broadphase order (min, max) of proxy ids
// (b3BroadPhase::Report, broad_phase.cpp:341-342) followed by the factory's
// primary-type swap (b3Contact::Create, contact.cpp:306-317). x = fixture A,
// y = fixture B.
__device__ __forceinline__ uint2 canon_pair_keys(uint32_t pa, uint32_t keyA, uint32_t typeA, uint32_t pb,
	uint32_t keyB, uint32_t typeB)
{
	const bool aFirst = keyA < keyB;
	uint32_t f1 = aFirst ? pa : pb, f2 = aFirst ? pb : pa;
	uint32_t t1 = aFirst ? typeA : typeB, t2 = aFirst ? typeB : typeA;
	if (!primary(t1, t2))
		return make_uint2(f2, f1);
	return make_uint2(f1, f2);
}

// Rope walk from leaf j's own rope. A node is read as two float4:
// (lower, left child | proxy) and (upper, rope); a leaf's proxy word and key
// (leafData) load beside it, so a found pair costs no further dependent
// load. The walk counts the filtered
// overlaps, keeps the first TRAV_SLOTS contact records in the leaf's scratch
// slots (slot-major) and appends the others, with their leaf and index, to
// the overflow list. MW: several worlds share the tree, so the walk stops at
// the first node past the query's world (worlds are contiguous in
// depth-first order).
constexpr uint32_t TRAV_SLOTS = B3G_TRAV_SLOTS;

template <bool MW>
__device__ __forceinline__ uint32_t walk(const DevScene& S, Buffers& B, int n, int j, uint32_t cap, uint32_t limit)
{
	uint32_t leaf = n - 1 + j;
	float4 ql = __ldg(B.nodeLo + leaf), qh = __ldg(B.nodeHi + leaf);
	uint32_t pa = __float_as_uint(ql.w);
	const uint2 da = __ldg(B.leafData + j);
	const uint32_t infoA = da.x, keyA = da.y;
	uint32_t wend = MW ? B.worldEnd[S.bodyWorld[S.fixBody[pa]]] : 0xFFFFFFFFu;
	uint32_t count = 0;
	uint32_t node = __float_as_uint(qh.w);
	uint2* scratch = reinterpret_cast<uint2*>(B.pairScratch);
	// A depth-first walk visits each of the 2n - 1 nodes at most once.
	uint32_t steps = 0;
	const uint32_t maxSteps = limit ? limit : 2u * (uint32_t)n + 1u;
	const uint32_t nodes = 2u * (uint32_t)n - 1u;
	while (node != SENT)
	{
		if (++steps > maxSteps || node >= nodes)
		{
			atomicOr(&B.counters[CTR_STATUS], B3G_ST_WAIT_TIMEOUT);
			break;
		}
		if (MW && B.nodeFirst[node] > wend)
			break;
		// The tree is read-only here: the read-only data path caches it in L1.
		float4 lo = __ldg(B.nodeLo + node), hi = __ldg(B.nodeHi + node);
		const bool leafNode = node >= (uint32_t)(n - 1);
		const uint2 db = leafNode ? __ldg(B.leafData + (node - (uint32_t)(n - 1))) : make_uint2(0u, 0u);
		bool overlap = !(hi.x < ql.x || lo.x > qh.x || hi.y < ql.y || lo.y > qh.y || hi.z < ql.z || lo.z > qh.z);
		if (overlap && !leafNode)
		{
			node = __float_as_uint(lo.w); // descend
			continue;
		}
		if (overlap)
		{
			uint32_t pb = __float_as_uint(lo.w);
			if (pair_filter(infoA, db.x))
			{
				uint2 p = canon_pair_keys(pa, keyA, infoA >> 29, pb, db.y, db.x >> 29);
				if (count < TRAV_SLOTS)
					scratch[(size_t)count * n + j] = p;
				else
				{
					uint32_t o = atomicAdd(&B.counters[CTR_TRAV_OVERFLOW], 1u);
					if (o < cap)
						B.travOverflow[o] = make_uint4(p.x, p.y, (uint32_t)j, count);
				}
				++count;
			}
		}
		node = __float_as_uint(hi.w);
	}
	return count;
}

// limit: node visits allowed per walk (0: 2n + 1, more than a depth-first
// walk makes), see b3g_set_walk_limit. Each leaf's pairs then take a range of
// the pass's pair list (rawA, rawB): one atomic per warp reserves the warp's
// ranges (the order of the pairs is free: the contact order follows the proxy
// keys), leafCount[j] keeps the range's start for the overflow records, and
// the thread copies its scratch slots there.
template <bool MW>
__global__ void k_traverse_count(DevScene S, Buffers B, int n, uint32_t cur, uint32_t cap, uint32_t limit)
{
	const int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= n)
		return;
	const uint32_t count = S.fixLife[B.valsA[j]] == FIX_DEAD ? 0u : walk<MW>(S, B, n, j, cap, limit);
	// The warp's lanes with a leaf: a prefix of the warp.
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t live = min(32u, (uint32_t)n - ((uint32_t)j - lane));
	const uint32_t mask = live == 32u ? 0xFFFFFFFFu : (1u << live) - 1u;
	__syncwarp(mask);
	uint32_t incl = count;
	for (uint32_t o = 1; o < 32u; o <<= 1)
	{
		const uint32_t y = __shfl_up_sync(mask, incl, o);
		if (lane >= o)
			incl += y;
	}
	uint32_t base = 0;
	if (lane == live - 1u)
		base = atomicAdd(&B.counters[CTR_RAW], incl);
	base = __shfl_sync(mask, base, live - 1u) + incl - count;
	B.leafCount[j] = base;
	const uint2* scratch = reinterpret_cast<const uint2*>(B.pairScratch);
	const uint32_t kept = min(count, TRAV_SLOTS);
	for (uint32_t k = 0; k < kept; ++k)
	{
		const uint32_t slot = base + k;
		if (slot < cap)
		{
			const uint2 p = scratch[(size_t)k * n + j];
			B.rawA[slot] = p.x;
			B.rawB[slot] = p.y;
		}
	}
}

// The overflow records: record k of leaf j goes to leafCount[j] + k. A list
// longer than the contact capacity means more pairs than contacts fit, which
// the status already reports.
__global__ void k_traverse_overflow(Buffers B, uint32_t cap)
{
	uint32_t n = min(B.counters[CTR_TRAV_OVERFLOW], cap);
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint4 r = B.travOverflow[t];
		uint32_t slot = B.leafCount[r.z] + r.w;
		if (slot < cap)
		{
			B.rawA[slot] = r.x;
			B.rawB[slot] = r.y;
		}
	}
}

// One-pass exclusive scan of u32 in place (decoupled look-back, as the
// one-sweep sort): a block takes the next tile through a counter, reduces its
// SC_TILE entries, publishes the tile's sum, adds up the sums of the tiles
// before it (walking back until a tile that already published its inclusive
// prefix; bounded wait) and writes its entries' offsets. n: *nPtr (at most
// cap) when nPtr is set, else nHost. state: the tile counter, then one word
// per tile (flag in bits 62-63, sum in bits 0-31), zeroed before the launch.
// The tile holding the last entry writes the total (0 for an empty scan).
constexpr int SC_THREADS = 256;
constexpr int SC_ITEMS = 8;
constexpr uint32_t SC_TILE = SC_THREADS * SC_ITEMS;
constexpr unsigned long long SC_AGG = 1ull << 62;
constexpr unsigned long long SC_INC = 2ull << 62;
constexpr uint32_t SC_SPIN = 1u << 22;

__global__ void __launch_bounds__(SC_THREADS) k_scan_tiles(uint32_t* data, const uint32_t* nPtr, uint32_t nHost,
	uint32_t cap, unsigned long long* state, uint32_t* total, uint32_t* err)
{
	__shared__ uint32_t sTile, sPrefix;
	__shared__ uint32_t warpSums[SC_THREADS / 32];
	const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
	const uint32_t n = nPtr ? min(*nPtr, cap) : nHost;
	if (t == 0)
		sTile = atomicAdd(reinterpret_cast<unsigned int*>(state), 1u);
	__syncthreads();
	const uint32_t tile = sTile;
	const uint32_t numTiles = (n + SC_TILE - 1) / SC_TILE;
	if (tile >= numTiles)
	{
		if (tile == 0 && t == 0 && total)
			*total = 0u;
		return;
	}
	// Thread t owns entries [t * SC_ITEMS, t * SC_ITEMS + SC_ITEMS) of the tile.
	const uint32_t first = tile * SC_TILE + t * SC_ITEMS;
	uint32_t v[SC_ITEMS];
	uint32_t sum = 0;
#pragma unroll
	for (int r = 0; r < SC_ITEMS; ++r)
	{
		v[r] = first + r < n ? data[first + r] : 0u;
		sum += v[r];
	}
	uint32_t incl = sum;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1)
	{
		uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
		if (lane >= (uint32_t)o)
			incl += y;
	}
	if (lane == 31)
		warpSums[warp] = incl;
	__syncthreads();
	if (warp == 0)
	{
		uint32_t w = lane < SC_THREADS / 32 ? warpSums[lane] : 0u;
		uint32_t wi = w;
#pragma unroll
		for (int o = 1; o < SC_THREADS / 32; o <<= 1)
		{
			uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
			if (lane >= (uint32_t)o)
				wi += y;
		}
		const uint32_t agg = __shfl_sync(0xFFFFFFFFu, wi, SC_THREADS / 32 - 1);
		if (lane < SC_THREADS / 32)
			warpSums[lane] = wi - w;
		// Look-back by the whole warp: lane k reads the tile k + 1 places
		// back, so a round trip covers 32 tiles. A window is taken once every
		// tile in it has published; the nearest inclusive prefix in it ends
		// the walk (tiles before the first one count as an inclusive 0).
		volatile unsigned long long* st = state + 1;
		if (lane == 0)
			st[tile] = (tile == 0 ? SC_INC : SC_AGG) | agg;
		uint32_t prefix = 0;
		int32_t look = (int32_t)tile - 1;
		uint32_t spins = 0;
		while (tile > 0)
		{
			const int32_t idx = look - (int32_t)lane;
			unsigned long long w8 = 2ull << 62; // before tile 0: an inclusive 0
			if (idx >= 0)
				w8 = st[idx];
			if (!__all_sync(0xFFFFFFFFu, (w8 >> 62) != 0ull))
			{
				if (++spins > SC_SPIN)
				{
					if (lane == 0)
						atomicOr(err, B3G_ST_WAIT_TIMEOUT);
					break;
				}
				continue;
			}
			const uint32_t inc = __ballot_sync(0xFFFFFFFFu, (w8 & SC_INC) != 0ull);
			const uint32_t last = inc ? (uint32_t)(__ffs(inc) - 1) : 31u;
			uint32_t v = lane <= last ? (uint32_t)w8 : 0u;
#pragma unroll
			for (int o = 16; o > 0; o >>= 1)
				v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
			prefix += v;
			if (inc)
				break;
			look -= 32;
		}
		if (lane == 0)
		{
			if (tile > 0)
			{
				__threadfence();
				st[tile] = SC_INC | (uint32_t)(prefix + agg);
			}
			sPrefix = prefix;
			if (tile == numTiles - 1 && total)
				*total = prefix + agg;
		}
	}
	__syncthreads();
	uint32_t run = sPrefix + warpSums[warp] + incl - sum;
#pragma unroll
	for (int r = 0; r < SC_ITEMS; ++r)
	{
		if (first + r < n)
			data[first + r] = run;
		run += v[r];
	}
}

} // namespace

// Words of scan state (u32) a scan of up to n entries needs in aux.
uint32_t scan_aux_words(uint32_t n)
{
	return 2u * ((n + SC_TILE - 1) / SC_TILE + 1u);
}

void scan_exclusive(uint32_t* data, uint32_t n, uint32_t* aux, uint32_t* total, uint32_t* err, cudaStream_t s)
{
	const uint32_t tiles = (n + SC_TILE - 1) / SC_TILE;
	cudaMemsetAsync(aux, 0, sizeof(unsigned long long) * (tiles + 1u), s);
	k_scan_tiles<<<tiles ? tiles : 1u, SC_THREADS, 0, s>>>(data, nullptr, n, n,
		reinterpret_cast<unsigned long long*>(aux), total, err);
}

void scan_exclusive_device(uint32_t* data, const uint32_t* nPtr, uint32_t cap, uint32_t* aux, uint32_t* total,
	uint32_t* err, cudaStream_t s)
{
	const uint32_t tiles = (cap + SC_TILE - 1) / SC_TILE;
	cudaMemsetAsync(aux, 0, sizeof(unsigned long long) * (tiles + 1u), s);
	k_scan_tiles<<<tiles ? tiles : 1u, SC_THREADS, 0, s>>>(data, nPtr, 0u, cap,
		reinterpret_cast<unsigned long long*>(aux), total, err);
}

// Stable sort of n (key, value) records by the low `bits` bits of the keys
// (the one-sweep passes of the broadphase sort). scratch holds
// radix_sort_scratch_words(n, bits) words. Returns the buffer pair holding
// the result: (keys, vals) or (keysTmp, valsTmp).
uint32_t radix_sort_scratch_words(uint32_t n, int bits)
{
	uint32_t passes = (uint32_t)(bits + 7) / 8;
	return 256u * (9u + passes * ((n + OS_TILE - 1) / OS_TILE));
}

bool radix_sort_pairs(unsigned long long* keys, uint32_t* vals, unsigned long long* keysTmp, uint32_t* valsTmp,
	uint32_t n, int bits, uint32_t* scratch, uint32_t* err, cudaStream_t s)
{
	SortShifts sh;
	sh.n = 0;
	for (int sft = 0; sft < bits && sh.n < 8; sft += 8)
		sh.s[sh.n++] = sft;
	if (n == 0 || sh.n == 0)
		return false;
	const uint32_t numTiles = (n + OS_TILE - 1) / OS_TILE;
	cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * (9 * 256 + (size_t)sh.n * numTiles * 256), s);
	k_os_hist<<<min((n + 255) / 256, 148u * 4u), 256, 0, s>>>(keys, n, sh, scratch);
	k_os_scan<<<sh.n, 256, 0, s>>>(scratch);
	unsigned long long *kin = keys, *kout = keysTmp;
	uint32_t *vin = vals, *vout = valsTmp;
	for (int p = 0; p < sh.n; ++p)
	{
		k_onesweep<<<numTiles, OS_THREADS, 0, s>>>(kin, vin, kout, vout, n, sh.s[p], scratch + 256 * p,
			scratch + 9 * 256 + (size_t)p * numTiles * 256, scratch + 8 * 256 + p, err);
		std::swap(kin, kout);
		std::swap(vin, vout);
	}
	return kin != keys;
}

void launch_sync(b3g_ctx* c, cudaStream_t s)
{
	uint32_t n = c->nFixtures;
	if (n == 0)
		return;
	const size_t groups = std::max<size_t>(n, c->nBodies);
	// A pass that reuses the LBVH refits it from here (grow_leaf).
	const int grow = !c->treeRebuild && c->treeLeaves == n ? 1 : 0;
	k_sync<<<(uint32_t)((groups * SYNC_LANES + 127) / 128), 128, 0, s>>>(c->scene, c->buf, n, c->nBodies,
		c->creationPass ? 1 : 0, grow);
	if (c->creationPass)
		launch_mesh_fat(c, s);
}

// Kernels launched by launch_broadphase for the current scene (kept next to
// the launcher so the count follows its structure).
uint32_t broadphase_launches(const b3g_ctx* c)
{
	uint32_t n = c->nFixtures;
	if (n == 0)
		return 0;
	uint32_t wb = 0;
	while ((1u << wb) < c->nWorlds)
		++wb;
	uint32_t passes = 4 + (wb + 7) / 8;
	// traversal: walk (with the pair list's ranges), overflow records
	if (!c->treeRebuild)
		return 2; // the tree refit by the sync kernel
	// bounds init, bounds, Morton; sort: histogram, scan, one kernel per
	// pass; build; leaves, refit
	return 3 + (passes + 2) + (n > 1 ? 1 : 0) + 2 + 2;
}

void launch_broadphase(b3g_ctx* c, cudaStream_t s)
{
	Buffers& B = c->buf;
	int n = (int)c->nFixtures;
	c->treeLeaves = (uint32_t)n;
	if (n == 0)
	{
		cudaMemsetAsync(B.counters + CTR_RAW, 0, sizeof(uint32_t), s);
		return;
	}
	if (!c->treeRebuild)
	{
		// Same tree as the last pass, refit by k_sync (grow_leaf): walk.
		prof_mark(c, PM_SORTED, s);
		prof_mark(c, PM_BUILT, s);
		launch_traverse(c, s);
		prof_mark(c, PM_TRAVERSED, s);
		return;
	}
	int* bnd = (int*)B.sceneBounds;
	k_bounds_init<<<1, 32, 0, s>>>(bnd);
	k_bounds<<<min((n + 255) / 256, 148 * 4), 256, 0, s>>>(c->scene, B, (uint32_t)n, bnd);
	k_morton<<<(n + 255) / 256, 256, 0, s>>>(c->scene, B, (uint32_t)n, bnd);

	// Radix sort over the Morton bits and, for several worlds, the world bits.
	SortShifts sh;
	sh.n = 0;
	for (int sft = 0; sft < 32; sft += 8)
		sh.s[sh.n++] = sft;
	uint32_t wb = 0;
	while ((1u << wb) < c->nWorlds)
		++wb;
	for (uint32_t sft = 0; sft < wb; sft += 8)
		sh.s[sh.n++] = 32 + (int)sft;
	const uint32_t numTiles = ((uint32_t)n + OS_TILE - 1) / OS_TILE;
	// sortHist: digit counts (8 x 256), tile counters (256), tile status (8 x tiles x 256)
	uint32_t* ghist = B.sortHist;
	uint32_t* tileCounters = B.sortHist + 8 * 256;
	uint32_t* status = B.sortHist + 9 * 256;
	cudaMemsetAsync(B.sortHist, 0, sizeof(uint32_t) * (9 * 256 + (size_t)sh.n * numTiles * 256), s);
	k_os_hist<<<min((n + 255) / 256, 148 * 4), 256, 0, s>>>(B.keysA, (uint32_t)n, sh, ghist);
	k_os_scan<<<sh.n, 256, 0, s>>>(ghist);
	unsigned long long *kin = B.keysA, *kout = B.keysB;
	uint32_t *vin = B.valsA, *vout = B.valsB;
	for (int p = 0; p < sh.n; ++p)
	{
		k_onesweep<<<numTiles, OS_THREADS, 0, s>>>(kin, vin, kout, vout, (uint32_t)n, sh.s[p], ghist + 256 * p,
			status + (size_t)p * numTiles * 256, tileCounters + p, B.counters + CTR_STATUS);
		std::swap(kin, kout);
		std::swap(vin, vout);
	}
	if (kin != B.keysA)
	{
		cudaMemcpyAsync(B.keysA, kin, sizeof(unsigned long long) * n, cudaMemcpyDeviceToDevice, s);
		cudaMemcpyAsync(B.valsA, vin, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s);
	}
	prof_mark(c, PM_SORTED, s);

	if (n > 1)
		k_build<<<(n - 1 + 255) / 256, 256, 0, s>>>(B, n);
	k_leaves<<<(n + 255) / 256, 256, 0, s>>>(c->scene, B, n);
	k_refit<<<(n + 255) / 256, 256, 0, s>>>(B, n);
	prof_mark(c, PM_BUILT, s);

	launch_traverse(c, s);
	prof_mark(c, PM_TRAVERSED, s);
}

// LBVH traversal (count, offsets, emit) of the tree built by this pass; the
// count kernel runs with the tuned block size. Re-running it on the same tree
// writes the same pairs.
void launch_traverse(b3g_ctx* c, cudaStream_t s)
{
	Buffers& B = c->buf;
	int n = (int)c->nFixtures;
	uint32_t cur = c->cur;
	if (n == 0)
		return;
	const int tb = (int)c->tune.v[B3G_TUNE_TRAVERSE];
	cudaMemsetAsync(B.counters + CTR_TRAV_OVERFLOW, 0, sizeof(uint32_t), s);
	cudaMemsetAsync(B.counters + CTR_RAW, 0, sizeof(uint32_t), s);
	if (c->nWorlds > 1)
		k_traverse_count<true><<<(n + tb - 1) / tb, tb, 0, s>>>(c->scene, B, n, cur, c->cfg.max_contacts,
			c->walkLimit);
	else
		k_traverse_count<false><<<(n + tb - 1) / tb, tb, 0, s>>>(c->scene, B, n, cur, c->cfg.max_contacts,
			c->walkLimit);
	k_traverse_overflow<<<persistent_blocks(2), 256, 0, s>>>(B, c->cfg.max_contacts);
}

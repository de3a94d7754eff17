// Persistent-pair bookkeeping of one pass and the narrowphase dispatch.
//
//  k_diff      looks each overlapping pair up in the previous pass's hash
//              table (pair key -> contact index) and inserts it into this
//              pass's table: found = the contact persists (its manifold and
//              feature cache are carried over), missing = a new contact
//              (b3ContactManager::AddPair, contact_manager.cpp:98-201)
//  k_ended     previous contacts whose pair was not found again are the ones
//              UpdateContacts destroys because their fat AABBs stopped
//              overlapping (contact_manager.cpp:270-281)
//  k_bucket    one work list per b3Contact subclass (contact.cpp:253-288)
//  k_finalize  touching counts and the host-facing contact records

#include "collide_common.cuh"

void launch_convex_buckets(const NPArgs& base, const uint32_t* lists, const uint32_t* counts, uint32_t cap,
	cudaStream_t s);
void launch_hulls(const NPArgs& base, const uint32_t* list, const uint32_t* count, uint32_t maxUE, cudaStream_t s);
void scan_exclusive(uint32_t* data, uint32_t n, uint32_t* aux, uint32_t* total, cudaStream_t s);

namespace {

constexpr unsigned long long EMPTY_KEY = 0xFFFFFFFFFFFFFFFFull;

__device__ __forceinline__ uint32_t hash64(unsigned long long k)
{
	k ^= k >> 33;
	k *= 0xff51afd7ed558ccdull;
	k ^= k >> 33;
	k *= 0xc4ceb9fe1a85ec53ull;
	k ^= k >> 33;
	return (uint32_t)k;
}

__global__ void k_diff(Buffers B, uint32_t cur, uint32_t cap, int havePrev)
{
	uint32_t n = min(B.counters[CTR_PAIRS], cap);
	uint32_t prevBuf = cur ^ 1u;
	uint32_t mask = B.hashCap - 1u;
	const unsigned long long* pk = B.hashKeys[prevBuf];
	const uint32_t* pv = B.hashVals[prevBuf];
	unsigned long long* ck = B.hashKeys[cur];
	uint32_t* cv = B.hashVals[cur];
	uint32_t begun = 0;
	for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
	{
		unsigned long long key = ((unsigned long long)B.pairA[cur][c] << 32) | B.pairB[cur][c];
		uint32_t h = hash64(key) & mask;
		int32_t prev = -1;
		if (havePrev)
		{
			for (uint32_t probe = 0; probe <= mask; ++probe)
			{
				unsigned long long k = pk[h];
				if (k == key)
				{
					prev = (int32_t)pv[h];
					break;
				}
				if (k == EMPTY_KEY)
					break;
				h = (h + 1) & mask;
			}
		}
		B.prevIndex[c] = prev;
		if (prev >= 0)
			B.prevFound[prev] = 1;
		else
			++begun;
		h = hash64(key) & mask;
		bool done = false;
		for (uint32_t probe = 0; probe <= mask; ++probe)
		{
			unsigned long long old = atomicCAS(&ck[h], EMPTY_KEY, key);
			if (old == EMPTY_KEY || old == key)
			{
				cv[h] = c;
				done = true;
				break;
			}
			h = (h + 1) & mask;
		}
		if (!done)
			atomicOr(&B.counters[CTR_STATUS], B3G_ST_HASH_OVERFLOW);
	}
	for (int o = 16; o > 0; o >>= 1)
		begun += __shfl_xor_sync(0xffffffffu, begun, o);
	if ((threadIdx.x & 31) == 0 && begun)
		atomicAdd(&B.counters[CTR_BEGUN], begun);
}

__global__ void k_ended(Buffers B, uint32_t cur, uint32_t cap)
{
	uint32_t prevBuf = cur ^ 1u;
	uint32_t n = min(B.counters[CTR_PREV_PAIRS], cap);
	for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
	{
		if (B.prevFound[p])
			continue;
		uint32_t slot = atomicAdd(&B.counters[CTR_ENDED], 1u);
		B.endedList[3 * slot + 0] = B.pairA[prevBuf][p];
		B.endedList[3 * slot + 1] = B.pairB[prevBuf][p];
		B.endedList[3 * slot + 2] = B.cstate[prevBuf][p];
	}
}

// Shape-type pair -> bucket (A carries the primary type).
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

__global__ void k_bucket(DevScene S, Buffers B, uint32_t cur, uint32_t cap)
{
	uint32_t n = min(B.counters[CTR_PAIRS], cap);
	for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
	{
		uint32_t fa = B.pairA[cur][c], fb = B.pairB[cur][c];
		uint32_t ba = S.fixBody[fa], bb = S.fixBody[fb];
		bool activeA = S.bodyAwake[ba] && S.bodyType[ba] != B3G_BODY_STATIC;
		bool activeB = S.bodyAwake[bb] && S.bodyType[bb] != B3G_BODY_STATIC;
		uint32_t bk;
		if (!activeA && !activeB)
			bk = BK_INACTIVE;
		else if ((S.fixFlags[fa] | S.fixFlags[fb]) & B3G_FIXTURE_SENSOR)
			bk = BK_SENSOR;
		else
			bk = bucket_of(S.fixType[fa], S.fixType[fb]);
		if (bk >= BK_COUNT)
			bk = BK_INACTIVE;
		// Warp-aggregated append.
		uint32_t peers = __match_any_sync(__activemask(), bk);
		uint32_t leader = __ffs(peers) - 1;
		uint32_t lane = threadIdx.x & 31;
		uint32_t base = 0;
		if (lane == leader)
			base = atomicAdd(&B.counters[CTR_BUCKET0 + bk], (uint32_t)__popc(peers));
		base = __shfl_sync(peers, base, leader);
		uint32_t rank = __popc(peers & ((1u << lane) - 1u));
		B.bucketList[(size_t)bk * cap + base + rank] = c;
	}
}

__global__ void k_finalize(Buffers B, uint32_t cur, uint32_t cap)
{
	uint32_t n = min(B.counters[CTR_PAIRS], cap);
	uint32_t touching = 0, manifolds = 0, points = 0;
	for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
	{
		uint32_t st = B.cstate[cur][c];
		uint32_t pc = ((st >> 8) & 0xFFu) ? B.man[cur][c].pointCount : 0u;
		touching += st & 1u;
		manifolds += pc > 0 ? 1u : 0u;
		points += pc;
		uint32_t flags = (st & 1u) | ((st >> 16 & 1u) << 1) | (st & 0xFF00u);
		B.contactOut[3 * c + 0] = B.pairA[cur][c];
		B.contactOut[3 * c + 1] = B.pairB[cur][c];
		B.contactOut[3 * c + 2] = flags;
	}
	for (int o = 16; o > 0; o >>= 1)
	{
		touching += __shfl_xor_sync(0xffffffffu, touching, o);
		manifolds += __shfl_xor_sync(0xffffffffu, manifolds, o);
		points += __shfl_xor_sync(0xffffffffu, points, o);
	}
	if ((threadIdx.x & 31) == 0)
	{
		if (touching)
			atomicAdd(&B.counters[CTR_TOUCHING], touching);
		if (manifolds)
			atomicAdd(&B.counters[CTR_MANIFOLDS], manifolds);
		if (points)
			atomicAdd(&B.counters[CTR_POINTS], points);
		if (manifolds)
			atomicAdd(&B.totals[2], (unsigned long long)manifolds);
		if (points)
			atomicAdd(&B.totals[3], (unsigned long long)points);
	}
}

__global__ void k_pass_end(Buffers B, uint32_t cap)
{
	if (threadIdx.x == 0)
	{
		B.totals[0] += 1;
		B.totals[1] += min(B.counters[CTR_PAIRS], cap);
		B.totals[4] += B.counters[CTR_BEGUN];
		B.totals[5] += B.counters[CTR_ENDED];
	}
}

__global__ void k_count_moved(Buffers B, uint32_t n)
{
	uint32_t m = 0;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		m += B.moved[i];
	for (int o = 16; o > 0; o >>= 1)
		m += __shfl_xor_sync(0xffffffffu, m, o);
	if ((threadIdx.x & 31) == 0 && m)
		atomicAdd(&B.counters[CTR_MOVED], m);
}

__global__ void k_overflow_check(Buffers B, uint32_t cap)
{
	if (B.counters[CTR_PAIRS] > cap)
		atomicOr(&B.counters[CTR_STATUS], B3G_ST_PAIR_OVERFLOW);
}

} // namespace

void launch_pairs_diff(b3g_ctx* c, cudaStream_t s)
{
	Buffers& B = c->buf;
	uint32_t cap = c->cfg.max_contacts;
	uint32_t cur = c->cur;
	cudaMemsetAsync(B.hashKeys[cur], 0xFF, sizeof(unsigned long long) * B.hashCap, s);
	cudaMemsetAsync(B.prevFound, 0, sizeof(uint32_t) * cap, s);
	k_overflow_check<<<1, 1, 0, s>>>(B, cap);
	k_diff<<<persistent_blocks(8), 256, 0, s>>>(B, cur, cap, c->havePass ? 1 : 0);
	if (c->havePass)
		k_ended<<<persistent_blocks(4), 256, 0, s>>>(B, cur, cap);
	k_count_moved<<<persistent_blocks(2), 256, 0, s>>>(B, c->nFixtures);
}

void launch_narrowphase(b3g_ctx* c, cudaStream_t s)
{
	Buffers& B = c->buf;
	uint32_t cap = c->cfg.max_contacts;
	uint32_t cur = c->cur, prev = cur ^ 1u;
	k_bucket<<<persistent_blocks(8), 256, 0, s>>>(c->scene, B, cur, cap);
	NPArgs a;
	a.S = c->scene;
	a.pairA = B.pairA[cur];
	a.pairB = B.pairB[cur];
	a.cstate = B.cstate[cur];
	a.cache = B.cache[cur];
	a.man = B.man[cur];
	a.prevState = B.cstate[prev];
	a.prevCache = B.cache[prev];
	a.prevMan = B.man[prev];
	a.prevIndex = B.prevIndex;
	a.list = nullptr;
	a.listCount = nullptr;
	a.status = B.counters + CTR_STATUS;
	a.warmStarting = (c->cfg.flags & B3G_FLAG_WARM_STARTING) ? 1 : 0;
	a.convexCache = (c->cfg.flags & B3G_FLAG_CONVEX_CACHE) ? 1 : 0;
	a.impN = c->impulsesLoaded ? B.impulseNormal : nullptr;
	a.impT = c->impulsesLoaded ? B.impulseTangent : nullptr;
	a.impM = c->impulsesLoaded ? B.impulseMotor : nullptr;
	a.exA = a.exB = a.ex0A = a.ex0B = nullptr;
	a.missList = B.missList;
	a.missCount = B.counters + CTR_HULL_MISS;
	launch_convex_buckets(a, B.bucketList, B.counters + CTR_BUCKET0, cap, s);
	prof_mark(c, PM_CONVEX, s);
	launch_hulls(a, B.bucketList + (size_t)BK_HULLS * cap, B.counters + CTR_BUCKET0 + BK_HULLS,
		c->maxUniqueEdges, s);
	prof_mark(c, PM_HULLS, s);
}

void launch_finalize(b3g_ctx* c, cudaStream_t s)
{
	k_finalize<<<persistent_blocks(4), 256, 0, s>>>(c->buf, c->cur, c->cfg.max_contacts);
	k_pass_end<<<1, 32, 0, s>>>(c->buf, c->cfg.max_contacts);
}

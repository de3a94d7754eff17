// Persistent-pair bookkeeping of one pass and the narrowphase dispatch.
//
//  k_diff      looks each overlapping pair up in the previous pass's hash
//              table (pair key -> contact index): found = the contact persists
//              (its manifold and feature cache are carried over), missing = a
//              new contact (b3ContactManager::AddPair, contact_manager.cpp:63-140);
//              new pairs are listed and counted per smaller proxy key for the
//              list-order layout (order.cu), which also lists the contacts
//              UpdateContacts destroys (contact_manager.cpp:263-276)
//  k_bucket    one work list per b3Contact subclass (contact.cpp:253-288)
//  k_finalize  touching counts and the host-facing contact records

#include "collide_common.cuh"

void launch_order(b3g_ctx* c, cudaStream_t s);
uint32_t order_launches(const b3g_ctx* c);

namespace {

// The previous contact of overlapping pair (a, b), or -1.
__device__ __forceinline__ int32_t previous_contact(const DevScene& S, const Buffers& B, uint32_t prevBuf, int havePrev,
	uint32_t a, uint32_t b)
{
	// A fresh fixture continues no contact of its slot's previous holder.
	bool fresh = S.fixLife[a] == FIX_FRESH || S.fixLife[b] == FIX_FRESH;
	return havePrev && !fresh
		? pair_hash_find(B.hashKeys[prevBuf], B.hashVals[prevBuf], B.hashMask[prevBuf] + 1u, pair_key(a, b))
		: -1;
}

// Whether overlapping pair (a, b), whose previous contact is prev (or -1), is
// no contact this pass under the joints, the per-contact veto and the moved
// rule (FilterArgs).
__device__ __forceinline__ bool filter_drop(const DevScene& S, const Buffers& B, const FilterArgs& F, uint32_t a,
	uint32_t b, int32_t prev)
{
	if (joint_excluded(F, S.fixBody[a], S.fixBody[b]))
		return true;
	if (prev >= 0)
		return F.vetoPrev && (uint32_t)prev < F.nVeto && F.vetoPrev[prev] != 0;
	return B.moved[a] == 0 && B.moved[b] == 0;
}

__global__ void k_diff(DevScene S, Buffers B, FilterArgs F, uint32_t cur, uint32_t cap, uint32_t nf, int havePrev)
{
	uint32_t n = min(B.counters[CTR_RAW], cap);
	uint32_t prevBuf = cur ^ 1u;
	const uint32_t lane = threadIdx.x & 31;
	for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x)
	{
		uint32_t c = base + threadIdx.x;
		bool isNew = false;
		if (c < n)
		{
			uint32_t a = B.rawA[c], b = B.rawB[c];
			int32_t prev = previous_contact(S, B, prevBuf, havePrev, a, b);
			bool drop = false;
			if (F.mode == 2)
				drop = F.rawDrop[c] != 0;
			else if (F.mode == 1)
				drop = filter_drop(S, B, F, a, b, prev);
			if (drop)
			{
				// No contact: a previous one is destroyed (k_kept), none is created.
			}
			else if (prev >= 0)
				B.prevFound[prev] = 1;
			else
			{
				isNew = true;
				atomicAdd(&B.newOff[nf - 1u - min(S.fixRank[a], S.fixRank[b])], 1u);
			}
		}
		// Warp-aggregated append to the new-pair list.
		uint32_t ballot = __ballot_sync(0xffffffffu, isNew);
		uint32_t slot = 0;
		if (lane == 0 && ballot)
			slot = atomicAdd(&B.counters[CTR_BEGUN], (uint32_t)__popc(ballot));
		slot = __shfl_sync(0xffffffffu, slot, 0);
		if (isNew)
			B.newList[slot + __popc(ballot & ((1u << lane) - 1u))] = c;
	}
}

// Contact filter (mode 2), before the contact list: the drop flag of every
// overlapping pair, and the pairs that would be new contacts (the AddPair
// calls the caller's filter decides) listed for the host.
__global__ void k_candidates(DevScene S, Buffers B, FilterArgs F, uint32_t* cand, uint32_t cur, uint32_t cap,
	int havePrev)
{
	uint32_t n = min(B.counters[CTR_RAW], cap);
	uint32_t prevBuf = cur ^ 1u;
	for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
	{
		uint32_t a = B.rawA[c], b = B.rawB[c];
		int32_t prev = previous_contact(S, B, prevBuf, havePrev, a, b);
		bool drop = filter_drop(S, B, F, a, b, prev);
		F.rawDrop[c] = drop ? 1 : 0;
		if (!drop && prev < 0)
		{
			uint32_t slot = atomicAdd(&B.counters[CTR_CANDIDATES], 1u);
			if (slot < cap)
				cand[slot] = c;
		}
	}
}

// Per candidate: the two fixtures as AddPair receives them (the fixture of
// the smaller proxy key first, broad_phase.cpp:341-342) and their keys.
__global__ void k_candidate_pairs(DevScene S, Buffers B, const uint32_t* cand, uint32_t n, uint4* out)
{
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = cand[t];
		uint32_t a = B.rawA[c], b = B.rawB[c];
		uint32_t ka = S.fixKey[a], kb = S.fixKey[b];
		out[t] = ka < kb ? make_uint4(a, b, ka, kb) : make_uint4(b, a, kb, ka);
	}
}

// The caller's filter rejected these candidates (raw indices).
__global__ void k_apply_veto(FilterArgs F, const uint32_t* rejected, uint32_t n)
{
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
		F.rawDrop[rejected[t]] = 1;
}

// Contacts to their narrowphase lists. The lists' counters are a dozen
// addresses that every contact of the pass adds to, so a block takes a tile of
// BUCKET_THREADS contacts, counts them per list in shared memory, reserves each
// list's range with one atomic, and then writes its contacts there.
constexpr int BUCKET_THREADS = 256;

__global__ void __launch_bounds__(BUCKET_THREADS) k_bucket(DevScene S, Buffers B, uint32_t cur, uint32_t cap)
{
	__shared__ uint32_t sCount[BK_COUNT], sBase[BK_COUNT];
	const uint32_t n = min(B.counters[CTR_PAIRS], cap);
	const uint32_t lane = threadIdx.x & 31;
	for (uint32_t tile = blockIdx.x * BUCKET_THREADS; tile < n; tile += gridDim.x * BUCKET_THREADS)
	{
		if (threadIdx.x < BK_COUNT)
			sCount[threadIdx.x] = 0;
		__syncthreads();
		const uint32_t c = tile + threadIdx.x;
		uint32_t bk = BK_COUNT, off = 0;
		if (c < n)
		{
			uint32_t fa = B.pairA[cur][c], fb = B.pairB[cur][c];
			uint32_t ba = S.fixBody[fa], bb = S.fixBody[fb];
			bool activeA = S.bodyAwake[ba] && S.bodyType[ba] != B3G_BODY_STATIC;
			bool activeB = S.bodyAwake[bb] && S.bodyType[bb] != B3G_BODY_STATIC;
			if (!activeA && !activeB)
				bk = BK_INACTIVE;
			else if (S.fixType[fa] == B3G_SHAPE_MESH || S.fixType[fb] == B3G_SHAPE_MESH)
				bk = BK_MESH; // b3MeshContact, sensors included (its TestOverlap runs per triangle)
			else if ((S.fixFlags[fa] | S.fixFlags[fb]) & B3G_FIXTURE_SENSOR)
				bk = BK_SENSOR;
			else
				bk = bucket_of(S.fixType[fa], S.fixType[fb]);
			if (bk >= BK_COUNT)
				bk = BK_INACTIVE;
			// Convex pairs whose bounding spheres are apart skip their routine
			// (spheres_apart); taking them out keeps the routines' warps full.
			if (bk <= BK_HULL_CAPSULE)
			{
				XF xfA = body_xf(S, ba), xfB = body_xf(S, bb);
				if (spheres_apart(S, fa, xfA, fb, xfB) ||
					(bk == BK_HULL_CAPSULE && hull_capsule_apart(S, fa, xfA, fb, xfB)))
					bk = BK_APART;
			}
			// The warp's contacts of one list take one shared-memory atomic.
			uint32_t peers = __match_any_sync(__activemask(), bk);
			uint32_t leader = __ffs(peers) - 1;
			uint32_t base = 0;
			if (lane == leader)
				base = atomicAdd(&sCount[bk], (uint32_t)__popc(peers));
			off = __shfl_sync(peers, base, leader) + __popc(peers & ((1u << lane) - 1u));
		}
		__syncthreads();
		if (threadIdx.x < BK_COUNT && sCount[threadIdx.x])
			sBase[threadIdx.x] = atomicAdd(&B.counters[CTR_BUCKET0 + threadIdx.x], sCount[threadIdx.x]);
		__syncthreads();
		if (bk < BK_COUNT)
			B.bucketList[(size_t)bk * cap + sBase[bk] + off] = c;
		__syncthreads();
	}
}

// Counters of the pass and the contact records (A, B, flags). A thread takes
// FIN_BATCH contacts a grid stride apart and loads all of their words before
// it uses any (the manifold's point count too, whether or not the contact
// has a manifold), so the loads of a contact do not wait on one another.
constexpr int FIN_BATCH = 4;
constexpr int FIN_THREADS = 256;

__global__ void __launch_bounds__(FIN_THREADS) k_finalize(DevScene S, Buffers B, uint32_t cur, uint32_t cap, uint32_t nf)
{
	// The pass's totals (counts the kernel does not change), and the fresh
	// fixtures become ordinary live ones.
	if (blockIdx.x == 0 && threadIdx.x == 0)
	{
		B.totals[0] += 1;
		B.totals[1] += min(B.counters[CTR_PAIRS], cap);
		B.totals[4] += B.counters[CTR_BEGUN];
		B.totals[5] += B.counters[CTR_ENDED];
	}
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x)
		if (S.fixLife[i] == FIX_FRESH)
			S.fixLife[i] = FIX_LIVE;
	uint32_t n = min(B.counters[CTR_PAIRS], cap);
	uint32_t touching = 0, manifolds = 0, points = 0;
	const uint32_t* __restrict__ cst = B.cstate[cur];
	const uint32_t* __restrict__ pA = B.pairA[cur];
	const uint32_t* __restrict__ pB = B.pairB[cur];
	const DevManifold* __restrict__ man = B.man[cur];
	const uint32_t stride = gridDim.x * blockDim.x;
	for (uint32_t c0 = blockIdx.x * blockDim.x + threadIdx.x; c0 < n; c0 += FIN_BATCH * stride)
	{
		uint32_t st[FIN_BATCH], pc0[FIN_BATCH], a[FIN_BATCH], b[FIN_BATCH];
#pragma unroll
		for (int k = 0; k < FIN_BATCH; ++k)
		{
			const uint32_t c = c0 + k * stride;
			const bool in = c < n;
			st[k] = in ? __ldg(cst + c) : 0u;
			pc0[k] = in ? __ldg(&man[c].pointCount) : 0u;
			a[k] = in ? __ldg(pA + c) : 0u;
			b[k] = in ? __ldg(pB + c) : 0u;
		}
#pragma unroll
		for (int k = 0; k < FIN_BATCH; ++k)
		{
			const uint32_t c = c0 + k * stride;
			if (c >= n)
				break;
			uint32_t mc = (st[k] >> 8) & 0xFFu;
			uint32_t pc = mc ? pc0[k] : 0u;
			touching += st[k] & 1u;
			manifolds += pc > 0 ? 1u : 0u;
			points += pc;
			for (uint32_t j = 1; j < mc && B.extraMan[cur]; ++j)
			{
				// Manifolds 1 and 2 of a mesh contact (b3MeshContact::m_stackManifolds).
				uint32_t xp = B.extraMan[cur][2 * (size_t)c + j - 1].pointCount;
				manifolds += xp > 0 ? 1u : 0u;
				points += xp;
			}
			uint32_t flags = (st[k] & 1u) | ((st[k] >> 16 & 1u) << 1) | (st[k] & 0xFF00u);
			B.contactOut[3 * c + 0] = a[k];
			B.contactOut[3 * c + 1] = b[k];
			B.contactOut[3 * c + 2] = flags;
		}
	}
	for (int o = 16; o > 0; o >>= 1)
	{
		touching += __shfl_xor_sync(0xffffffffu, touching, o);
		manifolds += __shfl_xor_sync(0xffffffffu, manifolds, o);
		points += __shfl_xor_sync(0xffffffffu, points, o);
	}
	// One atomic per counter and block: the counters are a handful of
	// addresses that every block adds to.
	__shared__ uint32_t sSum[3][FIN_THREADS / 32];
	const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (lane == 0)
	{
		sSum[0][warp] = touching;
		sSum[1][warp] = manifolds;
		sSum[2][warp] = points;
	}
	__syncthreads();
	if (threadIdx.x == 0)
	{
		touching = manifolds = points = 0;
		for (uint32_t w = 0; w < FIN_THREADS / 32; ++w)
		{
			touching += sSum[0][w];
			manifolds += sSum[1][w];
			points += sSum[2][w];
		}
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

// The pair-overflow status; with clearFound, also clears the previous
// contacts' found flags (k_diff sets them), only as many as the previous pass
// had.
__global__ void k_overflow_check(Buffers B, uint32_t cap, int clearFound, uint32_t nf)
{
	if (blockIdx.x == 0 && threadIdx.x == 0 && B.counters[CTR_RAW] > cap)
		atomicOr(&B.counters[CTR_STATUS], B3G_ST_PAIR_OVERFLOW);
	if (!clearFound)
		return;
	const uint32_t n = min(B.counters[CTR_PREV_PAIRS], cap);
	for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
		B.prevFound[p] = 0;
	// The proxies the broadphase re-inserted, one atomic per block.
	__shared__ uint32_t sMoved[32];
	uint32_t m = 0;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x)
		m += B.moved[i];
	for (int o = 16; o > 0; o >>= 1)
		m += __shfl_xor_sync(0xffffffffu, m, o);
	if ((threadIdx.x & 31) == 0)
		sMoved[threadIdx.x >> 5] = m;
	__syncthreads();
	if (threadIdx.x == 0)
	{
		m = 0;
		for (uint32_t w = 0; w < blockDim.x / 32; ++w)
			m += sMoved[w];
		if (m)
			atomicAdd(&B.counters[CTR_MOVED], m);
	}
}

} // namespace

FilterArgs make_filter_args(const b3g_ctx* c)
{
	FilterArgs F;
	F.mode = c->filterMode;
	F.jointKeys = c->dJointKeys;
	F.nJoints = c->nJoints;
	F.bodyJoint = c->dBodyJoint;
	F.vetoPrev = c->nVeto ? c->dVetoPrev : nullptr;
	F.nVeto = c->nVeto;
	F.rawDrop = c->dRawDrop;
	return F;
}

void launch_candidates(b3g_ctx* c, cudaStream_t s)
{
	Buffers& B = c->buf;
	uint32_t cap = c->cfg.max_contacts;
	k_overflow_check<<<1, 1, 0, s>>>(B, cap, 0, 0);
	k_candidates<<<persistent_blocks(8), 256, 0, s>>>(c->scene, B, make_filter_args(c), c->dCand, c->cur, cap,
		c->havePass ? 1 : 0);
}

void launch_candidate_pairs(b3g_ctx* c, uint32_t n, cudaStream_t s)
{
	if (n)
		k_candidate_pairs<<<persistent_blocks(2), 256, 0, s>>>(c->scene, c->buf, c->dCand, n, c->dCandPairs);
}

void launch_apply_veto(b3g_ctx* c, const uint32_t* rejected, uint32_t n, cudaStream_t s)
{
	if (n)
		k_apply_veto<<<persistent_blocks(2), 256, 0, s>>>(make_filter_args(c), rejected, n);
}

void launch_pairs_diff(b3g_ctx* c, cudaStream_t s)
{
	Buffers& B = c->buf;
	uint32_t cap = c->cfg.max_contacts;
	uint32_t cur = c->cur;
	uint32_t nf = c->nFixtures;
	cudaMemsetAsync(B.newOff, 0, sizeof(uint32_t) * (nf + 1), s);
	cudaMemsetAsync(B.newFill, 0, sizeof(uint32_t) * (nf + 1), s);
	k_overflow_check<<<persistent_blocks(2), 256, 0, s>>>(B, cap, 1, nf);
	k_diff<<<persistent_blocks(8), 256, 0, s>>>(c->scene, B, make_filter_args(c), cur, cap, nf,
		c->havePass ? 1 : 0);
	launch_order(c, s);
}

uint32_t pairs_diff_launches(const b3g_ctx* c)
{
	// overflow check (with the found flags and the moved count), diff, order
	return 2 + order_launches(c);
}

NPArgs make_np_args(b3g_ctx* c)
{
	Buffers& B = c->buf;
	uint32_t cur = c->cur, prev = cur ^ 1u;
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
	a.hcPost = B.hcPost;
	a.hcPostCount = B.counters + CTR_HC_POST;
	a.hcPostCap = c->cfg.max_contacts;
	a.hsPost = B.hsPost;
	a.hsPostCount = B.counters + CTR_HS_POST;
	a.extraCur = B.extraMan[cur];
	a.extraPrev = B.extraMan[prev];
	return a;
}

void launch_narrowphase(b3g_ctx* c, cudaStream_t s)
{
	Buffers& B = c->buf;
	uint32_t cap = c->cfg.max_contacts;
	// Mesh midphase on its own stream beside the bucketing and the convex
	// and hull kernels (joined before the mesh work items).
	const bool meshSide = !c->profiling && c->nMeshFix;
	cudaStream_t ms = meshSide ? c->meshStream : s;
	if (meshSide)
	{
		cudaEventRecord(c->meshFork, s);
		cudaStreamWaitEvent(ms, c->meshFork, 0);
	}
	launch_mesh_prepare(c, ms);
	if (meshSide)
		cudaEventRecord(c->meshJoin, ms);
	k_bucket<<<persistent_blocks(8), BUCKET_THREADS, 0, s>>>(c->scene, B, c->cur, cap);
	prof_mark(c, PM_BUCKETED, s);
	NPArgs a = make_np_args(c);
	// The buckets are disjoint sets of contacts: the hull-hull and
	// hull-triangle kernels run on a second stream beside the convex ones
	// (joined before the mesh work; a stream capture takes both branches).
	// Under profiling they stay on one stream so the stage marks hold.
	cudaStream_t side = c->profiling ? s : c->sideStream;
	if (side != s)
	{
		cudaEventRecord(c->forkEvent, s);
		cudaStreamWaitEvent(side, c->forkEvent, 0);
	}
	launch_hulls(a, B.bucketList + (size_t)BK_HULLS * cap, B.counters + CTR_BUCKET0 + BK_HULLS,
		c->maxUniqueEdges, c->tune, side);
	if (c->anyTriangle)
		launch_hull_triangles(a, B.bucketList + (size_t)BK_HULL_TRIANGLE * cap,
			B.counters + CTR_BUCKET0 + BK_HULL_TRIANGLE, c->maxUniqueEdges, c->tune, side);
	prof_mark(c, PM_HULLS, s);
	launch_apart(a, B.bucketList + (size_t)BK_APART * cap, B.counters + CTR_BUCKET0 + BK_APART, s);
	// The convex kernels (hull-sphere and hull-capsule each a scan kernel and
	// a follow-up kernel on the contacts the scan hands on) run beside the
	// hull-hull probe and SAT: the two branches take about as long.
	for (int k = 0; k < B3G_CONVEX_KERNELS; ++k)
		if (convex_bucket_possible(c, k))
			launch_convex_one(k, a, B.bucketList, B.counters + CTR_BUCKET0, cap, c->tune, s);
	prof_mark(c, PM_CONVEX, s);
	if (side != s)
	{
		cudaEventRecord(c->joinEvent, side);
		cudaStreamWaitEvent(s, c->joinEvent, 0);
	}
	if (meshSide)
		cudaStreamWaitEvent(s, c->meshJoin, 0);
	launch_mesh_collide(c, B.bucketList + (size_t)BK_MESH * cap, B.counters + CTR_BUCKET0 + BK_MESH, s);
	prof_mark(c, PM_MESH, s);
}

bool convex_bucket_possible(const b3g_ctx* c, int k)
{
	switch (k)
	{
	case 3:
	case 4:
		return c->anyTriangle;
	case 7:
		return c->anySensor;
	case 8:
		return c->asleep > 0;
	default:
		return true;
	}
}

void launch_finalize(b3g_ctx* c, cudaStream_t s)
{
	k_finalize<<<persistent_blocks(4), FIN_THREADS, 0, s>>>(c->scene, c->buf, c->cur, c->cfg.max_contacts,
		c->nFixtures);
}

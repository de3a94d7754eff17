// Contact-list order and the wake-ups of UpdateContacts.
//
// Bounce keeps its contacts in one linked list (b3ContactManager::m_contactList).
// FindPairs reports each new pair once, in ascending (proxy1, proxy2) order
// (broad_phase.h:158-206), and AddPair prepends it (contact_manager.cpp:105-111),
// so when UpdateContacts walks the list (contact_manager.cpp:214-287) it
// meets this pass's new contacts in DESCENDING pair order first, then every
// older contact in its previous order. The pass lays out its contact arrays
// in that order: contact index = position in the reference's list, and the
// host solver, the listener callbacks and the warm start see the reference's
// sequence.
//
// Which older contacts survive: UpdateContacts destroys a contact whose fat
// AABBs stopped overlapping only if one of its bodies is active (awake and not
// static) when the walk reaches it; a contact between two inactive bodies is
// skipped and kept as it is. Waking happens during the walk: a contact that
// starts or stops touching wakes both bodies (contact.cpp:249-254) and a
// destroyed contact with points wakes both (contact.cpp:108-126), so contacts
// LATER in the list see those bodies awake. With every non-static body awake
// (the common case) none of this changes anything and the layout is final
// after one pass over the contacts. Otherwise resolve_wakeups replays the walk:
// each wake event stores, per body, the earliest list position that woke it
// (atomicMin); a skipped contact becomes active iff one of its bodies was woken
// at an earlier position; activated contacts run the narrowphase (or are
// destroyed) and may wake more bodies; repeat until nothing changes. Each
// event found is one the sequential walk also makes (activity only grows), and
// every event of the walk is found by induction on its position, so the fixed
// point is the walk's result.

#include "collide_common.cuh"

namespace {

__device__ __forceinline__ void insert_contact(Buffers& B, uint32_t cur, uint32_t mask, uint32_t a, uint32_t b,
	uint32_t index)
{
	if (!pair_hash_insert(B.hashKeys[cur], B.hashVals[cur], mask + 1u, pair_key(a, b), index))
		atomicOr(&B.counters[CTR_STATUS], B3G_ST_HASH_OVERFLOW);
}

// The pass's table of (fixture pair -> contact), read by the next pass's
// lookup: sized to twice this pass's contacts (rounded up to a power of two,
// at most the allocation), so the table the lookups and inserts touch stays
// small enough for L2 rather than spanning the capacity's allocation.
__device__ __forceinline__ uint32_t hash_mask_for(const Buffers& B, uint32_t contacts)
{
	uint32_t slots = 1024u;
	while (slots < 2u * contacts && slots < B.hashCap)
		slots <<= 1;
	return min(slots, B.hashCap) - 1u;
}

// Clears the slots the table of this pass will use (total contacts, or the
// pass's new plus kept contacts when total is ~0u) and records its size.
__global__ void k_hash_clear(Buffers B, uint32_t cur, uint32_t cap, uint32_t total)
{
	const uint32_t n = total == ~0u ? min(B.counters[CTR_BEGUN] + B.counters[CTR_KEPT], cap) : total;
	const uint32_t mask = hash_mask_for(B, n);
	if (blockIdx.x == 0 && threadIdx.x == 0)
		B.hashMask[cur] = mask;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= mask; i += gridDim.x * blockDim.x)
		B.hashKeys[cur][i] = B3G_EMPTY_KEY;
}

// New contacts grouped by the smaller key rank, reversed (descending order).
__global__ void k_new_scatter(DevScene S, Buffers B, uint32_t nf)
{
	uint32_t n = B.counters[CTR_BEGUN];
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = B.newList[t];
		uint32_t ra = S.fixRank[B.rawA[c]], rb = S.fixRank[B.rawB[c]];
		uint32_t bucket = nf - 1u - min(ra, rb);
		uint32_t slot = B.newOff[bucket] + atomicAdd(&B.newFill[bucket], 1u);
		B.newTmp[slot] = c;
		B.newTmpMax[slot] = max(ra, rb);
	}
}

// Final place of each new contact: its group's offset plus the number of
// group members with a larger key (the ranks in a group are distinct).
__global__ void k_new_place(DevScene S, Buffers B, uint32_t cur, uint32_t nf, int havePrev)
{
	uint32_t n = B.counters[CTR_BEGUN];
	const uint32_t mask = B.hashMask[cur];
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = B.newTmp[t];
		uint32_t a = B.rawA[c], b = B.rawB[c];
		uint32_t mx = B.newTmpMax[t];
		uint32_t bucket = nf - 1u - min(S.fixRank[a], S.fixRank[b]);
		uint32_t beg = B.newOff[bucket], cnt = B.newFill[bucket];
		uint32_t rank = 0;
		for (uint32_t j = beg; j < beg + cnt; ++j)
			rank += B.newTmpMax[j] > mx ? 1u : 0u;
		uint32_t pos = beg + rank;
		B.pairA[cur][pos] = a;
		B.pairB[cur][pos] = b;
		B.prevIndex[pos] = -1;
		B.posKey[pos] = pos;
		insert_contact(B, cur, mask, a, b, pos);
	}
	if (!havePrev && blockIdx.x == 0 && threadIdx.x == 0)
		B.counters[CTR_PAIRS] = n;
}

__device__ __forceinline__ bool body_active(const DevScene& S, uint32_t b)
{
	return S.bodyAwake[b] != 0 && S.bodyType[b] != B3G_BODY_STATIC;
}

// Previous contacts: kept when their pair overlaps again, or when neither body
// is active (UpdateContacts skips the contact without testing the overlap).
// With filters (FilterArgs), a contact whose bodies a joint keeps apart or
// that the caller's filter rejects is destroyed whatever its bodies' state:
// UpdateContacts tests both before the inactive skip
// (contact_manager.cpp:176-199).
__global__ void k_kept(DevScene S, Buffers B, FilterArgs F, uint32_t cur, uint32_t cap)
{
	uint32_t prevBuf = cur ^ 1u;
	uint32_t n = min(B.counters[CTR_PREV_PAIRS], cap);
	for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
	{
		uint32_t kept = 1;
		uint32_t fa = B.pairA[prevBuf][p], fb = B.pairB[prevBuf][p];
		if (S.fixLife[fa] != FIX_LIVE || S.fixLife[fb] != FIX_LIVE)
			kept = 0; // a fixture was replaced or removed by a scene update
		else if (F.mode != 0 && ((F.vetoPrev && p < F.nVeto && F.vetoPrev[p]) ||
									joint_excluded(F, S.fixBody[fa], S.fixBody[fb])))
			kept = 0;
		else if (!B.prevFound[p])
		{
			uint32_t ba = S.fixBody[fa], bb = S.fixBody[fb];
			kept = (body_active(S, ba) || body_active(S, bb)) ? 0u : 1u;
		}
		B.keptScan[p] = kept;
	}
}

// Kept previous contacts follow the new ones in their previous order; the
// others are destroyed, listed in list order.
__global__ void k_layout_prev(Buffers B, uint32_t cur, uint32_t cap)
{
	const uint32_t mask = B.hashMask[cur];
	uint32_t prevBuf = cur ^ 1u;
	uint32_t n = min(B.counters[CTR_PREV_PAIRS], cap);
	uint32_t numNew = B.counters[CTR_BEGUN];
	uint32_t keptTotal = B.counters[CTR_KEPT];
	for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
	{
		uint32_t off = B.keptScan[p];
		uint32_t next = p + 1 < n ? B.keptScan[p + 1] : keptTotal;
		uint32_t a = B.pairA[prevBuf][p], b = B.pairB[prevBuf][p];
		if (next != off)
		{
			uint32_t pos = numNew + off;
			if (pos < cap)
			{
				B.pairA[cur][pos] = a;
				B.pairB[cur][pos] = b;
				B.prevIndex[pos] = (int32_t)p;
				B.posKey[pos] = numNew + p;
				insert_contact(B, cur, mask, a, b, pos);
			}
		}
		else
		{
			uint32_t slot = p - off;
			B.endedList[3 * slot + 0] = a;
			B.endedList[3 * slot + 1] = b;
			B.endedList[3 * slot + 2] = B.cstate[prevBuf][p];
		}
	}
	if (blockIdx.x == 0 && threadIdx.x == 0)
	{
		uint32_t total = numNew + keptTotal;
		if (total > cap)
			atomicOr(&B.counters[CTR_STATUS], B3G_ST_PAIR_OVERFLOW);
		B.counters[CTR_PAIRS] = min(total, cap);
		B.counters[CTR_ENDED] = n - keptTotal;
	}
}

// ---------------------------------------------------------------------------
// Wake-ups.

__device__ __forceinline__ bool sensor_pair(const DevScene& S, uint32_t fa, uint32_t fb)
{
	return ((S.fixFlags[fa] | S.fixFlags[fb]) & B3G_FIXTURE_SENSOR) != 0;
}

// b3Body::SetAwake(true) at list position pos: only bodies that start the
// pass asleep are tracked (static ones too: the call sets their flag).
__device__ __forceinline__ void wake_at(const DevScene& S, Buffers& B, uint32_t body, uint32_t pos, uint32_t& events)
{
	if (S.bodyAwake[body] == 0)
	{
		atomicMin(&B.tWake[body], pos);
		if (S.bodyType[body] != B3G_BODY_STATIC)
			++events;
	}
}

// Touching changes of the contacts in `list` (every contact when list is
// null: skipped contacts carry their state, so they show no change) and, with
// withEnded, the destroyed previous contacts that had points.
__global__ void k_wake_events(DevScene S, Buffers B, uint32_t cur, uint32_t cap, const uint32_t* list,
	const uint32_t* listCount, int withEnded)
{
	uint32_t prevBuf = cur ^ 1u;
	uint32_t events = 0;
	uint32_t n = list ? *listCount : min(B.counters[CTR_PAIRS], cap);
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = list ? list[t] : t;
		uint32_t fa = B.pairA[cur][c], fb = B.pairB[cur][c];
		if (sensor_pair(S, fa, fb))
			continue;
		int32_t prev = B.prevIndex[c];
		uint32_t was = prev >= 0 ? (B.cstate[prevBuf][prev] & 1u) : 0u;
		if ((B.cstate[cur][c] & 1u) != was)
		{
			wake_at(S, B, S.fixBody[fa], B.posKey[c], events);
			wake_at(S, B, S.fixBody[fb], B.posKey[c], events);
		}
	}
	if (withEnded)
	{
		uint32_t np = min(B.counters[CTR_PREV_PAIRS], cap);
		uint32_t numNew = B.counters[CTR_BEGUN];
		uint32_t keptTotal = B.counters[CTR_KEPT];
		for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x)
		{
			uint32_t next = p + 1 < np ? B.keptScan[p + 1] : keptTotal;
			if (next != B.keptScan[p])
				continue;
			uint32_t fa = B.pairA[prevBuf][p], fb = B.pairB[prevBuf][p];
			uint32_t mc = (B.cstate[prevBuf][p] >> 8) & 0xFFu;
			if (mc == 0 || B.man[prevBuf][p].pointCount == 0 || sensor_pair(S, fa, fb))
				continue;
			wake_at(S, B, S.fixBody[fa], numNew + p, events);
			wake_at(S, B, S.fixBody[fb], numNew + p, events);
		}
	}
	for (int o = 16; o > 0; o >>= 1)
		events += __shfl_xor_sync(0xffffffffu, events, o);
	if ((threadIdx.x & 31) == 0 && events)
		atomicAdd(&B.counters[CTR_WAKE_EVENTS], events);
}

__device__ __forceinline__ bool woken_before(const DevScene& S, const Buffers& B, uint32_t body, uint32_t pos)
{
	return S.bodyType[body] != B3G_BODY_STATIC && B.tWake[body] < pos;
}

// Skipped contacts whose body was woken at an earlier list position become
// active: a contact whose pair still overlaps runs the narrowphase (appended
// to the bucket lists and to wakeList), a retained one whose pair does not is
// destroyed now and wakes its bodies if it had points.
__global__ void k_wake_activate(DevScene S, Buffers B, uint32_t cur, uint32_t cap, uint32_t nInactive)
{
	uint32_t events = 0;
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nInactive; t += gridDim.x * blockDim.x)
	{
		if (B.activated[t])
			continue;
		uint32_t c = B.inactiveSave[t];
		uint32_t fa = B.pairA[cur][c], fb = B.pairB[cur][c];
		uint32_t ba = S.fixBody[fa], bb = S.fixBody[fb];
		uint32_t pos = B.posKey[c];
		if (!woken_before(S, B, ba, pos) && !woken_before(S, B, bb, pos))
			continue;
		B.activated[t] = 1;
		int32_t prev = B.prevIndex[c];
		if (prev >= 0 && !B.prevFound[prev])
		{
			B.lateDestroyed[c] = 1;
			atomicAdd(&B.counters[CTR_LATE_DESTROYED], 1u);
			uint32_t mc = (B.cstate[cur][c] >> 8) & 0xFFu;
			if (mc && B.man[cur][c].pointCount && !sensor_pair(S, fa, fb))
			{
				wake_at(S, B, ba, pos, events);
				wake_at(S, B, bb, pos, events);
			}
			continue;
		}
		uint32_t bk;
		if (S.fixType[fa] == B3G_SHAPE_MESH || S.fixType[fb] == B3G_SHAPE_MESH)
			bk = BK_MESH;
		else
			bk = sensor_pair(S, fa, fb) ? (uint32_t)BK_SENSOR : bucket_of(S.fixType[fa], S.fixType[fb]);
		if (bk >= BK_COUNT)
			continue;
		uint32_t slot = atomicAdd(&B.counters[CTR_BUCKET0 + bk], 1u);
		B.bucketList[(size_t)bk * cap + slot] = c;
		uint32_t w = atomicAdd(&B.counters[CTR_WAKE_ACTIVATED], 1u);
		B.wakeList[w] = c;
	}
	for (int o = 16; o > 0; o >>= 1)
		events += __shfl_xor_sync(0xffffffffu, events, o);
	if ((threadIdx.x & 31) == 0 && events)
		atomicAdd(&B.counters[CTR_WAKE_EVENTS], events);
}

// Awake flags after the pass (written back for the next pass) and the count
// of non-static bodies still asleep.
__global__ void k_awake_out(DevScene S, Buffers B, uint8_t* awake, uint32_t nb)
{
	uint32_t asleep = 0;
	for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
	{
		uint8_t on = (S.bodyAwake[b] != 0 || B.tWake[b] != 0xFFFFFFFFu) ? 1 : 0;
		awake[b] = on;
		if (!on && S.bodyType[b] != B3G_BODY_STATIC)
			++asleep;
	}
	for (int o = 16; o > 0; o >>= 1)
		asleep += __shfl_xor_sync(0xffffffffu, asleep, o);
	if ((threadIdx.x & 31) == 0 && asleep)
		atomicAdd(&B.counters[CTR_ASLEEP], asleep);
}

// Compaction after late destructions: keep flags without them (into kept2).
__global__ void k_compact_flags(Buffers B, uint32_t np, uint32_t numNew, uint32_t keptTotal, uint32_t* kept2)
{
	for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x)
	{
		uint32_t off = B.keptScan[p];
		uint32_t next = p + 1 < np ? B.keptScan[p + 1] : keptTotal;
		kept2[p] = (next != off && !B.lateDestroyed[numNew + off]) ? 1u : 0u;
	}
}

__global__ void k_compact_ended(Buffers B, uint32_t cur, uint32_t np, const uint32_t* kept2Scan, uint32_t kept2Total)
{
	uint32_t prevBuf = cur ^ 1u;
	for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x)
	{
		uint32_t off = kept2Scan[p];
		uint32_t next = p + 1 < np ? kept2Scan[p + 1] : kept2Total;
		if (next != off)
			continue;
		uint32_t slot = p - off;
		B.endedList[3 * slot + 0] = B.pairA[prevBuf][p];
		B.endedList[3 * slot + 1] = B.pairB[prevBuf][p];
		B.endedList[3 * slot + 2] = B.cstate[prevBuf][p];
	}
}

// Moves the kept previous contacts down over the destroyed ones. Their
// results for the old layout were copied to the start of the previous pass's
// state, cache and manifold arrays, which this pass no longer reads (its
// pair arrays stay intact and give each contact's fixtures).
__global__ void k_compact_move(Buffers B, uint32_t cur, uint32_t cap, uint32_t np, uint32_t numNew,
	uint32_t copied, const uint32_t* kept2Scan, uint32_t kept2Total)
{
	uint32_t prevBuf = cur ^ 1u;
	for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x)
	{
		uint32_t off2 = kept2Scan[p];
		uint32_t next2 = p + 1 < np ? kept2Scan[p + 1] : kept2Total;
		if (next2 == off2)
			continue;
		uint32_t old = B.keptScan[p];
		uint32_t pos = numNew + off2;
		if (old >= copied || pos >= cap)
			continue;
		B.pairA[cur][pos] = B.pairA[prevBuf][p];
		B.pairB[cur][pos] = B.pairB[prevBuf][p];
		B.prevIndex[pos] = (int32_t)p;
		B.posKey[pos] = numNew + p;
		B.cstate[cur][pos] = B.cstate[prevBuf][old];
		B.cache[cur][pos] = B.cache[prevBuf][old];
		B.man[cur][pos] = B.man[prevBuf][old];
		if (B.extraMan[cur])
		{
			B.extraMan[cur][2 * (size_t)pos] = B.extraMan[prevBuf][2 * (size_t)old];
			B.extraMan[cur][2 * (size_t)pos + 1] = B.extraMan[prevBuf][2 * (size_t)old + 1];
			B.meshAABB[cur][2 * (size_t)pos] = B.meshAABB[prevBuf][2 * (size_t)old];
			B.meshAABB[cur][2 * (size_t)pos + 1] = B.meshAABB[prevBuf][2 * (size_t)old + 1];
		}
	}
}

// Refills the pass's table with its first total contacts (after the
// wake-up rounds moved them), after k_hash_clear.
__global__ void k_rehash(Buffers B, uint32_t cur, uint32_t total)
{
	const uint32_t n = total;
	const uint32_t mask = B.hashMask[cur];
	for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
		insert_contact(B, cur, mask, B.pairA[cur][c], B.pairB[cur][c], c);
}

__global__ void k_set_counts(Buffers B, uint32_t pairs, uint32_t ended)
{
	B.counters[CTR_PAIRS] = pairs;
	B.counters[CTR_ENDED] = ended;
}

} // namespace

// After the previous-contact lookup: lays out this pass's contacts in list
// order, fills the hash table of this pass and lists the destroyed contacts.
FilterArgs make_filter_args(const b3g_ctx* c);

void launch_order(b3g_ctx* c, cudaStream_t s)
{
	Buffers& B = c->buf;
	const uint32_t cap = c->cfg.max_contacts, cur = c->cur, nf = c->nFixtures;
	const int havePrev = c->havePass ? 1 : 0;
	scan_exclusive(B.newOff, nf + 1, B.scanAux, B.counters + CTR_SCRATCH, B.counters + CTR_STATUS, s);
	if (havePrev)
	{
		k_kept<<<persistent_blocks(8), 256, 0, s>>>(c->scene, B, make_filter_args(c), cur, cap);
		scan_exclusive_device(B.keptScan, B.counters + CTR_PREV_PAIRS, cap, B.scanAux, B.counters + CTR_KEPT,
			B.counters + CTR_STATUS, s);
	}
	// New and kept counts known: the pass's table, filled as the contacts
	// take their places.
	k_hash_clear<<<persistent_blocks(8), 256, 0, s>>>(B, cur, cap, ~0u);
	k_new_scatter<<<persistent_blocks(4), 256, 0, s>>>(c->scene, B, nf);
	k_new_place<<<persistent_blocks(4), 256, 0, s>>>(c->scene, B, cur, nf, havePrev);
	if (havePrev)
		k_layout_prev<<<persistent_blocks(8), 256, 0, s>>>(B, cur, cap);
}

uint32_t order_launches(const b3g_ctx* c)
{
	// scan, scatter, place; kept, scan, layout of the previous contacts;
	// the table's clear
	return 3 + (c->havePass ? 3 : 0) + 1;
}

// Host-driven replay of the wake-ups; runs only when some non-static body is
// asleep at the start of the pass. Reads the counters back once per round.
int resolve_wakeups(b3g_ctx* c, cudaStream_t s)
{
	Buffers& B = c->buf;
	const uint32_t cap = c->cfg.max_contacts, cur = c->cur;
	uint32_t launches = 0;
	uint32_t h[CTR_COUNT];
	auto fetch = [&]() -> bool {
		return cudaMemcpyAsync(h, B.counters, sizeof(h), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
			cudaStreamSynchronize(s) == cudaSuccess;
	};
	cudaMemsetAsync(B.tWake, 0xFF, sizeof(uint32_t) * c->nBodies, s);
	k_wake_events<<<persistent_blocks(4), 256, 0, s>>>(c->scene, B, cur, cap, nullptr, nullptr,
		c->havePass ? 1 : 0);
	++launches;
	if (!fetch())
		return B3G_E_CUDA;
	const uint32_t nInactive = h[CTR_BUCKET0 + BK_INACTIVE];
	uint32_t late = 0;
	if (h[CTR_WAKE_EVENTS] != 0 && nInactive != 0)
	{
		// The bucket lists are reused for the contacts each round activates.
		cudaMemcpyAsync(B.inactiveSave, B.bucketList + (size_t)BK_INACTIVE * cap, sizeof(uint32_t) * nInactive,
			cudaMemcpyDeviceToDevice, s);
		cudaMemsetAsync(B.activated, 0, sizeof(uint32_t) * nInactive, s);
		cudaMemsetAsync(B.lateDestroyed, 0, sizeof(uint32_t) * cap, s);
		NPArgs a = make_np_args(c);
		// Every round but the last activates at least one skipped contact.
		for (uint32_t round = 0; round <= nInactive; ++round)
		{
			cudaMemsetAsync(B.counters + CTR_BUCKET0, 0, sizeof(uint32_t) * BK_COUNT, s);
			cudaMemsetAsync(B.counters + CTR_WAKE_ACTIVATED, 0, sizeof(uint32_t), s);
			cudaMemsetAsync(B.counters + CTR_HULL_MISS, 0, sizeof(uint32_t), s);
			k_wake_activate<<<persistent_blocks(4), 256, 0, s>>>(c->scene, B, cur, cap, nInactive);
			++launches;
			if (!fetch())
				return B3G_E_CUDA;
			const uint32_t act = h[CTR_WAKE_ACTIVATED];
			const bool lateNow = h[CTR_LATE_DESTROYED] != late;
			late = h[CTR_LATE_DESTROYED];
			if (act == 0 && !lateNow)
				break;
			if (act)
			{
				launch_convex_buckets(a, B.bucketList, B.counters + CTR_BUCKET0, cap, c->tune, s);
				launch_hulls(a, B.bucketList + (size_t)BK_HULLS * cap, B.counters + CTR_BUCKET0 + BK_HULLS,
					c->maxUniqueEdges, c->tune, s);
				launch_hull_triangles(a, B.bucketList + (size_t)BK_HULL_TRIANGLE * cap,
					B.counters + CTR_BUCKET0 + BK_HULL_TRIANGLE, c->maxUniqueEdges, c->tune, s);
				launch_mesh_collide(c, B.bucketList + (size_t)BK_MESH * cap, B.counters + CTR_BUCKET0 + BK_MESH, s);
				launches += c->nMeshFix ? 3 : 0;
				k_wake_events<<<persistent_blocks(4), 256, 0, s>>>(c->scene, B, cur, cap, B.wakeList,
					B.counters + CTR_WAKE_ACTIVATED, 0);
				launches += B3G_CONVEX_KERNELS + 2 + 1 + 1;
			}
		}
		cudaMemsetAsync(B.counters + CTR_BUCKET0, 0, sizeof(uint32_t) * BK_COUNT, s);
	}
	if (late)
	{
		// Rare: a retained contact whose pair no longer overlaps was destroyed
		// by a wake-up. Recompute the kept set and move the contacts after it.
		const uint32_t np = h[CTR_PREV_PAIRS], numNew = h[CTR_BEGUN], keptTotal = h[CTR_KEPT];
		const uint32_t prevBuf = cur ^ 1u;
		// Contacts of the old layout that fit the capacity (all of them unless
		// the pass already reported an overflow).
		const uint32_t copied = std::min(keptTotal, cap - std::min(numNew, cap));
		uint32_t* kept2 = B.newTmp;
		k_compact_flags<<<persistent_blocks(4), 256, 0, s>>>(B, np, numNew, keptTotal, kept2);
		scan_exclusive(kept2, np, B.scanAux, B.counters + CTR_SCRATCH, B.counters + CTR_STATUS, s);
		if (!fetch())
			return B3G_E_CUDA;
		const uint32_t kept2Total = h[CTR_SCRATCH];
		k_compact_ended<<<persistent_blocks(4), 256, 0, s>>>(B, cur, np, kept2, kept2Total);
		if (copied)
		{
			cudaMemcpyAsync(B.cstate[prevBuf], B.cstate[cur] + numNew, sizeof(uint32_t) * copied,
				cudaMemcpyDeviceToDevice, s);
			cudaMemcpyAsync(B.cache[prevBuf], B.cache[cur] + numNew, sizeof(uint4) * copied,
				cudaMemcpyDeviceToDevice, s);
			cudaMemcpyAsync(B.man[prevBuf], B.man[cur] + numNew, sizeof(DevManifold) * copied,
				cudaMemcpyDeviceToDevice, s);
			if (B.extraMan[cur])
			{
				cudaMemcpyAsync(B.extraMan[prevBuf], B.extraMan[cur] + 2 * (size_t)numNew,
					sizeof(DevManifold) * 2 * copied, cudaMemcpyDeviceToDevice, s);
				cudaMemcpyAsync(B.meshAABB[prevBuf], B.meshAABB[cur] + 2 * (size_t)numNew,
					sizeof(float4) * 2 * copied, cudaMemcpyDeviceToDevice, s);
			}
		}
		k_compact_move<<<persistent_blocks(4), 256, 0, s>>>(B, cur, cap, np, numNew, copied, kept2, kept2Total);
		const uint32_t total = std::min(numNew + kept2Total, cap);
		k_hash_clear<<<persistent_blocks(8), 256, 0, s>>>(B, cur, cap, total);
		k_rehash<<<persistent_blocks(8), 256, 0, s>>>(B, cur, total);
		k_set_counts<<<1, 1, 0, s>>>(B, total, np - kept2Total);
		launches += 1 + 3 + 1 + 1 + 1 + 1;
	}
	cudaMemsetAsync(B.counters + CTR_ASLEEP, 0, sizeof(uint32_t), s);
	const int nbBlocks = (int)std::min<uint32_t>((c->nBodies + 255) / 256, 148u * 4u);
	k_awake_out<<<nbBlocks, 256, 0, s>>>(c->scene, B, c->dBodyAwake, c->nBodies);
	++launches;
	if (!fetch())
		return B3G_E_CUDA;
	c->asleep = h[CTR_ASLEEP];
	// Bodies past the processed prefix keep their flags.
	if (c->hAwake.size() >= c->nBodies &&
		cudaMemcpy(c->hAwake.data(), c->dBodyAwake, c->nBodies, cudaMemcpyDeviceToHost) != cudaSuccess)
		return B3G_E_CUDA;
	for (uint32_t b = c->nBodies; b < c->hAwake.size(); ++b)
		if (c->hAwake[b] == 0 && c->hBodyType[b] != B3G_BODY_STATIC)
			++c->asleep;
	c->launches += launches;
	return cudaGetLastError() == cudaSuccess ? B3G_OK : B3G_E_CUDA;
}

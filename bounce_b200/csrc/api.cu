// C ABI of the pipeline (include/b3g.h): context lifetime, scene upload, the
// pass sequence and result transfers. Device memory is allocated once in
// b3g_create for the configured capacities.

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "collide_common.cuh"

namespace {

int fail(b3g_ctx* c, int code, const char* fmt, ...)
{
	if (c)
	{
		char buf[512];
		va_list ap;
		va_start(ap, fmt);
		vsnprintf(buf, sizeof(buf), fmt, ap);
		va_end(ap);
		c->err = buf;
	}
	return code;
}

// Non-static bodies with a cleared awake flag.
uint32_t count_asleep(const b3g_ctx* c, const uint8_t* awake)
{
	uint32_t n = 0;
	for (size_t i = 0; i < c->hBodyType.size(); ++i)
		n += (awake[i] == 0 && c->hBodyType[i] != B3G_BODY_STATIC) ? 1u : 0u;
	return n;
}

#define CK(call)                                                                                 \
	do                                                                                           \
	{                                                                                            \
		cudaError_t e_ = (call);                                                                 \
		if (e_ != cudaSuccess)                                                                   \
			return fail(c, B3G_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));         \
	} while (0)

template <class T>
cudaError_t dalloc(T** p, size_t count)
{
	if (count == 0)
		count = 1;
	return cudaMalloc((void**)p, sizeof(T) * count);
}

template <class T>
void dfree(T*& p)
{
	if (p)
		cudaFree((void*)p);
	p = nullptr;
}

// Captured passes become invalid when the scene or a launch shape changes.
void destroy_graphs(b3g_ctx* c)
{
	// Whatever made the captured passes stale may have changed the proxy set:
	// the next pass rebuilds the LBVH.
	c->treeForce = true;
	for (int i = 0; i < 2; ++i)
		for (int j = 0; j < 2; ++j)
			for (int r = 0; r < 2; ++r)
			{
				PassGraph& g = c->graphs[i][j][r];
				if (g.exec)
					cudaGraphExecDestroy(g.exec);
				if (g.graph)
					cudaGraphDestroy(g.graph);
				g = PassGraph{nullptr, nullptr, nullptr, nullptr, nullptr};
			}
}

// Launch shapes before any tuning.
void default_tuning(Tune& t)
{
	for (int k = 0; k < B3G_CONVEX_KERNELS; ++k)
		t.v[B3G_TUNE_CONVEX + k] = 4;
	// The hull-sphere face scan holds few registers: twice the blocks fit.
	t.v[B3G_TUNE_CONVEX + 5] = 8;
	t.v[B3G_TUNE_PROBE] = 4;
	t.v[B3G_TUNE_SAT_WARPS] = 4;
	t.v[B3G_TUNE_SAT_BLOCKS] = 2;
	t.v[B3G_TUNE_TRAVERSE] = 128;
}

uint32_t pow2_at_least(uint32_t v)
{
	uint32_t p = 1;
	while (p < v)
		p <<= 1;
	return p;
}

__global__ void k_pass_begin(uint32_t* counters, int havePass, uint32_t cap)
{
	uint32_t i = threadIdx.x;
	if (i >= CTR_COUNT)
		return;
	uint32_t pairs = counters[CTR_PAIRS];
	__syncthreads();
	if (i == CTR_PREV_PAIRS)
		counters[i] = havePass ? min(pairs, cap) : 0u;
	else
		counters[i] = 0;
}

// b3TriangleHull::Set (triangle_hull.h:36-69) for every triangle fixture:
// vertices, the two face planes (normal from (B - A) x (C - A), through the
// centroid) and the centroid.
__global__ void k_triangle_hulls(DevScene S, uint32_t nf, float4* tri)
{
	uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
	if (f >= nf || S.fixType[f] != B3G_SHAPE_TRIANGLE)
		return;
	float4 p0 = S.fixParams[3 * f], p1 = S.fixParams[3 * f + 1], p2 = S.fixParams[3 * f + 2];
	V3 A = V3{p0.x, p0.y, p0.z}, B = V3{p0.w, p1.x, p1.y}, C = V3{p1.z, p1.w, p2.x};
	V3 centroid = ((A + B) + C) / 3.0f;
	V3 N = normalized(cross(B - A, C - A));
	float4* t = tri + 6 * (size_t)f;
	t[0] = make_float4(A.x, A.y, A.z, 0.0f);
	t[1] = make_float4(B.x, B.y, B.z, 0.0f);
	t[2] = make_float4(C.x, C.y, C.z, 0.0f);
	t[3] = make_float4(N.x, N.y, N.z, dot(N, centroid));
	V3 M = -N;
	t[4] = make_float4(M.x, M.y, M.z, dot(M, centroid));
	t[5] = make_float4(centroid.x, centroid.y, centroid.z, 0.0f);
}

// Manifolds with points per contact: the first, and for a mesh contact its
// other cluster manifolds.
__global__ void k_touch_flags(const DevManifold* man, const DevManifold* extra, const uint32_t* cstate, uint32_t n,
	uint32_t* flags)
{
	uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= n)
		return;
	uint32_t mc = (cstate[c] >> 8) & 0xFFu;
	uint32_t k = 0;
	for (uint32_t j = 0; j < mc && j < 3; ++j)
	{
		const DevManifold& m = j == 0 ? man[c] : extra[2 * (size_t)c + j - 1];
		k += m.pointCount > 0 ? 1u : 0u;
	}
	flags[c] = k;
}

__global__ void k_touch_scatter(const DevManifold* man, const DevManifold* extra, const uint32_t* cstate,
	const uint32_t* offsets, uint32_t n, uint32_t* index, DevManifold* out)
{
	uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= n)
		return;
	uint32_t mc = (cstate[c] >> 8) & 0xFFu;
	uint32_t o = offsets[c];
	for (uint32_t j = 0; j < mc && j < 3; ++j)
	{
		const DevManifold& m = j == 0 ? man[c] : extra[2 * (size_t)c + j - 1];
		if (m.pointCount == 0)
			continue;
		index[o] = c;
		out[o] = m;
		++o;
	}
}

// Packed touching output: per manifold with points, its 32-byte tail
// (pointCount, impulses, speeds: the b3Manifold fields after points) then
// its pointCount points (72 bytes each).
__global__ void k_pack_sizes(const DevManifold* man, const DevManifold* extra, const uint32_t* cstate, uint32_t n,
	uint32_t* count, uint32_t* bytes)
{
	uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= n)
		return;
	uint32_t mc = (cstate[c] >> 8) & 0xFFu;
	uint32_t k = 0, b = 0;
	for (uint32_t j = 0; j < mc && j < 3; ++j)
	{
		const DevManifold& m = j == 0 ? man[c] : extra[2 * (size_t)c + j - 1];
		uint32_t pc = m.pointCount;
		k += pc > 0 ? 1u : 0u;
		b += pc > 0 ? 32u + 72u * pc : 0u;
	}
	count[c] = k;
	bytes[c] = b;
}

__global__ void k_pack_scatter(const DevManifold* man, const DevManifold* extra, const uint32_t* cstate, uint32_t n,
	const uint32_t* countOff, const uint32_t* byteOff, uint32_t* index, unsigned long long* out)
{
	uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= n)
		return;
	uint32_t mc = (cstate[c] >> 8) & 0xFFu;
	uint32_t o = countOff[c];
	size_t w = byteOff[c] / 8; // every record is a multiple of 8 bytes
	for (uint32_t j = 0; j < mc && j < 3; ++j)
	{
		const DevManifold& m = j == 0 ? man[c] : extra[2 * (size_t)c + j - 1];
		uint32_t pc = m.pointCount;
		if (pc == 0)
			continue;
		index[o++] = c;
		const unsigned long long* tail = reinterpret_cast<const unsigned long long*>(&m.pointCount);
		for (int q = 0; q < 4; ++q)
			out[w++] = tail[q];
		const unsigned long long* pts = reinterpret_cast<const unsigned long long*>(m.points);
		for (uint32_t q = 0; q < 9 * pc; ++q)
			out[w++] = pts[q];
	}
}

// Contact edges of the fixtures: record 2c is (fixture A of contact c, c),
// 2c + 1 is (fixture B, c); counts per fixture.
__global__ void k_edge_records(const uint32_t* pairA, const uint32_t* pairB, uint32_t n, unsigned long long* keys,
	uint32_t* vals, uint32_t* counts)
{
	uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= n)
		return;
	uint32_t a = pairA[c], b = pairB[c];
	keys[2 * (size_t)c] = a;
	vals[2 * (size_t)c] = c;
	keys[2 * (size_t)c + 1] = b;
	vals[2 * (size_t)c + 1] = c;
	atomicAdd(&counts[a], 1u);
	atomicAdd(&counts[b], 1u);
}

} // namespace

// ---------------------------------------------------------------------------
// Stage profiling.

static const char* kStageNames[PROF_STAGES] = {
	"upload",        // body state copy + counter reset
	"sync",          // fat-AABB update (MoveProxy rule)
	"sort",          // bounds, Morton keys, radix sort
	"build",         // Karras tree, leaves, ropes, refit
	"traverse",      // pair count, scan, pair write
	"diff",          // persistent-pair hash, ended contacts
	"bucket",        // narrowphase buckets (and the mesh midphase)
	"narrow_hulls",  // hull-hull and hull-triangle kernels
	"narrow_convex", // apart, sphere/capsule/hull-sphere/hull-capsule/sensor/inactive kernels
	"narrow_mesh",   // mesh work items and clustering
	"finalize",      // counters, contact records
};
// Under profiling every kernel of a pass runs on the pass's stream, one after
// the other, so that each stage's events enclose its own kernels; without
// profiling the hull and mesh stages overlap the convex stage on their own
// streams, and a pass takes less than the sum of the stages.

void prof_mark(b3g_ctx* c, int mark, cudaStream_t s)
{
	if (!c->profiling)
		return;
	size_t slot = (size_t)(c->profPass % PROF_RING);
	cudaEventRecord(c->profEvents[slot * PROF_MARKS + mark], s);
}

static void prof_harvest_one(b3g_ctx* c)
{
	size_t slot = (size_t)(c->profHarvest % PROF_RING);
	cudaEvent_t* ev = c->profEvents + slot * PROF_MARKS;
	cudaEventSynchronize(ev[PROF_MARKS - 1]);
	for (int k = 0; k < PROF_STAGES; ++k)
	{
		float ms = 0.0f;
		if (cudaEventElapsedTime(&ms, ev[k], ev[k + 1]) == cudaSuccess)
		{
			c->profMs[k] += ms;
			c->profCount[k] += 1;
		}
	}
	++c->profHarvest;
}

static int prof_begin_pass(b3g_ctx* c)
{
	// Reuse a ring slot only after its events were read.
	while (c->profPass - c->profHarvest >= (uint64_t)PROF_RING)
		prof_harvest_one(c);
	return B3G_OK;
}

extern "C" int b3g_set_profiling(b3g_ctx* c, int enable)
{
	if (!c)
		return B3G_E_INVALID;
	CK(cudaSetDevice(c->device));
	if (enable && !c->profEvents)
	{
		c->profEvents = new cudaEvent_t[PROF_RING * PROF_MARKS];
		for (int i = 0; i < PROF_RING * PROF_MARKS; ++i)
			CK(cudaEventCreate(&c->profEvents[i]));
	}
	c->profiling = enable != 0;
	c->profPass = c->profHarvest = 0;
	for (int k = 0; k < 16; ++k)
	{
		c->profMs[k] = 0.0;
		c->profCount[k] = 0;
	}
	return B3G_OK;
}

extern "C" int b3g_get_profile(b3g_ctx* c, double* ms, uint32_t* passes, uint32_t capacity)
{
	if (!c || !ms || !passes)
		return fail(c, B3G_E_INVALID, "null argument");
	CK(cudaSetDevice(c->device));
	while (c->profHarvest < c->profPass)
		prof_harvest_one(c);
	uint32_t n = std::min<uint32_t>(capacity, PROF_STAGES);
	for (uint32_t k = 0; k < n; ++k)
	{
		ms[k] = c->profMs[k];
		passes[k] = c->profCount[k];
	}
	return (int)n;
}

extern "C" const char* b3g_stage_name(uint32_t stage)
{
	return stage < PROF_STAGES ? kStageNames[stage] : nullptr;
}

extern "C" int b3g_get_totals(b3g_ctx* c, uint64_t* out, int reset)
{
	if (!c || !out)
		return fail(c, B3G_E_INVALID, "null argument");
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	CK(cudaDeviceSynchronize());
	unsigned long long t[8];
	CK(cudaMemcpy(t, c->buf.totals, sizeof(t), cudaMemcpyDeviceToHost));
	for (int k = 0; k < 6; ++k)
		out[k] = t[k];
	out[6] = c->launches;
	out[7] = c->graphLaunches;
	if (reset)
	{
		CK(cudaMemset(c->buf.totals, 0, sizeof(t)));
		c->launches = 0;
		c->graphLaunches = 0;
	}
	return B3G_OK;
}

// ---------------------------------------------------------------------------

extern "C" int b3g_create(const b3g_config* cfg, b3g_ctx** out)
{
	if (!cfg || !out)
		return B3G_E_INVALID;
	*out = nullptr;
	b3g_ctx* c = new b3g_ctx();
	std::memset(&c->scene, 0, sizeof(c->scene));
	std::memset(&c->buf, 0, sizeof(c->buf));
	c->cfg = *cfg;
	c->device = cfg->device;
	c->stream = nullptr;
	c->nHulls = c->nBodies = c->nFixtures = 0;
	c->nWorlds = 1;
	c->hullVerts = c->hullEdges = c->hullFaces = 0;
	c->maxUniqueEdges = 0;
	c->cur = 0;
	c->creationPass = true;
	c->havePass = false;
	c->impulsesLoaded = false;
	c->dHulls = nullptr;
	c->dHverts = nullptr;
	c->dHedges = nullptr;
	c->dHfaces = nullptr;
	c->dHplanes = nullptr;
	c->dBodyWorld = c->dBodyType = nullptr;
	c->dBodyAwake = nullptr;
	c->dBodyState = nullptr;
	c->dFixBody = c->dFixType = c->dFixHull = c->dFixFlags = c->dFixKey = c->dFixRank = nullptr;
	c->dFixLife = nullptr;
	c->dFixTri = nullptr;
	c->dFixWing = nullptr;
	c->triSlots = 0;
	c->nMeshes = 0;
	c->dMeshes = nullptr;
	c->dMeshVerts = nullptr;
	c->dMeshTris = nullptr;
	c->dMeshWings = nullptr;
	c->dMeshNodes = nullptr;
	c->dMeshFix = nullptr;
	c->nMeshFix = 0;
	c->capBodies = c->capFixtures = 0;
	c->keysAreIndex = true;
	for (int i = 0; i < B3G_STAGE_RING; ++i)
		c->stage[i] = StageSlot{nullptr, nullptr, 0, nullptr};
	c->stageNext = 0;
	c->dWorldCounts = nullptr;
	c->dUpdateBad = nullptr;
	c->fixTypeStale = false;
	c->asleep = 0;
	c->graphLaunches = 0;
	c->lastPassImpulses = false;
	for (int i = 0; i < 2; ++i)
		for (int j = 0; j < 2; ++j)
			for (int r = 0; r < 2; ++r)
				c->graphs[i][j][r] = PassGraph{nullptr, nullptr, nullptr, nullptr, nullptr};
	default_tuning(c->tune);
	c->dFixParams = nullptr;
	c->dFixBound = nullptr;
	c->hCounters = nullptr;
	c->profiling = false;
	c->launches = 0;
	c->profPass = c->profHarvest = 0;
	c->profEvents = nullptr;
	c->dJointKeys = nullptr;
	c->nJoints = c->jointCap = 0;
	c->dBodyJoint = nullptr;
	c->bodyJointCap = 0;
	c->dVetoPrev = nullptr;
	c->nVeto = 0;
	c->dRawDrop = nullptr;
	c->dCand = nullptr;
	c->dCandPairs = nullptr;
	c->nCand = 0;
	c->candFetched = false;
	c->passOpen = false;
	c->filterMode = 0;
	c->walkLimit = 0;
	c->treeLeaves = 0;
	c->treeWorlds = 0;
	c->treeInterval = B3G_TREE_REBUILD_INTERVAL;
	c->treeSince = 0;
	c->treeForce = true;
	c->treeRebuild = true;
	if (cfg->max_proxies == 0 || cfg->max_contacts == 0)
	{
		delete c;
		return B3G_E_INVALID;
	}
	int rc = B3G_OK;
	auto step = [&](cudaError_t e, const char* what) {
		if (rc == B3G_OK && e != cudaSuccess)
			rc = fail(c, B3G_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
	};
	step(cudaSetDevice(cfg->device), "cudaSetDevice");
	step(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
	step(cudaStreamCreateWithFlags(&c->copyStream, cudaStreamNonBlocking), "cudaStreamCreate");
	step(cudaEventCreateWithFlags(&c->copyReady, cudaEventDisableTiming), "cudaEventCreate");
	step(cudaEventCreateWithFlags(&c->copyDone, cudaEventDisableTiming), "cudaEventCreate");
	step(cudaStreamCreateWithFlags(&c->sideStream, cudaStreamNonBlocking), "cudaStreamCreate");
	step(cudaEventCreateWithFlags(&c->forkEvent, cudaEventDisableTiming), "cudaEventCreate");
	step(cudaEventCreateWithFlags(&c->joinEvent, cudaEventDisableTiming), "cudaEventCreate");
	step(cudaStreamCreateWithFlags(&c->meshStream, cudaStreamNonBlocking), "cudaStreamCreate");
	step(cudaEventCreateWithFlags(&c->meshFork, cudaEventDisableTiming), "cudaEventCreate");
	step(cudaEventCreateWithFlags(&c->meshJoin, cudaEventDisableTiming), "cudaEventCreate");
	const uint32_t P = cfg->max_proxies, C = cfg->max_contacts;
	Buffers& B = c->buf;
	step(dalloc(&B.fatLo, P), "alloc");
	step(dalloc(&B.fatHi, P), "alloc");
	step(dalloc(&B.moved, P), "alloc");
	step(dalloc(&B.keysA, P), "alloc");
	step(dalloc(&B.keysB, P), "alloc");
	step(dalloc(&B.valsA, P), "alloc");
	step(dalloc(&B.valsB, P), "alloc");
	step(dalloc(&B.sortHist, 256 * (9 + 8 * ((size_t)(P + 1023) / 1024 + 1))), "alloc"); // digit counts, tile status
	step(dalloc(&B.sceneBounds, 8), "alloc");
	step(dalloc(&B.nodeLo, 2 * P), "alloc");
	step(dalloc(&B.nodeHi, 2 * P), "alloc");
	step(dalloc(&B.nodeLeft, 2 * P), "alloc");
	step(dalloc(&B.nodeRight, 2 * P), "alloc");
	step(dalloc(&B.nodeRope, 2 * P), "alloc");
	step(dalloc(&B.nodeFirst, 2 * P), "alloc");
	step(dalloc(&B.leafData, P), "alloc");
	step(dalloc(&B.leafOf, P), "alloc");
	step(dalloc(&B.nodeParent, 2 * P), "alloc");
	step(dalloc(&B.nodeEnd, P), "alloc");
	step(dalloc(&B.splitRight, P), "alloc");
	step(dalloc(&B.refitFlag, P), "alloc");
	step(dalloc(&B.worldEnd, P), "alloc");
	step(dalloc(&B.proxyInfo, P), "alloc");
	step(dalloc(&B.leafCount, std::max(P, C)), "alloc");
	step(dalloc(&B.pairScratch, 2 * B3G_TRAV_SLOTS * (size_t)P), "alloc"); // uint2 records per leaf
	step(dalloc(&B.scanAux, scan_aux_words(std::max(P, C) + 1)), "alloc");
	for (int k = 0; k < 2; ++k)
	{
		step(dalloc(&B.pairA[k], C), "alloc");
		step(dalloc(&B.pairB[k], C), "alloc");
		step(dalloc(&B.cstate[k], C), "alloc");
		step(dalloc(&B.cache[k], C), "alloc");
		step(dalloc(&B.man[k], C), "alloc");
	}
	B.hashCap = pow2_at_least(2 * C);
	step(dalloc(&B.hashMask, 2), "alloc");
	for (int k = 0; k < 2; ++k)
	{
		step(dalloc(&B.hashKeys[k], B.hashCap), "alloc");
		step(dalloc(&B.hashVals[k], B.hashCap), "alloc");
	}
	step(dalloc(&B.prevIndex, C), "alloc");
	step(dalloc(&B.prevFound, C), "alloc");
	step(dalloc(&B.rawA, C), "alloc");
	step(dalloc(&B.rawB, C), "alloc");
	step(dalloc(&B.travOverflow, C), "alloc");
	step(dalloc(&B.newList, C), "alloc");
	step(dalloc(&B.newOff, (size_t)P + 1), "alloc");
	step(dalloc(&B.newFill, (size_t)P + 1), "alloc");
	step(dalloc(&B.newTmp, C), "alloc");
	step(dalloc(&B.newTmpMax, C), "alloc");
	step(dalloc(&B.keptScan, C), "alloc");
	step(dalloc(&B.posKey, C), "alloc");
	step(dalloc(&B.wakeList, C), "alloc");
	step(dalloc(&B.inactiveSave, C), "alloc");
	step(dalloc(&B.activated, C), "alloc");
	step(dalloc(&B.lateDestroyed, C), "alloc");
	step(dalloc(&B.bucketList, (size_t)BK_COUNT * C), "alloc");
	step(dalloc(&B.missList, C), "alloc");
	step(dalloc(&B.hcPost, 2 * (size_t)C), "alloc");
	step(dalloc(&B.hsPost, C), "alloc");
	step(dalloc(&B.counters, CTR_COUNT), "alloc");
	step(dalloc(&c->dUpdateBad, 1), "alloc");
	step(dalloc(&B.totals, 8), "alloc");
	step(dalloc(&B.endedList, 3 * (size_t)C), "alloc");
	step(dalloc(&B.touchIndex, C), "alloc");
	step(dalloc(&B.touchMan, C), "alloc");
	step(dalloc(&B.contactOut, 3 * (size_t)C), "alloc");
	// The packed result copies' per-contact byte counts, allocated here so no
	// fetch pays for an allocation.
	step(dalloc(&c->touchBytes, C), "alloc");
	step(dalloc(&B.impulseNormal, 4 * (size_t)C), "alloc");
	step(dalloc(&B.impulseTangent, 2 * (size_t)C), "alloc");
	step(dalloc(&B.impulseMotor, C), "alloc");
	step(cudaMallocHost((void**)&c->hCounters, sizeof(uint32_t) * CTR_COUNT), "cudaMallocHost");
	if (rc == B3G_OK)
	{
		step(cudaMemsetAsync(B.counters, 0, sizeof(uint32_t) * CTR_COUNT, c->stream), "memset");
		step(cudaMemsetAsync(c->dUpdateBad, 0, sizeof(uint32_t), c->stream), "memset");
		step(cudaMemsetAsync(B.totals, 0, sizeof(unsigned long long) * 8, c->stream), "memset");
		step(cudaMemsetAsync(B.cstate[0], 0, sizeof(uint32_t) * C, c->stream), "memset");
		step(cudaMemsetAsync(B.cstate[1], 0, sizeof(uint32_t) * C, c->stream), "memset");
		step(cudaMemsetAsync(B.hashKeys[0], 0xFF, sizeof(unsigned long long) * B.hashCap, c->stream), "memset");
		step(cudaMemsetAsync(B.hashKeys[1], 0xFF, sizeof(unsigned long long) * B.hashCap, c->stream), "memset");
		const uint32_t fullMask[2] = {B.hashCap - 1u, B.hashCap - 1u};
		step(cudaMemcpyAsync(B.hashMask, fullMask, sizeof(fullMask), cudaMemcpyHostToDevice, c->stream), "memcpy");
		step(cudaStreamSynchronize(c->stream), "sync");
	}
	if (rc != B3G_OK)
	{
		std::string msg = c->err;
		b3g_destroy(c);
		fprintf(stderr, "b3g_create: %s\n", msg.c_str());
		return rc;
	}
	*out = c;
	return B3G_OK;
}

extern "C" void b3g_destroy(b3g_ctx* c)
{
	if (!c)
		return;
	cudaSetDevice(c->device);
	if (c->stream)
		cudaStreamSynchronize(c->stream);
	destroy_graphs(c);
	Buffers& B = c->buf;
	dfree(B.fatLo);
	dfree(B.fatHi);
	dfree(B.moved);
	dfree(B.keysA);
	dfree(B.keysB);
	dfree(B.valsA);
	dfree(B.valsB);
	dfree(B.sortHist);
	dfree(B.sceneBounds);
	dfree(B.nodeLo);
	dfree(B.nodeHi);
	dfree(B.nodeLeft);
	dfree(B.nodeRight);
	dfree(B.nodeRope);
	dfree(B.nodeFirst);
	dfree(B.leafData);
	dfree(B.leafOf);
	dfree(B.nodeParent);
	dfree(B.nodeEnd);
	dfree(B.splitRight);
	dfree(B.refitFlag);
	dfree(B.worldEnd);
	dfree(B.proxyInfo);
	dfree(B.leafCount);
	dfree(B.pairScratch);
	dfree(B.scanAux);
	for (int k = 0; k < 2; ++k)
	{
		dfree(B.pairA[k]);
		dfree(B.pairB[k]);
		dfree(B.cstate[k]);
		dfree(B.cache[k]);
		dfree(B.man[k]);
		dfree(B.hashKeys[k]);
		if (k == 0)
			dfree(B.hashMask);
		dfree(B.hashVals[k]);
	}
	dfree(B.prevIndex);
	dfree(B.prevFound);
	dfree(B.rawA);
	dfree(B.rawB);
	dfree(B.travOverflow);
	dfree(B.newList);
	dfree(B.newOff);
	dfree(B.newFill);
	dfree(B.newTmp);
	dfree(B.newTmpMax);
	dfree(B.keptScan);
	dfree(B.posKey);
	dfree(B.wakeList);
	dfree(B.inactiveSave);
	dfree(B.activated);
	dfree(B.lateDestroyed);
	dfree(B.tWake);
	dfree(B.bucketList);
	dfree(B.missList);
	dfree(B.hcPost);
	dfree(B.hsPost);
	dfree(B.counters);
	dfree(B.totals);
	if (c->profEvents)
	{
		for (int i = 0; i < PROF_RING * PROF_MARKS; ++i)
			cudaEventDestroy(c->profEvents[i]);
		delete[] c->profEvents;
	}
	dfree(B.endedList);
	dfree(B.touchIndex);
	dfree(B.touchMan);
	dfree(B.contactOut);
	dfree(B.impulseNormal);
	dfree(B.impulseTangent);
	dfree(B.impulseMotor);
	dfree(c->dHulls);
	dfree(c->dHverts);
	dfree(c->dHedges);
	dfree(c->dHfaces);
	dfree(c->dHplanes);
	dfree(c->dBodyWorld);
	dfree(c->dBodyType);
	dfree(c->dBodyAwake);
	dfree(c->dBodyState);
	dfree(c->scene.bodyXf);
	dfree(c->scene.bodyXf0);
	dfree(c->dFixBody);
	dfree(c->dFixType);
	dfree(c->dFixHull);
	dfree(c->dFixFlags);
	dfree(c->dFixKey);
	dfree(c->dFixRank);
	dfree(c->dFixLife);
	dfree(c->dFixTri);
	dfree(c->dFixWing);
	dfree(c->dFixParams);
	dfree(c->dFixBound);
	dfree(c->dMeshFix);
	free_mesh(c);
	free_queries(c);
	for (int i = 0; i < B3G_STAGE_RING; ++i)
	{
		if (c->stage[i].done)
			cudaEventDestroy(c->stage[i].done);
		if (c->stage[i].host)
			cudaFreeHost(c->stage[i].host);
		if (c->stage[i].dev)
			cudaFree(c->stage[i].dev);
	}
	dfree(c->dWorldCounts);
	dfree(c->dUpdateBad);
	dfree(c->dJointKeys);
	dfree(c->dBodyJoint);
	dfree(c->dVetoPrev);
	dfree(c->dRawDrop);
	dfree(c->dCand);
	dfree(c->dCandPairs);
	if (c->hCounters)
		cudaFreeHost(c->hCounters);
	if (c->copyStream)
	{
		cudaStreamSynchronize(c->copyStream);
		cudaStreamDestroy(c->copyStream);
	}
	if (c->copyReady)
		cudaEventDestroy(c->copyReady);
	if (c->touchBytes)
		cudaFree(c->touchBytes);
	if (c->edgeBuf)
		cudaFree(c->edgeBuf);
	dfree(c->dFixMaterial);
	dfree(c->ciTiles);
	if (c->ciHost)
		cudaFree(c->ciHost);
	if (c->toiScratch)
		cudaFree(c->toiScratch);
	if (c->sideStream)
	{
		cudaStreamSynchronize(c->sideStream);
		cudaStreamDestroy(c->sideStream);
	}
	if (c->meshStream)
	{
		cudaStreamSynchronize(c->meshStream);
		cudaStreamDestroy(c->meshStream);
	}
	if (c->meshFork)
		cudaEventDestroy(c->meshFork);
	if (c->meshJoin)
		cudaEventDestroy(c->meshJoin);
	if (c->forkEvent)
		cudaEventDestroy(c->forkEvent);
	if (c->joinEvent)
		cudaEventDestroy(c->joinEvent);
	if (c->copyDone)
		cudaEventDestroy(c->copyDone);
	if (c->stream)
		cudaStreamDestroy(c->stream);
	delete c;
}

extern "C" const char* b3g_last_error(const b3g_ctx* c)
{
	return c ? c->err.c_str() : "null context";
}

extern "C" int b3g_set_hulls(b3g_ctx* c, uint32_t nh, const uint32_t* desc, const float* verts,
	const uint32_t* edges, const uint32_t* faces, const float* planes, const float* centroids)
{
	if (!c || (nh && (!desc || !verts || !edges || !faces || !planes || !centroids)))
		return fail(c, B3G_E_INVALID, "b3g_set_hulls: null argument");
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	destroy_graphs(c);
	uint32_t nv = 0, ne = 0, nf = 0, maxUE = 0, maxV = 0, maxE = 0, maxF = 0;
	std::vector<HullDesc> hd(nh);
	for (uint32_t h = 0; h < nh; ++h)
	{
		const uint32_t* d = desc + 6 * h;
		if (d[1] < 1 || d[3] < 2 || (d[3] & 1u) || d[5] < 1)
			return fail(c, B3G_E_INVALID, "hull %u: bad counts", h);
		for (uint32_t e = 0; e < d[3]; ++e)
		{
			const uint32_t* E = edges + 5 * (size_t)(d[2] + e);
			if (E[1] != (e ^ 1u))
				return fail(c, B3G_E_INVALID, "hull %u: twin of half-edge %u is not %u", h, e, e ^ 1u);
			if (E[0] >= d[1] || E[2] >= d[5] || E[3] >= d[3] || E[4] >= d[3])
				return fail(c, B3G_E_INVALID, "hull %u: half-edge %u out of range", h, e);
		}
		for (uint32_t f = 0; f < d[5]; ++f)
		{
			uint32_t begin = faces[d[4] + f];
			if (begin >= d[3])
				return fail(c, B3G_E_INVALID, "hull %u: face %u edge out of range", h, f);
			// Every face loop must close within the hull's half-edge count and
			// stay on its face (b3Hull::Validate, hull.cpp:21-78).
			uint32_t e = begin, steps = 0;
			do
			{
				const uint32_t* E = edges + 5 * (size_t)(d[2] + e);
				if (E[2] != f || ++steps > d[3])
					return fail(c, B3G_E_INVALID, "hull %u: face %u loop is broken", h, f);
				e = E[4];
			} while (e != begin);
		}
		hd[h] = HullDesc{d[0], d[1], d[2], d[3], d[4], d[5], centroids[3 * h], centroids[3 * h + 1],
			centroids[3 * h + 2], {0, 0, 0}};
		nv = std::max(nv, d[0] + d[1]);
		ne = std::max(ne, d[2] + d[3]);
		nf = std::max(nf, d[4] + d[5]);
		maxUE = std::max(maxUE, d[3] / 2);
		maxV = std::max(maxV, d[1]);
		maxE = std::max(maxE, d[3]);
		maxF = std::max(maxF, d[5]);
	}
	if (c->cfg.max_hull_data && (size_t)nv + ne + nf > c->cfg.max_hull_data)
		return fail(c, B3G_E_CAPACITY, "hull data %zu exceeds max_hull_data %u", (size_t)nv + ne + nf,
			c->cfg.max_hull_data);
	std::vector<float4> v4(nv), p4(nf);
	std::vector<uint4> e4(ne);
	for (uint32_t i = 0; i < nv; ++i)
		v4[i] = make_float4(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2], 0.0f);
	for (uint32_t i = 0; i < nf; ++i)
		p4[i] = make_float4(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2], planes[4 * i + 3]);
	for (uint32_t i = 0; i < ne; ++i)
		e4[i] = make_uint4(edges[5 * i + 0], edges[5 * i + 2], edges[5 * i + 3], edges[5 * i + 4]);
	dfree(c->dHulls);
	dfree(c->dHverts);
	dfree(c->dHedges);
	dfree(c->dHfaces);
	dfree(c->dHplanes);
	CK(dalloc(&c->dHulls, nh));
	CK(dalloc(&c->dHverts, nv));
	CK(dalloc(&c->dHedges, ne));
	CK(dalloc(&c->dHfaces, nf));
	CK(dalloc(&c->dHplanes, nf));
	if (nh)
	{
		CK(cudaMemcpy(c->dHulls, hd.data(), sizeof(HullDesc) * nh, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dHverts, v4.data(), sizeof(float4) * nv, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dHedges, e4.data(), sizeof(uint4) * ne, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dHfaces, faces, sizeof(uint32_t) * nf, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dHplanes, p4.data(), sizeof(float4) * nf, cudaMemcpyHostToDevice));
	}
	c->hHullDesc.assign(desc, desc + 6 * (size_t)nh);
	c->hHullVerts.assign(verts, verts + 3 * (size_t)nv);
	c->nHulls = nh;
	c->hullVerts = nv;
	c->hullEdges = ne;
	c->hullFaces = nf;
	c->maxUniqueEdges = maxUE;
	c->scene.hullMaxV = maxV;
	c->scene.hullMaxE = maxE;
	c->scene.hullMaxF = maxF;
	c->scene.hulls = c->dHulls;
	c->scene.hverts = c->dHverts;
	c->scene.hedges = c->dHedges;
	c->scene.hfaces = c->dHfaces;
	c->scene.hplanes = c->dHplanes;
	return B3G_OK;
}

extern "C" int b3g_set_bodies(b3g_ctx* c, uint32_t nb, const uint32_t* world, const uint32_t* type,
	const uint8_t* awake)
{
	if (!c || (nb && (!world || !type || !awake)))
		return fail(c, B3G_E_INVALID, "b3g_set_bodies: null argument");
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	destroy_graphs(c);
	uint32_t nw = 1;
	for (uint32_t i = 0; i < nb; ++i)
	{
		if (type[i] > B3G_BODY_DYNAMIC)
			return fail(c, B3G_E_INVALID, "body %u: bad type %u", i, type[i]);
		nw = std::max(nw, world[i] + 1);
	}
	if (nw > c->cfg.max_proxies)
		return fail(c, B3G_E_CAPACITY, "too many worlds");
	dfree(c->dBodyWorld);
	dfree(c->dBodyType);
	dfree(c->dBodyAwake);
	dfree(c->dBodyState);
	dfree(c->scene.bodyXf);
	dfree(c->scene.bodyXf0);
	dfree(c->buf.tWake);
	CK(dalloc(&c->dBodyWorld, nb));
	CK(dalloc(&c->dBodyType, nb));
	CK(dalloc(&c->dBodyAwake, nb));
	CK(dalloc(&c->dBodyState, 17 * (size_t)nb));
	CK(dalloc(&c->scene.bodyXf, 2 * (size_t)nb));
	CK(dalloc(&c->scene.bodyXf0, 2 * (size_t)nb));
	CK(dalloc(&c->buf.tWake, nb));
	if (nb)
	{
		CK(cudaMemcpy(c->dBodyWorld, world, sizeof(uint32_t) * nb, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dBodyType, type, sizeof(uint32_t) * nb, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dBodyAwake, awake, nb, cudaMemcpyHostToDevice));
	}
	c->nBodies = nb;
	c->capBodies = nb;
	c->nWorlds = nw;
	c->hBodyType.assign(type, type + nb);
	c->hAwake.assign(awake, awake + nb);
	c->asleep = count_asleep(c, awake);
	c->scene.bodyWorld = c->dBodyWorld;
	c->scene.bodyType = c->dBodyType;
	c->scene.bodyAwake = c->dBodyAwake;
	c->scene.bodyState = c->dBodyState;
	c->creationPass = true;
	c->havePass = false;
	// Joints and a contact veto name bodies and contacts of the old scene.
	c->nJoints = 0;
	c->nVeto = 0;
	return B3G_OK;
}

extern "C" int b3g_set_fixtures(b3g_ctx* c, uint32_t nf, const uint32_t* body, const uint32_t* shapeType,
	const uint32_t* hull, const float* params, const uint32_t* flags, const uint32_t* proxyKey)
{
	if (!c || (nf && (!body || !shapeType || !hull || !params || !flags)))
		return fail(c, B3G_E_INVALID, "b3g_set_fixtures: null argument");
	if (nf > c->cfg.max_proxies)
		return fail(c, B3G_E_CAPACITY, "%u fixtures exceed max_proxies %u", nf, c->cfg.max_proxies);
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	destroy_graphs(c);
	std::vector<uint32_t> key(nf);
	std::vector<uint32_t> meshFix;
	bool hasTriangles = false;
	for (uint32_t i = 0; i < nf; ++i)
	{
		if (body[i] >= c->nBodies)
			return fail(c, B3G_E_INVALID, "fixture %u: body %u out of range", i, body[i]);
		if (shapeType[i] > B3G_SHAPE_MESH)
			return fail(c, B3G_E_INVALID, "fixture %u: shape type %u not supported", i, shapeType[i]);
		if (shapeType[i] == B3G_SHAPE_TRIANGLE)
			hasTriangles = true;
		if (shapeType[i] == B3G_SHAPE_MESH)
		{
			if (hull[i] >= c->nMeshes)
				return fail(c, B3G_E_INVALID, "fixture %u: mesh %u out of range", i, hull[i]);
			if (c->hBodyType[body[i]] != B3G_BODY_STATIC)
				return fail(c, B3G_E_INVALID, "fixture %u: a mesh needs a static body", i);
			const float* p = params + 12 * (size_t)i;
			if (p[0] == 0.0f || p[1] == 0.0f || p[2] == 0.0f)
				return fail(c, B3G_E_INVALID, "fixture %u: zero mesh scale", i);
			meshFix.push_back(i);
		}
		if (shapeType[i] == B3G_SHAPE_HULL && hull[i] >= c->nHulls)
			return fail(c, B3G_E_INVALID, "fixture %u: hull %u out of range", i, hull[i]);
		key[i] = proxyKey ? proxyKey[i] : i;
	}
	// Rank of each proxy key: pairs are ordered by (smaller key, larger key).
	std::vector<uint32_t> rank(nf);
	{
		std::vector<uint32_t> order(nf);
		for (uint32_t i = 0; i < nf; ++i)
			order[i] = i;
		std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
		for (uint32_t r = 0; r < nf; ++r)
		{
			if (r > 0 && key[order[r]] == key[order[r - 1]])
				return fail(c, B3G_E_INVALID, "fixtures %u and %u share proxy key %u", order[r - 1], order[r],
					key[order[r]]);
			rank[order[r]] = r;
		}
	}
	std::vector<float4> p4(3 * (size_t)nf);
	for (size_t i = 0; i < 3 * (size_t)nf; ++i)
		p4[i] = make_float4(params[4 * i], params[4 * i + 1], params[4 * i + 2], params[4 * i + 3]);
	// Bounding spheres in the body frame: a float centre and a radius computed
	// in double from that centre and rounded up, so the sphere contains the
	// shape (with its skin radius) exactly.
	std::vector<float4> bound(nf);
	for (uint32_t i = 0; i < nf; ++i)
	{
		const float* p = params + 12 * (size_t)i;
		if (shapeType[i] == B3G_SHAPE_MESH)
		{
			bound[i] = make_float4(0.0f, 0.0f, 0.0f, INFINITY);
			continue;
		}
		std::vector<double> pts;
		double skin = 0.0;
		switch (shapeType[i])
		{
		case B3G_SHAPE_SPHERE:
			pts = {p[0], p[1], p[2]};
			skin = p[3];
			break;
		case B3G_SHAPE_CAPSULE:
			pts = {p[0], p[1], p[2], p[3], p[4], p[5]};
			skin = p[6];
			break;
		case B3G_SHAPE_TRIANGLE:
			pts = {p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8]};
			skin = p[9];
			break;
		default:
		{
			const uint32_t* d = c->hHullDesc.data() + 6 * (size_t)hull[i];
			for (uint32_t v = 0; v < d[1]; ++v)
				for (int k = 0; k < 3; ++k)
					pts.push_back(c->hHullVerts[3 * (size_t)(d[0] + v) + k]);
			skin = p[0];
			break;
		}
		}
		size_t np = pts.size() / 3;
		double cx = 0, cy = 0, cz = 0;
		for (size_t v = 0; v < np; ++v)
		{
			cx += pts[3 * v];
			cy += pts[3 * v + 1];
			cz += pts[3 * v + 2];
		}
		float fx = (float)(cx / np), fy = (float)(cy / np), fz = (float)(cz / np);
		double r = 0;
		for (size_t v = 0; v < np; ++v)
		{
			double dx = pts[3 * v] - fx, dy = pts[3 * v + 1] - fy, dz = pts[3 * v + 2] - fz;
			r = std::max(r, std::sqrt(dx * dx + dy * dy + dz * dz));
		}
		r += std::fabs(skin);
		float fr = (float)r;
		fr = std::nextafter(std::nextafter(fr, INFINITY), INFINITY);
		bound[i] = make_float4(fx, fy, fz, fr);
	}
	dfree(c->dFixBound);
	CK(dalloc(&c->dFixBound, nf));
	if (nf)
		CK(cudaMemcpy(c->dFixBound, bound.data(), sizeof(float4) * nf, cudaMemcpyHostToDevice));
	c->scene.fixBound = c->dFixBound;
	dfree(c->dFixBody);
	dfree(c->dFixType);
	dfree(c->dFixHull);
	dfree(c->dFixFlags);
	dfree(c->dFixKey);
	dfree(c->dFixRank);
	dfree(c->dFixLife);
	dfree(c->dFixParams);
	CK(dalloc(&c->dFixBody, nf));
	CK(dalloc(&c->dFixType, nf));
	CK(dalloc(&c->dFixHull, nf));
	CK(dalloc(&c->dFixFlags, nf));
	CK(dalloc(&c->dFixKey, nf));
	CK(dalloc(&c->dFixRank, nf));
	CK(dalloc(&c->dFixLife, nf));
	CK(cudaMemset(c->dFixLife, FIX_LIVE, nf ? nf : 1));
	CK(dalloc(&c->dFixParams, 3 * (size_t)nf));
	{
		// b3FixtureDef's friction and restitution (fixture.h:46-47) until b3g_set_materials.
		dfree(c->dFixMaterial);
		CK(dalloc(&c->dFixMaterial, nf));
		std::vector<float2> mat(std::max(nf, 1u), make_float2(0.3f, 0.0f));
		CK(cudaMemcpy(c->dFixMaterial, mat.data(), sizeof(float2) * mat.size(), cudaMemcpyHostToDevice));
	}
	if (nf)
	{
		CK(cudaMemcpy(c->dFixBody, body, sizeof(uint32_t) * nf, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dFixType, shapeType, sizeof(uint32_t) * nf, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dFixHull, hull, sizeof(uint32_t) * nf, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dFixFlags, flags, sizeof(uint32_t) * nf, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dFixKey, key.data(), sizeof(uint32_t) * nf, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dFixRank, rank.data(), sizeof(uint32_t) * nf, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->dFixParams, p4.data(), sizeof(float4) * 3 * nf, cudaMemcpyHostToDevice));
	}
	c->hFixType.assign(shapeType, shapeType + nf);
	c->anyTriangle = c->anySensor = false;
	for (uint32_t i = 0; i < nf; ++i)
	{
		c->anyTriangle |= shapeType[i] == B3G_SHAPE_TRIANGLE;
		c->anySensor |= (flags[i] & B3G_FIXTURE_SENSOR) != 0;
	}
	c->nFixtures = nf;
	c->capFixtures = nf;
	c->keysAreIndex = true;
	if (proxyKey)
		for (uint32_t i = 0; i < nf && c->keysAreIndex; ++i)
			c->keysAreIndex = proxyKey[i] == i;
	c->scene.fixBody = c->dFixBody;
	c->scene.fixType = c->dFixType;
	c->scene.fixHull = c->dFixHull;
	c->scene.fixFlags = c->dFixFlags;
	c->scene.fixKey = c->dFixKey;
	c->scene.fixRank = c->dFixRank;
	c->scene.fixLife = c->dFixLife;
	c->scene.fixParams = c->dFixParams;
	// Triangle fixtures (after every scene pointer above is current): their b3TriangleHull, built on the device with the
	// pass's arithmetic, and wings (none until b3g_set_triangle_wings).
	dfree(c->dFixTri);
	dfree(c->dFixWing);
	const size_t triSlots = hasTriangles ? nf : 1;
	CK(dalloc(&c->dFixTri, 6 * triSlots));
	CK(dalloc(&c->dFixWing, 3 * triSlots));
	CK(cudaMemset(c->dFixTri, 0, sizeof(float4) * 6 * triSlots));
	CK(cudaMemset(c->dFixWing, 0, sizeof(float4) * 3 * triSlots));
	c->scene.fixTri = c->dFixTri;
	c->scene.fixWing = c->dFixWing;
	c->triSlots = (uint32_t)triSlots;
	if (hasTriangles)
	{
		k_triangle_hulls<<<(nf + 255) / 256, 256>>>(c->scene, nf, c->dFixTri);
		CK(cudaGetLastError());
		CK(cudaDeviceSynchronize());
	}
	// Mesh fixtures (their proxies are built by k_mesh_fat).
	dfree(c->dMeshFix);
	c->nMeshFix = (uint32_t)meshFix.size();
	CK(dalloc(&c->dMeshFix, meshFix.size()));
	if (!meshFix.empty())
		CK(cudaMemcpy(c->dMeshFix, meshFix.data(), sizeof(uint32_t) * meshFix.size(), cudaMemcpyHostToDevice));
	c->creationPass = true;
	c->havePass = false;
	return B3G_OK;
}

// ---------------------------------------------------------------------------
// Scene updates between passes (serving).

namespace {

// The bounding sphere b3g_set_fixtures computes on the host, computed the
// same way on the device (double sums in the same order, the radius rounded
// up twice).
__device__ float4 fixture_bound(const DevScene& S, uint32_t type, uint32_t hull, const float* p)
{
	double pts[9];
	uint32_t np = 0;
	double skin = 0.0;
	const float4* hv = nullptr;
	if (type == B3G_SHAPE_SPHERE)
	{
		pts[0] = p[0], pts[1] = p[1], pts[2] = p[2];
		np = 1;
		skin = p[3];
	}
	else if (type == B3G_SHAPE_CAPSULE)
	{
		for (int k = 0; k < 6; ++k)
			pts[k] = p[k];
		np = 2;
		skin = p[6];
	}
	else if (type == B3G_SHAPE_TRIANGLE)
	{
		for (int k = 0; k < 9; ++k)
			pts[k] = p[k];
		np = 3;
		skin = p[9];
	}
	else
	{
		HullDesc d = S.hulls[hull];
		hv = S.hverts + d.vOff;
		np = d.vCnt;
		skin = p[0];
	}
	auto at = [&](uint32_t v, int k) -> double {
		if (hv)
		{
			float4 w = hv[v];
			return k == 0 ? w.x : (k == 1 ? w.y : w.z);
		}
		return pts[3 * v + k];
	};
	double cx = 0, cy = 0, cz = 0;
	for (uint32_t v = 0; v < np; ++v)
	{
		cx += at(v, 0);
		cy += at(v, 1);
		cz += at(v, 2);
	}
	float fx = (float)(cx / np), fy = (float)(cy / np), fz = (float)(cz / np);
	double r = 0;
	for (uint32_t v = 0; v < np; ++v)
	{
		double dx = at(v, 0) - fx, dy = at(v, 1) - fy, dz = at(v, 2) - fz;
		r = fmax(r, sqrt(dx * dx + dy * dy + dz * dz));
	}
	r += fabs(skin);
	float fr = (float)r;
	fr = nextafterf(nextafterf(fr, INFINITY), INFINITY);
	return make_float4(fx, fy, fz, fr);
}

struct UpdateArgs
{
	uint32_t nb, nf, nr;
	const uint32_t* bIdx;
	const uint32_t* bWorld;
	const uint32_t* bType;
	const uint8_t* bAwake;
	const uint32_t* fIdx;
	const uint32_t* fBody;
	const uint32_t* fType;
	const uint32_t* fHull;
	const uint32_t* fFlags;
	const float* fParams;
	const uint32_t* rIdx;
};

// Limits the records are checked against on the device (records from device
// memory are not seen by the host): an invalid record is skipped and flagged.
struct UpdateLimits
{
	uint32_t bodies, fixtures, worlds, hulls;
	uint32_t* bad;
};

__global__ void k_retire(DevScene S, UpdateArgs u, UpdateLimits lim)
{
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < u.nr; t += gridDim.x * blockDim.x)
	{
		uint32_t f = u.rIdx[t];
		if (f >= lim.fixtures)
		{
			atomicOr(lim.bad, 1u);
			continue;
		}
		S.fixLife[f] = FIX_DEAD;
	}
}

__global__ void k_scatter(DevScene S, UpdateArgs u, UpdateLimits lim, uint32_t* world, uint32_t* btype,
	uint8_t* awake, uint32_t* fbody, uint32_t* ftype, uint32_t* fhull, uint32_t* fflags, float4* fparams,
	float4* fbound)
{
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < u.nb + u.nf; t += gridDim.x * blockDim.x)
	{
		if (t < u.nb)
		{
			uint32_t b = u.bIdx[t];
			if (b >= lim.bodies || u.bWorld[t] >= lim.worlds || u.bType[t] > B3G_BODY_DYNAMIC)
			{
				atomicOr(lim.bad, 1u);
				continue;
			}
			world[b] = u.bWorld[t];
			btype[b] = u.bType[t];
			awake[b] = u.bAwake ? u.bAwake[t] : 1;
			continue;
		}
		uint32_t j = t - u.nb;
		uint32_t f = u.fIdx[j];
		uint32_t ty = u.fType[j];
		if (f >= lim.fixtures || u.fBody[j] >= lim.bodies ||
			!(ty == B3G_SHAPE_SPHERE || ty == B3G_SHAPE_CAPSULE || ty == B3G_SHAPE_HULL) ||
			(ty == B3G_SHAPE_HULL && u.fHull[j] >= lim.hulls))
		{
			atomicOr(lim.bad, 1u);
			continue;
		}
		const float* p = u.fParams + 12 * (size_t)j;
		fbody[f] = u.fBody[j];
		ftype[f] = u.fType[j];
		fhull[f] = u.fHull[j];
		fflags[f] = u.fFlags[j];
		for (int k = 0; k < 3; ++k)
			fparams[3 * (size_t)f + k] = make_float4(p[4 * k], p[4 * k + 1], p[4 * k + 2], p[4 * k + 3]);
		fbound[f] = fixture_bound(S, u.fType[j], u.fHull[j], p);
		S.fixLife[f] = FIX_FRESH;
	}
}

__global__ void k_world_counts(DevScene S, Buffers B, uint32_t cur, uint32_t cap, uint32_t worlds, uint32_t* out)
{
	uint32_t n = min(B.counters[CTR_PAIRS], cap);
	for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
	{
		uint32_t w = S.bodyWorld[S.fixBody[B.pairA[cur][c]]];
		if (w >= worlds)
			continue;
		uint32_t st = B.cstate[cur][c];
		uint32_t pc = ((st >> 8) & 0xFFu) ? B.man[cur][c].pointCount : 0u;
		if (st & 1u)
			atomicAdd(&out[3 * w + 0], 1u);
		if (pc)
		{
			atomicAdd(&out[3 * w + 1], 1u);
			atomicAdd(&out[3 * w + 2], pc);
		}
	}
}

} // namespace

static void launch_update(b3g_ctx* c, const UpdateArgs& u, cudaStream_t s)
{
	UpdateLimits lim{c->capBodies, c->capFixtures, c->nWorlds, c->nHulls, c->dUpdateBad};
	const int blocks = persistent_blocks(2);
	if (u.nr)
		k_retire<<<blocks, 256, 0, s>>>(c->scene, u, lim);
	if (u.nb + u.nf)
		k_scatter<<<blocks, 256, 0, s>>>(c->scene, u, lim, c->dBodyWorld, c->dBodyType, c->dBodyAwake,
			c->dFixBody, c->dFixType, c->dFixHull, c->dFixFlags, c->dFixParams, c->dFixBound);
}

extern "C" int b3g_update_scene_device(b3g_ctx* c, uint32_t nb, const uint32_t* bodyIndex, const uint32_t* world,
	const uint32_t* type, uint32_t nf, const uint32_t* fixIndex, const uint32_t* body, const uint32_t* shapeType,
	const uint32_t* hull, const float* params, const uint32_t* flags, uint32_t nr, const uint32_t* retireIndex,
	void* stream)
{
	if (!c)
		return B3G_E_INVALID;
	if ((nb && (!bodyIndex || !world || !type)) ||
		(nf && (!fixIndex || !body || !shapeType || !hull || !params || !flags)) || (nr && !retireIndex))
		return fail(c, B3G_E_INVALID, "b3g_update_scene_device: null argument");
	if (c->capFixtures == 0 || c->capBodies == 0)
		return fail(c, B3G_E_STATE, "b3g_update_scene_device: no scene");
	if (!c->keysAreIndex)
		return fail(c, B3G_E_STATE, "b3g_update_scene_device: needs proxy keys equal to fixture indices");
	if (nb + nf + nr == 0)
		return B3G_OK;
	CK(cudaSetDevice(c->device));
	cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
	UpdateArgs u;
	u.nb = nb;
	u.nf = nf;
	u.nr = nr;
	u.bIdx = bodyIndex;
	u.bWorld = world;
	u.bType = type;
	u.bAwake = nullptr; // written bodies are awake
	u.fIdx = fixIndex;
	u.fBody = body;
	u.fType = shapeType;
	u.fHull = hull;
	u.fFlags = flags;
	u.fParams = params;
	u.rIdx = retireIndex;
	launch_update(c, u, s);
	CK(cudaGetLastError());
	c->treeForce = true; // fixtures created, replaced or retired: new leaves
	// The written fixtures' types and flags stay on the device.
	c->anyTriangle = c->anySensor = true;
	// The host copy of fixture types is refreshed when the stand-alone
	// narrowphase next needs it; written bodies are awake, so the sleep count
	// can only have dropped (it stays an upper bound until the next wake-up
	// replay recounts it).
	c->fixTypeStale = true;
	return B3G_OK;
}

extern "C" int b3g_update_scene(b3g_ctx* c, uint32_t nb, const uint32_t* bodyIndex, const uint32_t* world,
	const uint32_t* type, const uint8_t* awake, uint32_t nf, const uint32_t* fixIndex, const uint32_t* body,
	const uint32_t* shapeType, const uint32_t* hull, const float* params, const uint32_t* flags, uint32_t nr,
	const uint32_t* retireIndex, void* stream)
{
	if (!c)
		return B3G_E_INVALID;
	if ((nb && (!bodyIndex || !world || !type || !awake)) ||
		(nf && (!fixIndex || !body || !shapeType || !hull || !params || !flags)) || (nr && !retireIndex))
		return fail(c, B3G_E_INVALID, "b3g_update_scene: null argument");
	if (c->capFixtures == 0 || c->capBodies == 0)
		return fail(c, B3G_E_STATE, "b3g_update_scene: no scene");
	if (!c->keysAreIndex)
		return fail(c, B3G_E_STATE, "b3g_update_scene: needs proxy keys equal to fixture indices");
	for (uint32_t i = 0; i < nb; ++i)
		if (bodyIndex[i] >= c->capBodies || world[i] >= c->nWorlds || type[i] > B3G_BODY_DYNAMIC)
			return fail(c, B3G_E_INVALID, "b3g_update_scene: body record %u invalid", i);
	for (uint32_t i = 0; i < nf; ++i)
		if (fixIndex[i] >= c->capFixtures || body[i] >= c->capBodies ||
			!(shapeType[i] == B3G_SHAPE_SPHERE || shapeType[i] == B3G_SHAPE_CAPSULE ||
				shapeType[i] == B3G_SHAPE_HULL) ||
			(shapeType[i] == B3G_SHAPE_HULL && hull[i] >= c->nHulls))
			return fail(c, B3G_E_INVALID, "b3g_update_scene: fixture record %u invalid", i);
	for (uint32_t i = 0; i < nr; ++i)
		if (retireIndex[i] >= c->capFixtures)
			return fail(c, B3G_E_INVALID, "b3g_update_scene: retire index %u out of range", i);
	if (nb + nf + nr == 0)
		return B3G_OK;
	CK(cudaSetDevice(c->device));
	cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
	// One host staging block per call, copied in one transfer. The staging
	// buffers form a ring; a slot is reused once its previous copy finished.
	size_t words = 4 * (size_t)nb + (size_t)(nb + 3) / 4 + 17 * (size_t)nf + nr;
	size_t bytes = words * 4 + 64;
	StageSlot& slot = c->stage[c->stageNext];
	c->stageNext = (c->stageNext + 1) % B3G_STAGE_RING;
	if (slot.done)
		CK(cudaEventSynchronize(slot.done));
	if (slot.bytes < bytes)
	{
		CK(cudaStreamSynchronize(s));
		if (slot.host)
			cudaFreeHost(slot.host);
		if (slot.dev)
			cudaFree(slot.dev);
		slot.host = nullptr;
		slot.dev = nullptr;
		slot.bytes = 0;
		size_t grow = std::max(bytes, (size_t)1 << 20);
		CK(cudaMallocHost(&slot.host, grow));
		CK(cudaMalloc(&slot.dev, grow));
		slot.bytes = grow;
	}
	if (!slot.done)
		CK(cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming));
	uint32_t* h = (uint32_t*)slot.host;
	uint32_t* d = (uint32_t*)slot.dev;
	size_t o = 0;
	UpdateArgs u;
	u.nb = nb;
	u.nf = nf;
	u.nr = nr;
	auto put = [&](const void* src, size_t n32) -> const uint32_t* {
		std::memcpy(h + o, src, n32 * 4);
		const uint32_t* dp = d + o;
		o += n32;
		return dp;
	};
	u.bIdx = put(bodyIndex, nb);
	u.bWorld = put(world, nb);
	u.bType = put(type, nb);
	std::memcpy(h + o, awake, nb);
	u.bAwake = (const uint8_t*)(d + o);
	o += (nb + 3) / 4;
	u.fIdx = put(fixIndex, nf);
	u.fBody = put(body, nf);
	u.fType = put(shapeType, nf);
	u.fHull = put(hull, nf);
	u.fFlags = put(flags, nf);
	u.fParams = (const float*)put(params, 12 * (size_t)nf);
	u.rIdx = put(retireIndex, nr);
	CK(cudaMemcpyAsync(slot.dev, slot.host, o * 4, cudaMemcpyHostToDevice, s));
	CK(cudaEventRecord(slot.done, s));
	launch_update(c, u, s);
	CK(cudaGetLastError());
	c->treeForce = true; // fixtures created, replaced or retired: new leaves
	// Host shadows: fixture types (stand-alone narrowphase) and sleep count.
	for (uint32_t i = 0; i < nf; ++i)
	{
		c->hFixType[fixIndex[i]] = shapeType[i];
		c->anyTriangle |= shapeType[i] == B3G_SHAPE_TRIANGLE;
		c->anySensor |= (flags[i] & B3G_FIXTURE_SENSOR) != 0;
	}
	for (uint32_t i = 0; i < nb; ++i)
	{
		uint32_t b = bodyIndex[i];
		bool was = c->hAwake[b] == 0 && c->hBodyType[b] != B3G_BODY_STATIC;
		bool now = awake[i] == 0 && type[i] != B3G_BODY_STATIC;
		c->hBodyType[b] = type[i];
		c->hAwake[b] = awake[i];
		c->asleep = c->asleep - (was ? 1u : 0u) + (now ? 1u : 0u);
	}
	return B3G_OK;
}

extern "C" int b3g_set_active(b3g_ctx* c, uint32_t bodies, uint32_t fixtures)
{
	if (!c)
		return B3G_E_INVALID;
	if (bodies > c->capBodies || fixtures > c->capFixtures || fixtures == 0 || bodies == 0)
		return fail(c, B3G_E_INVALID, "b3g_set_active: %u bodies / %u fixtures outside 1..(%u, %u)", bodies,
			fixtures, c->capBodies, c->capFixtures);
	if (bodies == c->nBodies && fixtures == c->nFixtures)
		return B3G_OK;
	CK(cudaSetDevice(c->device));
	CK(cudaDeviceSynchronize());
	destroy_graphs(c);
	c->nBodies = bodies;
	c->nFixtures = fixtures;
	return B3G_OK;
}

extern "C" int b3g_world_counts(b3g_ctx* c, uint32_t worlds, uint32_t* out, void* stream)
{
	if (!c || (!out && worlds))
		return fail(c, B3G_E_INVALID, "b3g_world_counts: null argument");
	if (!c->havePass)
		return fail(c, B3G_E_STATE, "b3g_world_counts: no pass yet");
	if (worlds == 0)
		return B3G_OK;
	CK(cudaSetDevice(c->device));
	cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
	CK(cudaMemsetAsync(out, 0, sizeof(uint32_t) * 3 * (size_t)worlds, s));
	k_world_counts<<<persistent_blocks(4), 256, 0, s>>>(c->scene, c->buf, c->cur, c->cfg.max_contacts, worlds, out);
	CK(cudaGetLastError());
	return B3G_OK;
}

extern "C" int b3g_set_awake(b3g_ctx* c, const uint8_t* awake)
{
	if (!c || !awake)
		return fail(c, B3G_E_INVALID, "b3g_set_awake: null argument");
	CK(cudaSetDevice(c->device));
	if (c->nBodies)
	{
		CK(cudaMemcpyAsync(c->dBodyAwake, awake, c->nBodies, cudaMemcpyHostToDevice, c->stream));
		CK(cudaStreamSynchronize(c->stream));
	}
	c->asleep = count_asleep(c, awake);
	c->hAwake.assign(awake, awake + c->capBodies);
	return B3G_OK;
}

extern "C" int b3g_set_triangle_wings(b3g_ctx* c, uint32_t n, const uint32_t* fixture, const float* wings)
{
	if (!c || (n && (!fixture || !wings)))
		return fail(c, B3G_E_INVALID, "b3g_set_triangle_wings: null argument");
	if (c->nFixtures == 0)
		return fail(c, B3G_E_STATE, "b3g_set_triangle_wings: no fixtures");
	std::vector<float4> w(3 * (size_t)n);
	for (uint32_t i = 0; i < n; ++i)
	{
		if (fixture[i] >= c->capFixtures || c->hFixType[fixture[i]] != B3G_SHAPE_TRIANGLE ||
			fixture[i] >= c->triSlots)
			return fail(c, B3G_E_INVALID, "b3g_set_triangle_wings: fixture %u is not a triangle", fixture[i]);
		const float* x = wings + 12 * (size_t)i;
		for (int k = 0; k < 3; ++k)
			w[3 * i + k] = make_float4(x[3 * k], x[3 * k + 1], x[3 * k + 2], x[9 + k] != 0.0f ? 1.0f : 0.0f);
	}
	CK(cudaSetDevice(c->device));
	CK(cudaDeviceSynchronize());
	for (uint32_t i = 0; i < n; ++i)
		CK(cudaMemcpy(c->dFixWing + 3 * (size_t)fixture[i], &w[3 * i], sizeof(float4) * 3, cudaMemcpyHostToDevice));
	destroy_graphs(c);
	return B3G_OK;
}

extern "C" int b3g_fetch_awake(b3g_ctx* c, uint8_t* out, uint32_t capacity)
{
	if (!c || (!out && capacity))
		return fail(c, B3G_E_INVALID, "b3g_fetch_awake: null argument");
	CK(cudaSetDevice(c->device));
	CK(cudaDeviceSynchronize());
	uint32_t n = std::min(c->nBodies, capacity);
	if (n)
		CK(cudaMemcpy(out, c->dBodyAwake, n, cudaMemcpyDeviceToHost));
	return (int)c->nBodies;
}

// The contact list and the narrowphase of a pass whose broadphase has run.
static void issue_pass_rest(b3g_ctx* c, cudaStream_t s)
{
	launch_pairs_diff(c, s);
	prof_mark(c, PM_DIFFED, s);
	launch_narrowphase(c, s);
}

// Kernels of one pass up to the narrowphase, on s (profiling marks when on).
// While s is being captured, *copyNode receives the state copy's graph node.
static void issue_pass(b3g_ctx* c, cudaStream_t s, const float* state, size_t bytes, cudaMemcpyKind kind,
	cudaGraphNode_t* copyNode = nullptr)
{
	prof_mark(c, PM_BEGIN, s);
	cudaMemcpyAsync(c->dBodyState, state, bytes, kind, s);
	if (copyNode)
	{
		cudaStreamCaptureStatus st;
		const cudaGraphNode_t* deps = nullptr;
		size_t nd = 0;
		*copyNode = nullptr;
		if (cudaStreamGetCaptureInfo(s, &st, nullptr, nullptr, &deps, &nd) == cudaSuccess && nd == 1)
			*copyNode = deps[0];
	}
	k_pass_begin<<<1, CTR_COUNT, 0, s>>>(c->buf.counters, c->havePass ? 1 : 0, c->cfg.max_contacts);
	prof_mark(c, PM_UPLOADED, s);
	launch_sync(c, s);
	prof_mark(c, PM_SYNCED, s);
	launch_broadphase(c, s);
	if (c->filterMode == 2)
	{
		// The caller's contact filter decides the new pairs before the
		// contact list is built: the pass stops here (b3g_finish_pass).
		launch_candidates(c, s);
		return;
	}
	issue_pass_rest(c, s);
}

// Work that rewrites the contact records or the touching output waits for
// the copies b3g_fetch_results_async started from them.
static void wait_copies(b3g_ctx* c, cudaStream_t s)
{
	if (c->copyPending)
		cudaStreamWaitEvent(s, c->copyDone, 0);
}

// Kernels of a pass's narrowphase: bucketing, the apart pairs, the convex
// buckets (with the hull-sphere and hull-capsule follow-up kernels), the hull
// probe and SAT, hull-triangle, and the mesh work.
static uint32_t narrow_launches(const b3g_ctx* c)
{
	uint32_t k = 0;
	for (int b = 0; b < B3G_CONVEX_KERNELS; ++b)
		k += convex_bucket_possible(c, b) ? 1u : 0u;
	return 1 + 1 + k + 2 + 2 + (c->anyTriangle ? 1u : 0u) + mesh_launches(c);
}

// The LBVH bookkeeping once a pass's broadphase is issued.
static void tree_pass_issued(b3g_ctx* c)
{
	if (c->treeRebuild)
	{
		c->treeSince = 0;
		c->treeForce = false;
		c->treeWorlds = c->nWorlds;
	}
	else
		++c->treeSince;
}

extern "C" int b3g_collide(b3g_ctx* c, const float* state, int onDevice, void* stream)
{
	if (!c || !state)
		return fail(c, B3G_E_INVALID, "b3g_collide: null argument");
	if (c->nBodies == 0 || c->nFixtures == 0)
		return fail(c, B3G_E_STATE, "b3g_collide: no scene");
	CK(cudaSetDevice(c->device));
	cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
	size_t bytes = sizeof(float) * 17 * (size_t)c->nBodies;
	const cudaMemcpyKind kind = onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
	// LBVH plan of this pass (broadphase.cu): rebuild every treeInterval
	// passes and whenever the proxy set may have changed, else refit.
	c->treeRebuild = c->treeForce || c->treeLeaves != c->nFixtures || c->treeWorlds != c->nWorlds ||
		c->treeSince + 1 >= c->treeInterval;
	// pass_begin, sync, broadphase, diff + list order, bucket + apart + convex kernels + 2 hull +
	// hull-triangle, finalize
	const uint32_t passLaunches = 1 + 1 + (c->creationPass && c->nMeshFix ? 1 : 0) + broadphase_launches(c) +
		pairs_diff_launches(c) + narrow_launches(c) + 1;
	// Host state takes the graph path when it is pinned (a graph copies it
	// asynchronously; pageable memory would need the synchronous copy).
	bool pinnedHost = false;
	if (!onDevice)
	{
		cudaPointerAttributes attr;
		if (cudaPointerGetAttributes(&attr, state) == cudaSuccess)
			pinnedHost = attr.type == cudaMemoryTypeHost;
		else
			cudaGetLastError();
	}
	if (c->passOpen)
		return fail(c, B3G_E_INVALID, "b3g_collide: the last pass waits for b3g_finish_pass");
	// Filters of this pass: the caller's contact filter (a host round trip in
	// the middle of the pass), else joints or a contact veto (inside the pass).
	c->filterMode = (c->cfg.flags & B3G_FLAG_CONTACT_FILTER) ? 2 : ((c->nJoints || c->nVeto) ? 1 : 0);
	if (c->filterMode == 2 && (!c->dRawDrop || !c->dCand || !c->dCandPairs))
	{
		CK(dalloc(&c->dRawDrop, c->cfg.max_contacts));
		CK(dalloc(&c->dCand, c->cfg.max_contacts));
		CK(dalloc(&c->dCandPairs, c->cfg.max_contacts));
	}
	const bool graph = (c->cfg.flags & B3G_FLAG_GRAPH) && (onDevice || pinnedHost) && !c->profiling &&
		c->asleep == 0 && c->havePass && !c->creationPass && s != nullptr && c->filterMode == 0;
	c->lastPassImpulses = c->impulsesLoaded;
	if (graph)
	{
		c->cur ^= 1u;
		// A pass of this parity is captured in both forms (tree rebuilt,
		// tree refit) the first time either is needed, so a later pass never
		// pays for a capture.
		const bool rebuild = c->treeRebuild;
		for (int variant = 0; variant < 2; ++variant)
		{
			c->treeRebuild = variant == 0 ? rebuild : !rebuild;
			PassGraph& g = c->graphs[c->cur][c->impulsesLoaded ? 1 : 0][c->treeRebuild ? 1 : 0];
			if (g.exec && g.stream == s && g.kind == kind && g.state != state)
			{
				// Same pass, state at another address: re-point the copy node.
				if (g.copyNode && cudaGraphExecMemcpyNodeSetParams1D(g.exec, g.copyNode, c->dBodyState, state,
									   bytes, kind) == cudaSuccess)
					g.state = state;
				else
					cudaGetLastError();
			}
			if (g.exec && g.state == state && g.stream == s && g.kind == kind)
				continue;
			if (g.exec)
				cudaGraphExecDestroy(g.exec);
			if (g.graph)
				cudaGraphDestroy(g.graph);
			g = PassGraph{nullptr, nullptr, nullptr, nullptr, nullptr, cudaMemcpyDefault};
			// The captured kernels use the contact buffers of this parity and
			// the host-side pass state every later pass of this parity has.
			CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
			issue_pass(c, s, state, bytes, kind, &g.copyNode);
			// Copies of the previous results (b3g_fetch_results_async) finish
			// before finalize rewrites the contact records.
			cudaStreamWaitEvent(s, c->copyDone, cudaEventWaitExternal);
			launch_finalize(c, s);
			cudaError_t e = cudaStreamEndCapture(s, &g.graph);
			if (e != cudaSuccess)
			{
				g.graph = nullptr;
				c->treeRebuild = rebuild;
				return fail(c, B3G_E_CUDA, "b3g_collide: pass capture failed: %s", cudaGetErrorString(e));
			}
			e = cudaGraphInstantiate(&g.exec, g.graph, 0);
			if (e != cudaSuccess)
			{
				cudaGraphDestroy(g.graph);
				g = PassGraph{nullptr, nullptr, nullptr, nullptr, nullptr, cudaMemcpyDefault};
				c->treeRebuild = rebuild;
				return fail(c, B3G_E_CUDA, "b3g_collide: graph instantiation failed: %s", cudaGetErrorString(e));
			}
			g.state = state;
			g.stream = s;
			g.kind = kind;
		}
		c->treeRebuild = rebuild;
		CK(cudaGraphLaunch(c->graphs[c->cur][c->impulsesLoaded ? 1 : 0][rebuild ? 1 : 0].exec, s));
		++c->graphLaunches;
	}
	else
	{
		if (c->profiling)
		{
			int rc = prof_begin_pass(c);
			if (rc)
				return rc;
		}
		if (c->havePass)
			c->cur ^= 1u;
		issue_pass(c, s, state, bytes, kind);
		if (c->filterMode == 2)
		{
			c->passOpen = true;
			c->candFetched = false;
			c->passStream = s;
			// pass begin, sync, broadphase, candidates; the rest in b3g_finish_pass
			c->launches += 1 + 1 + (c->creationPass && c->nMeshFix ? 1 : 0) + broadphase_launches(c) + 2;
			CK(cudaGetLastError());
			tree_pass_issued(c);
			return B3G_OK;
		}
		if (c->asleep > 0)
		{
			int rc = resolve_wakeups(c, s);
			if (rc)
				return fail(c, rc, "b3g_collide: wake-up rounds failed: %s", cudaGetErrorString(cudaGetLastError()));
		}
		wait_copies(c, s);
		launch_finalize(c, s);
		prof_mark(c, PM_FINAL, s);
		if (c->profiling)
			++c->profPass;
	}
	c->launches += passLaunches;
	CK(cudaGetLastError());
	tree_pass_issued(c);
	c->creationPass = false;
	c->havePass = true;
	c->impulsesLoaded = false;
	c->nVeto = 0;
	return B3G_OK;
}

// ---------------------------------------------------------------------------
// Collision filters.

static int sync_counts(b3g_ctx* c);

extern "C" int b3g_set_joint_pairs(b3g_ctx* c, uint32_t count, const uint32_t* bodyPairs)
{
	if (!c || (count && !bodyPairs))
		return fail(c, B3G_E_INVALID, "b3g_set_joint_pairs: null argument");
	if (c->passOpen)
		return fail(c, B3G_E_INVALID, "b3g_set_joint_pairs: the last pass waits for b3g_finish_pass");
	if (c->nBodies == 0)
		return fail(c, B3G_E_STATE, "b3g_set_joint_pairs: no bodies");
	CK(cudaSetDevice(c->device));
	std::vector<unsigned long long> keys;
	keys.reserve(count);
	std::vector<uint8_t> flag(c->nBodies, 0);
	for (uint32_t i = 0; i < count; ++i)
	{
		uint32_t a = bodyPairs[2 * i], b = bodyPairs[2 * i + 1];
		if (a >= c->nBodies || b >= c->nBodies || a == b)
			return fail(c, B3G_E_INVALID, "b3g_set_joint_pairs: pair %u (%u, %u) is not two bodies of the scene", i,
				a, b);
		keys.push_back(a < b ? ((unsigned long long)a << 32) | b : ((unsigned long long)b << 32) | a);
		flag[a] = flag[b] = 1;
	}
	std::sort(keys.begin(), keys.end());
	keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
	CK(cudaStreamSynchronize(c->stream));
	if (keys.size() > c->jointCap)
	{
		dfree(c->dJointKeys);
		CK(dalloc(&c->dJointKeys, keys.size()));
		c->jointCap = (uint32_t)keys.size();
	}
	const uint32_t nb = std::max(c->capBodies, c->nBodies);
	if (c->bodyJointCap < nb)
	{
		dfree(c->dBodyJoint);
		CK(dalloc(&c->dBodyJoint, nb));
		c->bodyJointCap = nb;
	}
	flag.resize(nb, 0);
	if (!keys.empty())
		CK(cudaMemcpy(c->dJointKeys, keys.data(), sizeof(unsigned long long) * keys.size(), cudaMemcpyHostToDevice));
	CK(cudaMemcpy(c->dBodyJoint, flag.data(), flag.size(), cudaMemcpyHostToDevice));
	c->nJoints = (uint32_t)keys.size();
	return B3G_OK;
}

extern "C" int b3g_set_contact_veto(b3g_ctx* c, uint32_t count, const uint8_t* veto)
{
	if (!c || (count && !veto))
		return fail(c, B3G_E_INVALID, "b3g_set_contact_veto: null argument");
	if (c->passOpen)
		return fail(c, B3G_E_INVALID, "b3g_set_contact_veto: the last pass waits for b3g_finish_pass");
	int rc = sync_counts(c);
	if (rc)
		return rc;
	uint32_t n = std::min(c->hCounters[CTR_PAIRS], c->cfg.max_contacts);
	if (!c->havePass || count != n)
		return fail(c, B3G_E_INVALID, "b3g_set_contact_veto: %u flags for %u contacts of the last pass", count, n);
	if (!c->dVetoPrev)
		CK(dalloc(&c->dVetoPrev, c->cfg.max_contacts));
	if (count)
		CK(cudaMemcpy(c->dVetoPrev, veto, count, cudaMemcpyHostToDevice));
	c->nVeto = count;
	return B3G_OK;
}

extern "C" int b3g_fetch_new_pairs(b3g_ctx* c, uint32_t* out, uint32_t capacity)
{
	if (!c || (capacity && !out))
		return fail(c, B3G_E_INVALID, "b3g_fetch_new_pairs: null argument");
	if (!c->passOpen)
		return fail(c, B3G_E_INVALID, "b3g_fetch_new_pairs: no pass waits for the contact filter");
	CK(cudaSetDevice(c->device));
	cudaStream_t s = c->passStream;
	uint32_t n = 0;
	CK(cudaMemcpyAsync(&n, c->buf.counters + CTR_CANDIDATES, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
	CK(cudaStreamSynchronize(s));
	n = std::min(n, c->cfg.max_contacts);
	std::vector<uint4> rec(n);
	std::vector<uint32_t> raw(n);
	if (n)
	{
		launch_candidate_pairs(c, n, s);
		++c->launches;
		CK(cudaMemcpyAsync(rec.data(), c->dCandPairs, sizeof(uint4) * n, cudaMemcpyDeviceToHost, s));
		CK(cudaMemcpyAsync(raw.data(), c->dCand, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
		CK(cudaStreamSynchronize(s));
	}
	// AddPair order: the pairs FindPairs reports, ascending by (smaller proxy
	// key, larger proxy key) (broad_phase.h:181-206).
	std::vector<uint32_t> order(n);
	for (uint32_t i = 0; i < n; ++i)
		order[i] = i;
	std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
		return rec[x].z != rec[y].z ? rec[x].z < rec[y].z : rec[x].w < rec[y].w;
	});
	c->hCandOrder.resize(n);
	for (uint32_t i = 0; i < n; ++i)
	{
		c->hCandOrder[i] = raw[order[i]];
		if (i < capacity)
		{
			out[2 * i + 0] = rec[order[i]].x;
			out[2 * i + 1] = rec[order[i]].y;
		}
	}
	c->nCand = n;
	c->candFetched = true;
	return (int)n;
}

extern "C" int b3g_finish_pass(b3g_ctx* c, const uint8_t* keep, uint32_t count)
{
	if (!c)
		return B3G_E_INVALID;
	if (!c->passOpen)
		return fail(c, B3G_E_INVALID, "b3g_finish_pass: no pass waits for the contact filter");
	if (keep && (!c->candFetched || count != c->nCand))
		return fail(c, B3G_E_INVALID, "b3g_finish_pass: %u flags for %u new pairs (b3g_fetch_new_pairs first)", count,
			c->candFetched ? c->nCand : 0u);
	CK(cudaSetDevice(c->device));
	cudaStream_t s = c->passStream;
	std::vector<uint32_t> rejected;
	if (keep)
		for (uint32_t i = 0; i < count; ++i)
			if (!keep[i])
				rejected.push_back(c->hCandOrder[i]);
	uint32_t* dRejected = reinterpret_cast<uint32_t*>(c->dCandPairs);
	if (!rejected.empty())
	{
		// From pageable memory: the call returns once the host buffer is read.
		CK(cudaMemcpyAsync(dRejected, rejected.data(), sizeof(uint32_t) * rejected.size(), cudaMemcpyHostToDevice, s));
		launch_apply_veto(c, dRejected, (uint32_t)rejected.size(), s);
	}
	c->passOpen = false;
	issue_pass_rest(c, s);
	if (c->asleep > 0)
	{
		int rc = resolve_wakeups(c, s);
		if (rc)
			return fail(c, rc, "b3g_finish_pass: wake-up rounds failed: %s", cudaGetErrorString(cudaGetLastError()));
	}
	wait_copies(c, s);
	launch_finalize(c, s);
	prof_mark(c, PM_FINAL, s);
	if (c->profiling)
		++c->profPass;
	c->launches += pairs_diff_launches(c) + narrow_launches(c) + 1 +
		(rejected.empty() ? 0 : 1);
	CK(cudaGetLastError());
	c->creationPass = false;
	c->havePass = true;
	c->impulsesLoaded = false;
	c->nVeto = 0;
	return B3G_OK;
}

static int sync_counts(b3g_ctx* c)
{
	CK(cudaSetDevice(c->device));
	CK(cudaMemcpyAsync(c->hCounters, c->buf.counters, sizeof(uint32_t) * CTR_COUNT, cudaMemcpyDeviceToHost,
		c->stream));
	CK(cudaStreamSynchronize(c->stream));
	CK(cudaDeviceSynchronize());
	return B3G_OK;
}

static uint32_t status_code(uint32_t st)
{
	if (st & (B3G_ST_PAIR_OVERFLOW | B3G_ST_HASH_OVERFLOW | B3G_ST_POLY_OVERFLOW))
		return (uint32_t)(-B3G_E_CAPACITY);
	if (st & B3G_ST_WAIT_TIMEOUT)
		return (uint32_t)(-B3G_E_TIMEOUT);
	return 0;
}

extern "C" int b3g_get_counts(b3g_ctx* c, b3g_counts* out)
{
	if (!c || !out)
		return fail(c, B3G_E_INVALID, "b3g_get_counts: null argument");
	if (c->passOpen)
		return fail(c, B3G_E_INVALID, "b3g_get_counts: the last pass waits for b3g_finish_pass");
	int rc = sync_counts(c);
	if (rc)
		return rc;
	const uint32_t* h = c->hCounters;
	out->contacts = std::min(h[CTR_PAIRS], c->cfg.max_contacts);
	out->begun = h[CTR_BEGUN];
	out->ended = h[CTR_ENDED];
	out->touching = h[CTR_TOUCHING];
	out->manifolds = h[CTR_MANIFOLDS];
	out->points = h[CTR_POINTS];
	out->moved = h[CTR_MOVED];
	uint32_t bad = 0;
	if (c->dUpdateBad)
	{
		CK(cudaMemcpy(&bad, c->dUpdateBad, sizeof(uint32_t), cudaMemcpyDeviceToHost));
		if (bad)
		{
			CK(cudaMemset(c->dUpdateBad, 0, sizeof(uint32_t)));
			return fail(c, B3G_E_INVALID, "a device-side scene update held invalid records (skipped)");
		}
	}
	out->status = status_code(h[CTR_STATUS]);
	if (out->status)
		return fail(c, -(int)out->status, "pass status 0x%x (pairs %u, capacity %u)", h[CTR_STATUS],
			h[CTR_PAIRS], c->cfg.max_contacts);
	return B3G_OK;
}

extern "C" int b3g_get_pass_stats(b3g_ctx* c, uint32_t* out, uint32_t capacity)
{
	if (!c || !out)
		return fail(c, B3G_E_INVALID, "b3g_get_pass_stats: null argument");
	int rc = sync_counts(c);
	if (rc)
		return rc;
	const uint32_t* h = c->hCounters;
	uint32_t s[B3G_STAT_COUNT];
	s[B3G_STAT_RAW_PAIRS] = h[CTR_RAW];
	s[B3G_STAT_KEPT] = h[CTR_KEPT];
	s[B3G_STAT_HULL_MISS] = h[CTR_HULL_MISS];
	s[B3G_STAT_TRAV_OVERFLOW] = h[CTR_TRAV_OVERFLOW];
	s[B3G_STAT_MESH_ITEMS] = h[CTR_MESH_PAIRS];
	s[B3G_STAT_WAKE_EVENTS] = h[CTR_WAKE_EVENTS];
	s[B3G_STAT_WAKE_ACTIVATED] = h[CTR_WAKE_ACTIVATED];
	s[B3G_STAT_LATE_DESTROYED] = h[CTR_LATE_DESTROYED];
	s[B3G_STAT_ASLEEP] = h[CTR_ASLEEP];
	static_assert(B3G_STAT_BUCKET0 + BK_COUNT == B3G_STAT_COUNT, "one statistic per bucket");
	for (uint32_t b = 0; b < BK_COUNT; ++b)
		s[B3G_STAT_BUCKET0 + b] = h[CTR_BUCKET0 + b];
	uint32_t n = std::min<uint32_t>(capacity, B3G_STAT_COUNT);
	std::memcpy(out, s, sizeof(uint32_t) * n);
	return (int)n;
}

static int contacts_now(b3g_ctx* c, uint32_t& n)
{
	if (!c->havePass)
		return fail(c, B3G_E_STATE, "no pass yet");
	int rc = sync_counts(c);
	if (rc)
		return rc;
	n = std::min(c->hCounters[CTR_PAIRS], c->cfg.max_contacts);
	return B3G_OK;
}

extern "C" int b3g_fetch_contacts(b3g_ctx* c, uint32_t* out, uint32_t capacity)
{
	if (!c || !out)
		return fail(c, B3G_E_INVALID, "null argument");
	uint32_t n;
	int rc = contacts_now(c, n);
	if (rc)
		return rc;
	n = std::min(n, capacity);
	if (n)
		CK(cudaMemcpy(out, c->buf.contactOut, sizeof(uint32_t) * 3 * n, cudaMemcpyDeviceToHost));
	return (int)n;
}

extern "C" int b3g_fetch_manifolds(b3g_ctx* c, void* out, uint32_t capacity)
{
	if (!c || !out)
		return fail(c, B3G_E_INVALID, "null argument");
	uint32_t n;
	int rc = contacts_now(c, n);
	if (rc)
		return rc;
	n = std::min(n, capacity);
	if (n)
		CK(cudaMemcpy(out, c->buf.man[c->cur], sizeof(DevManifold) * n, cudaMemcpyDeviceToHost));
	return (int)n;
}

extern "C" int b3g_fetch_touching(b3g_ctx* c, uint32_t* index, void* manifolds, uint32_t capacity)
{
	if (!c || !index || !manifolds)
		return fail(c, B3G_E_INVALID, "null argument");
	uint32_t n;
	int rc = contacts_now(c, n);
	if (rc)
		return rc;
	Buffers& B = c->buf;
	if (n == 0)
		return 0;
	uint32_t* offsets = B.leafCount; // sized max(P, C)
	const DevManifold* extra = B.extraMan[c->cur] ? B.extraMan[c->cur] : B.man[c->cur];
	wait_copies(c, c->stream);
	k_touch_flags<<<(n + 255) / 256, 256, 0, c->stream>>>(B.man[c->cur], extra, B.cstate[c->cur], n, offsets);
	scan_exclusive(offsets, n, B.scanAux, B.counters + CTR_TOUCH_OUT, B.counters + CTR_STATUS, c->stream);
	uint32_t total = 0;
	CK(cudaMemcpyAsync(&total, B.counters + CTR_TOUCH_OUT, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	if (total > c->cfg.max_contacts)
		return fail(c, B3G_E_CAPACITY, "b3g_fetch_touching: %u manifolds exceed the output buffer", total);
	k_touch_scatter<<<(n + 255) / 256, 256, 0, c->stream>>>(B.man[c->cur], extra, B.cstate[c->cur], offsets, n,
		B.touchIndex, B.touchMan);
	CK(cudaStreamSynchronize(c->stream));
	uint32_t m = std::min(total, capacity);
	if (m)
	{
		CK(cudaMemcpy(index, B.touchIndex, sizeof(uint32_t) * m, cudaMemcpyDeviceToHost));
		CK(cudaMemcpy(manifolds, B.touchMan, sizeof(DevManifold) * m, cudaMemcpyDeviceToHost));
	}
	return (int)m;
}

extern "C" int b3g_fetch_results_async(b3g_ctx* c, uint32_t* contacts, uint32_t contactCapacity, uint32_t* index,
	void* manifolds, uint32_t touchCapacity, b3g_counts* counts)
{
	if (!c || !counts || (contactCapacity && !contacts) || (touchCapacity && (!index || !manifolds)))
		return fail(c, B3G_E_INVALID, "null argument");
	if (!c->havePass)
		return fail(c, B3G_E_STATE, "no pass yet");
	CK(cudaSetDevice(c->device));
	// The pass's counters (sizes of the outputs); only the pass stream is
	// waited for, so copies of earlier passes keep running.
	CK(cudaMemcpyAsync(c->hCounters, c->buf.counters, sizeof(uint32_t) * CTR_COUNT, cudaMemcpyDeviceToHost,
		c->stream));
	CK(cudaStreamSynchronize(c->stream));
	const uint32_t* h = c->hCounters;
	const uint32_t n = std::min(h[CTR_PAIRS], c->cfg.max_contacts);
	counts->contacts = n;
	counts->begun = h[CTR_BEGUN];
	counts->ended = h[CTR_ENDED];
	counts->touching = h[CTR_TOUCHING];
	counts->manifolds = h[CTR_MANIFOLDS];
	counts->points = h[CTR_POINTS];
	counts->moved = h[CTR_MOVED];
	counts->status = status_code(h[CTR_STATUS]);
	if (counts->status)
		return fail(c, -(int)counts->status, "pass status 0x%x (pairs %u, capacity %u)", h[CTR_STATUS], h[CTR_PAIRS],
			c->cfg.max_contacts);
	const uint32_t total = h[CTR_MANIFOLDS]; // manifolds with points = the touching output
	if (total > c->cfg.max_contacts)
		return fail(c, B3G_E_CAPACITY, "b3g_fetch_results_async: %u manifolds exceed the output buffer", total);
	Buffers& B = c->buf;
	wait_copies(c, c->stream);
	if (n && touchCapacity)
	{
		uint32_t* offsets = B.leafCount;
		const DevManifold* extra = B.extraMan[c->cur] ? B.extraMan[c->cur] : B.man[c->cur];
		k_touch_flags<<<(n + 255) / 256, 256, 0, c->stream>>>(B.man[c->cur], extra, B.cstate[c->cur], n, offsets);
		scan_exclusive(offsets, n, B.scanAux, B.counters + CTR_TOUCH_OUT, B.counters + CTR_STATUS, c->stream);
		k_touch_scatter<<<(n + 255) / 256, 256, 0, c->stream>>>(B.man[c->cur], extra, B.cstate[c->cur], offsets, n,
			B.touchIndex, B.touchMan);
	}
	CK(cudaEventRecord(c->copyReady, c->stream));
	CK(cudaStreamWaitEvent(c->copyStream, c->copyReady, 0));
	const uint32_t nc = std::min(n, contactCapacity);
	if (nc)
		CK(cudaMemcpyAsync(contacts, B.contactOut, sizeof(uint32_t) * 3 * nc, cudaMemcpyDeviceToHost, c->copyStream));
	const uint32_t nt = std::min(total, touchCapacity);
	if (n && nt)
	{
		CK(cudaMemcpyAsync(index, B.touchIndex, sizeof(uint32_t) * nt, cudaMemcpyDeviceToHost, c->copyStream));
		CK(cudaMemcpyAsync(manifolds, B.touchMan, sizeof(DevManifold) * nt, cudaMemcpyDeviceToHost, c->copyStream));
	}
	CK(cudaEventRecord(c->copyDone, c->copyStream));
	c->copyPending = true;
	return B3G_OK;
}

extern "C" int b3g_fetch_results_packed_async(b3g_ctx* c, uint32_t* contacts, uint32_t contactCapacity,
	uint32_t* index, void* packed, uint32_t touchCapacity, uint64_t packedCapacity, b3g_counts* counts)
{
	if (!c || !counts || (contactCapacity && !contacts) || (touchCapacity && (!index || !packed)))
		return fail(c, B3G_E_INVALID, "null argument");
	if (!c->havePass)
		return fail(c, B3G_E_STATE, "no pass yet");
	CK(cudaSetDevice(c->device));
	CK(cudaMemcpyAsync(c->hCounters, c->buf.counters, sizeof(uint32_t) * CTR_COUNT, cudaMemcpyDeviceToHost,
		c->stream));
	CK(cudaStreamSynchronize(c->stream));
	const uint32_t* h = c->hCounters;
	const uint32_t n = std::min(h[CTR_PAIRS], c->cfg.max_contacts);
	counts->contacts = n;
	counts->begun = h[CTR_BEGUN];
	counts->ended = h[CTR_ENDED];
	counts->touching = h[CTR_TOUCHING];
	counts->manifolds = h[CTR_MANIFOLDS];
	counts->points = h[CTR_POINTS];
	counts->moved = h[CTR_MOVED];
	counts->status = status_code(h[CTR_STATUS]);
	if (counts->status)
		return fail(c, -(int)counts->status, "pass status 0x%x (pairs %u, capacity %u)", h[CTR_STATUS], h[CTR_PAIRS],
			c->cfg.max_contacts);
	const uint32_t total = h[CTR_MANIFOLDS];
	const uint64_t bytes = 32ull * total + 72ull * h[CTR_POINTS];
	if (total > c->cfg.max_contacts)
		return fail(c, B3G_E_CAPACITY, "b3g_fetch_results_packed_async: %u manifolds exceed the output buffer", total);
	if (touchCapacity && (total > touchCapacity || bytes > packedCapacity))
		return fail(c, B3G_E_CAPACITY, "b3g_fetch_results_packed_async: %u manifolds, %llu bytes do not fit", total,
			(unsigned long long)bytes);
	Buffers& B = c->buf;
	if (!c->touchBytes)
		CK(cudaMalloc((void**)&c->touchBytes, sizeof(uint32_t) * std::max<size_t>(c->cfg.max_contacts, 1)));
	wait_copies(c, c->stream);
	if (n && touchCapacity)
	{
		const DevManifold* extra = B.extraMan[c->cur] ? B.extraMan[c->cur] : B.man[c->cur];
		k_pack_sizes<<<(n + 255) / 256, 256, 0, c->stream>>>(B.man[c->cur], extra, B.cstate[c->cur], n, B.leafCount,
			c->touchBytes);
		scan_exclusive(B.leafCount, n, B.scanAux, B.counters + CTR_TOUCH_OUT, B.counters + CTR_STATUS, c->stream);
		scan_exclusive(c->touchBytes, n, B.scanAux, B.counters + CTR_SCRATCH, B.counters + CTR_STATUS, c->stream);
		k_pack_scatter<<<(n + 255) / 256, 256, 0, c->stream>>>(B.man[c->cur], extra, B.cstate[c->cur], n, B.leafCount,
			c->touchBytes, B.touchIndex, reinterpret_cast<unsigned long long*>(B.touchMan));
	}
	CK(cudaEventRecord(c->copyReady, c->stream));
	CK(cudaStreamWaitEvent(c->copyStream, c->copyReady, 0));
	const uint32_t nc = std::min(n, contactCapacity);
	if (nc)
		CK(cudaMemcpyAsync(contacts, B.contactOut, sizeof(uint32_t) * 3 * nc, cudaMemcpyDeviceToHost, c->copyStream));
	if (n && touchCapacity && total)
	{
		CK(cudaMemcpyAsync(index, B.touchIndex, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost, c->copyStream));
		CK(cudaMemcpyAsync(packed, B.touchMan, (size_t)bytes, cudaMemcpyDeviceToHost, c->copyStream));
	}
	CK(cudaEventRecord(c->copyDone, c->copyStream));
	c->copyPending = true;
	return B3G_OK;
}

extern "C" int b3g_wait_results(b3g_ctx* c)
{
	if (!c)
		return B3G_E_INVALID;
	if (c->copyPending)
	{
		CK(cudaSetDevice(c->device));
		CK(cudaEventSynchronize(c->copyDone));
	}
	return B3G_OK;
}

extern "C" int b3g_fetch_fixture_contacts(b3g_ctx* c, uint32_t* offsets, uint32_t* contacts, uint32_t capacity)
{
	if (!c || !offsets || (capacity && !contacts))
		return fail(c, B3G_E_INVALID, "null argument");
	uint32_t n;
	int rc = contacts_now(c, n);
	if (rc)
		return rc;
	const uint32_t nf = c->nFixtures;
	const uint32_t m = 2 * n;
	int bits = 1;
	while (bits < 32 && (1u << bits) < nf)
		++bits;
	auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
	const size_t need = 2 * al(8 * (size_t)m) + 2 * al(4 * (size_t)m) + al(4 * ((size_t)nf + 1)) +
		al(4 * (size_t)radix_sort_scratch_words(std::max(m, 1u), bits));
	if (c->edgeBytes < need)
	{
		if (c->edgeBuf)
			CK(cudaFree(c->edgeBuf));
		c->edgeBuf = nullptr;
		c->edgeBytes = 0;
		CK(cudaMalloc(&c->edgeBuf, need));
		c->edgeBytes = need;
	}
	char* p = (char*)c->edgeBuf;
	unsigned long long* keys = (unsigned long long*)p;
	p += al(8 * (size_t)m);
	unsigned long long* keysTmp = (unsigned long long*)p;
	p += al(8 * (size_t)m);
	uint32_t* vals = (uint32_t*)p;
	p += al(4 * (size_t)m);
	uint32_t* valsTmp = (uint32_t*)p;
	p += al(4 * (size_t)m);
	uint32_t* counts = (uint32_t*)p;
	p += al(4 * ((size_t)nf + 1));
	uint32_t* scratch = (uint32_t*)p;
	Buffers& B = c->buf;
	cudaStream_t s = c->stream;
	CK(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * ((size_t)nf + 1), s));
	if (n)
		k_edge_records<<<(n + 255) / 256, 256, 0, s>>>(B.pairA[c->cur], B.pairB[c->cur], n, keys, vals, counts);
	// Fixture f's edges are the contact list filtered to f, in list order:
	// AddPair prepends a contact to the list and to both fixtures' edge lists
	// (contact_manager.cpp:105-137), Destroy unlinks it from all three. A
	// stable sort by fixture of the records, taken in contact order, gives
	// every fixture's edges in its own list's order.
	bool swapped = m ? radix_sort_pairs(keys, vals, keysTmp, valsTmp, m, bits, scratch, B.counters + CTR_STATUS, s)
					 : false;
	scan_exclusive(counts, nf, B.scanAux, counts + nf, B.counters + CTR_STATUS, s);
	CK(cudaStreamSynchronize(s));
	CK(cudaMemcpy(offsets, counts, sizeof(uint32_t) * ((size_t)nf + 1), cudaMemcpyDeviceToHost));
	const uint32_t k = std::min(m, capacity);
	if (k)
		CK(cudaMemcpy(contacts, swapped ? valsTmp : vals, sizeof(uint32_t) * k, cudaMemcpyDeviceToHost));
	return (int)m;
}

extern "C" int b3g_set_materials(b3g_ctx* c, const float* friction, const float* restitution)
{
	if (!c || !friction || !restitution)
		return fail(c, B3G_E_INVALID, "b3g_set_materials: null argument");
	if (!c->dFixMaterial)
		return fail(c, B3G_E_STATE, "b3g_set_materials: no fixtures yet");
	const uint32_t nf = c->nFixtures;
	std::vector<float2> mat(std::max(nf, 1u), make_float2(0.3f, 0.0f));
	for (uint32_t i = 0; i < nf; ++i)
		mat[i] = make_float2(friction[i], restitution[i]);
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	CK(cudaMemcpy(c->dFixMaterial, mat.data(), sizeof(float2) * nf, cudaMemcpyHostToDevice));
	return B3G_OK;
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

extern "C" int b3g_contact_constraints_device(b3g_ctx* c, uint32_t count, const uint32_t* contacts,
	const b3g_solver_body* bodies, float dtRatio, int warm, b3g_contact_constraint* constraints, uint32_t cCap,
	b3g_manifold_constraint* manifolds, uint32_t mCap, uint32_t* counts, void* stream)
{
	if (!c || !bodies || !counts)
		return fail(c, B3G_E_INVALID, "b3g_contact_constraints_device: null argument");
	if (!aligned16(bodies) || !aligned16(constraints) || !aligned16(manifolds))
		return fail(c, B3G_E_INVALID, "b3g_contact_constraints_device: buffers must be 16-byte aligned");
	if (!c->havePass)
		return fail(c, B3G_E_STATE, "b3g_contact_constraints_device: no pass yet");
	if (contacts && count > c->cfg.max_contacts)
		return fail(c, B3G_E_CAPACITY, "b3g_contact_constraints_device: %u contacts exceed max_contacts %u", count,
			c->cfg.max_contacts);
	CK(cudaSetDevice(c->device));
	// Tile counter and one status word per tile of the largest call.
	const uint32_t words = contact_constraint_tiles(c->cfg.max_contacts) + 1;
	if (c->ciTileCap < words)
	{
		dfree(c->ciTiles);
		c->ciTileCap = 0;
		CK(dalloc(&c->ciTiles, words));
		c->ciTileCap = words;
	}
	ConstraintCall q;
	q.list = contacts;
	q.listCount = contacts ? count : 0;
	q.material = c->dFixMaterial;
	q.bodies = bodies;
	q.dtRatio = dtRatio;
	q.warm = warm ? 1 : 0;
	q.tiles = c->ciTiles;
	q.counts = counts;
	q.constraints = constraints;
	q.constraintCap = constraints ? cCap : 0;
	q.manifolds = manifolds;
	q.manifoldCap = manifolds ? mCap : 0;
	launch_contact_constraints(c, q, stream ? (cudaStream_t)stream : c->stream);
	CK(cudaGetLastError());
	return B3G_OK;
}

extern "C" int b3g_contact_constraints(b3g_ctx* c, uint32_t count, const uint32_t* contacts,
	const b3g_solver_body* bodies, float dtRatio, int warm, b3g_contact_constraint* constraints, uint32_t cCap,
	b3g_manifold_constraint* manifolds, uint32_t mCap, uint32_t* counts)
{
	if (!c || !bodies || !counts || (cCap && !constraints) || (mCap && !manifolds))
		return fail(c, B3G_E_INVALID, "b3g_contact_constraints: null argument");
	uint32_t n;
	int rc = contacts_now(c, n);
	if (rc)
		return rc;
	if (contacts)
	{
		if (count > c->cfg.max_contacts)
			return fail(c, B3G_E_CAPACITY, "b3g_contact_constraints: %u contacts exceed max_contacts %u", count,
				c->cfg.max_contacts);
		for (uint32_t i = 0; i < count; ++i)
			if (contacts[i] >= n)
				return fail(c, B3G_E_INVALID, "b3g_contact_constraints: contact %u of %u past the list", contacts[i],
					n);
	}
	// Device copies: bodies, the list, counts, then the records (sized for
	// every selected contact: at most max_contacts constraints, 3 manifolds
	// each, bounded by the capacities asked for).
	auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
	const uint32_t nb = c->nBodies;
	const uint32_t cMax = std::min(cCap, contacts ? count : n);
	const uint32_t mMax = std::min<uint64_t>(mCap, 3ull * (contacts ? count : n));
	const size_t need = al(sizeof(b3g_solver_body) * std::max(nb, 1u)) + al(4 * (size_t)std::max(count, 1u)) +
		al(8) + al(sizeof(b3g_contact_constraint) * std::max(cMax, 1u)) +
		al(sizeof(b3g_manifold_constraint) * std::max(mMax, 1u));
	if (c->ciHostBytes < need)
	{
		if (c->ciHost)
			CK(cudaFree(c->ciHost));
		c->ciHost = nullptr;
		c->ciHostBytes = 0;
		CK(cudaMalloc(&c->ciHost, need));
		c->ciHostBytes = need;
	}
	char* p = (char*)c->ciHost;
	b3g_solver_body* dBodies = (b3g_solver_body*)p;
	p += al(sizeof(b3g_solver_body) * std::max(nb, 1u));
	uint32_t* dList = (uint32_t*)p;
	p += al(4 * (size_t)std::max(count, 1u));
	uint32_t* dCounts = (uint32_t*)p;
	p += al(8);
	b3g_contact_constraint* dCon = (b3g_contact_constraint*)p;
	p += al(sizeof(b3g_contact_constraint) * std::max(cMax, 1u));
	b3g_manifold_constraint* dMan = (b3g_manifold_constraint*)p;
	cudaStream_t s = c->stream;
	if (nb)
		CK(cudaMemcpyAsync(dBodies, bodies, sizeof(b3g_solver_body) * nb, cudaMemcpyHostToDevice, s));
	if (contacts && count)
		CK(cudaMemcpyAsync(dList, contacts, 4 * (size_t)count, cudaMemcpyHostToDevice, s));
	rc = b3g_contact_constraints_device(c, count, contacts ? dList : nullptr, dBodies, dtRatio, warm, dCon, cMax,
		dMan, mMax, dCounts, s);
	if (rc)
		return rc;
	CK(cudaMemcpyAsync(counts, dCounts, 8, cudaMemcpyDeviceToHost, s));
	CK(cudaStreamSynchronize(s));
	const uint32_t kc = std::min(counts[0], cMax), km = std::min(counts[1], mMax);
	if (kc)
		CK(cudaMemcpy(constraints, dCon, sizeof(b3g_contact_constraint) * kc, cudaMemcpyDeviceToHost));
	if (km)
		CK(cudaMemcpy(manifolds, dMan, sizeof(b3g_manifold_constraint) * km, cudaMemcpyDeviceToHost));
	return (int)counts[0];
}

extern "C" int b3g_fetch_ended(b3g_ctx* c, uint32_t* out, uint32_t capacity)
{
	if (!c || !out)
		return fail(c, B3G_E_INVALID, "null argument");
	uint32_t n;
	int rc = contacts_now(c, n);
	if (rc)
		return rc;
	uint32_t m = std::min(c->hCounters[CTR_ENDED], capacity);
	if (m)
		CK(cudaMemcpy(out, c->buf.endedList, sizeof(uint32_t) * 3 * m, cudaMemcpyDeviceToHost));
	return (int)m;
}

extern "C" int b3g_fetch_caches(b3g_ctx* c, uint32_t* out, uint32_t capacity)
{
	if (!c || !out)
		return fail(c, B3G_E_INVALID, "null argument");
	uint32_t n;
	int rc = contacts_now(c, n);
	if (rc)
		return rc;
	n = std::min(n, capacity);
	if (n)
		CK(cudaMemcpy(out, c->buf.cache[c->cur], sizeof(uint4) * n, cudaMemcpyDeviceToHost));
	return (int)n;
}

extern "C" int b3g_fetch_fat_aabbs(b3g_ctx* c, float* out, uint32_t capacity)
{
	if (!c || !out)
		return fail(c, B3G_E_INVALID, "null argument");
	if (!c->havePass)
		return fail(c, B3G_E_STATE, "no pass yet");
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	uint32_t n = std::min(c->nFixtures, capacity);
	std::vector<float4> lo(n), hi(n);
	if (n)
	{
		CK(cudaMemcpy(lo.data(), c->buf.fatLo, sizeof(float4) * n, cudaMemcpyDeviceToHost));
		CK(cudaMemcpy(hi.data(), c->buf.fatHi, sizeof(float4) * n, cudaMemcpyDeviceToHost));
	}
	for (uint32_t i = 0; i < n; ++i)
	{
		out[6 * i + 0] = lo[i].x;
		out[6 * i + 1] = lo[i].y;
		out[6 * i + 2] = lo[i].z;
		out[6 * i + 3] = hi[i].x;
		out[6 * i + 4] = hi[i].y;
		out[6 * i + 5] = hi[i].z;
	}
	return (int)n;
}

extern "C" int b3g_load_impulses(b3g_ctx* c, const float* normal, const float* tangent, const float* motor)
{
	if (!c || !normal || !tangent || !motor)
		return fail(c, B3G_E_INVALID, "null argument");
	uint32_t n;
	int rc = contacts_now(c, n);
	if (rc)
		return rc;
	if (n)
	{
		CK(cudaMemcpy(c->buf.impulseNormal, normal, sizeof(float) * 4 * n, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->buf.impulseTangent, tangent, sizeof(float) * 2 * n, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(c->buf.impulseMotor, motor, sizeof(float) * n, cudaMemcpyHostToDevice));
	}
	c->impulsesLoaded = true;
	return B3G_OK;
}

namespace {

// Writes the host solver's impulses into manifolds 1 and 2 of each mesh
// contact of the last pass; the next pass's warm start reads them there as
// b3Manifold::Initialize(old) reads the old manifolds (collision.cpp:40-61).
__global__ void k_load_extra_impulses(DevManifold* extra, const uint32_t* cstate, uint32_t n, const float* normal,
	const float* tangent, const float* motor)
{
	uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= n)
		return;
	uint32_t mc = (cstate[c] >> 8) & 0xFFu;
	for (uint32_t k = 0; k + 1 < mc && k < 2; ++k)
	{
		DevManifold& m = extra[2 * (size_t)c + k];
		m.tangentImpulse[0] = tangent[4 * (size_t)c + 2 * k];
		m.tangentImpulse[1] = tangent[4 * (size_t)c + 2 * k + 1];
		m.motorImpulse = motor[2 * (size_t)c + k];
		for (uint32_t j = 0; j < m.pointCount && j < 4; ++j)
			m.points[j].normalImpulse = normal[8 * (size_t)c + 4 * k + j];
	}
}

} // namespace

extern "C" int b3g_load_mesh_impulses(b3g_ctx* c, const float* normal, const float* tangent, const float* motor)
{
	if (!c || !normal || !tangent || !motor)
		return fail(c, B3G_E_INVALID, "null argument");
	uint32_t n;
	int rc = contacts_now(c, n);
	if (rc)
		return rc;
	Buffers& B = c->buf;
	if (n == 0 || !B.extraMan[c->cur])
		return B3G_OK;
	float* dn = B.meshImpulses; // 14 floats per contact slot
	float* dt = dn + 8 * (size_t)n;
	float* dm = dt + 4 * (size_t)n;
	CK(cudaMemcpyAsync(dn, normal, sizeof(float) * 8 * n, cudaMemcpyHostToDevice, c->stream));
	CK(cudaMemcpyAsync(dt, tangent, sizeof(float) * 4 * n, cudaMemcpyHostToDevice, c->stream));
	CK(cudaMemcpyAsync(dm, motor, sizeof(float) * 2 * n, cudaMemcpyHostToDevice, c->stream));
	k_load_extra_impulses<<<(n + 255) / 256, 256, 0, c->stream>>>(B.extraMan[c->cur], B.cstate[c->cur], n, dn, dt, dm);
	CK(cudaStreamSynchronize(c->stream));
	return B3G_OK;
}

extern "C" int b3g_device_results(b3g_ctx* c, const void** contacts, const void** manifolds)
{
	if (!c || !contacts || !manifolds)
		return fail(c, B3G_E_INVALID, "null argument");
	*contacts = c->buf.contactOut;
	*manifolds = c->buf.man[c->cur];
	return B3G_OK;
}

// Stand-alone narrowphase over a caller's pair list (see include/b3g.h).
extern "C" int b3g_collide_pairs(b3g_ctx* c, uint32_t n, const uint32_t* fixA, const uint32_t* fixB,
	const float* xfA, const float* xfB, const float* xf0A, const float* xf0B, uint32_t* cache4, void* manifolds)
{
	if (!c || (n && (!fixA || !fixB || !xfA || !xfB || !manifolds)))
		return fail(c, B3G_E_INVALID, "b3g_collide_pairs: null argument");
	if (n == 0)
		return B3G_OK;
	CK(cudaSetDevice(c->device));
	if (c->fixTypeStale)
	{
		CK(cudaDeviceSynchronize());
		CK(cudaMemcpy(c->hFixType.data(), c->dFixType, sizeof(uint32_t) * c->hFixType.size(), cudaMemcpyDeviceToHost));
		c->fixTypeStale = false;
	}
	std::vector<std::vector<uint32_t>> lists(BK_COUNT);
	for (uint32_t i = 0; i < n; ++i)
	{
		if (fixA[i] >= c->nFixtures || fixB[i] >= c->nFixtures)
			return fail(c, B3G_E_INVALID, "pair %u: fixture out of range", i);
		uint32_t ta = c->hFixType[fixA[i]], tb = c->hFixType[fixB[i]];
		uint32_t bk = BK_COUNT;
		if (ta == B3G_SHAPE_SPHERE && tb == B3G_SHAPE_SPHERE)
			bk = BK_SPHERES;
		else if (ta == B3G_SHAPE_CAPSULE && tb == B3G_SHAPE_SPHERE)
			bk = BK_CAPSULE_SPHERE;
		else if (ta == B3G_SHAPE_CAPSULE && tb == B3G_SHAPE_CAPSULE)
			bk = BK_CAPSULES;
		else if (ta == B3G_SHAPE_HULL && tb == B3G_SHAPE_SPHERE)
			bk = BK_HULL_SPHERE;
		else if (ta == B3G_SHAPE_HULL && tb == B3G_SHAPE_CAPSULE)
			bk = BK_HULL_CAPSULE;
		else if (ta == B3G_SHAPE_HULL && tb == B3G_SHAPE_HULL)
			bk = BK_HULLS;
		else if (ta == B3G_SHAPE_TRIANGLE && tb == B3G_SHAPE_SPHERE)
			bk = BK_TRIANGLE_SPHERE;
		else if (ta == B3G_SHAPE_TRIANGLE && tb == B3G_SHAPE_CAPSULE)
			bk = BK_TRIANGLE_CAPSULE;
		else if (ta == B3G_SHAPE_HULL && tb == B3G_SHAPE_TRIANGLE)
			bk = BK_HULL_TRIANGLE;
		if (bk == BK_COUNT)
			return fail(c, B3G_E_INVALID, "pair %u: shape pair (%u, %u) not supported here", i, ta, tb);
		lists[bk].push_back(i);
	}
	uint32_t *dA = nullptr, *dB = nullptr, *dState = nullptr, *dList = nullptr, *dCount = nullptr, *dPrevState = nullptr;
	uint32_t* dStatus = nullptr;
	uint32_t *dMiss = nullptr, *dMissCount = nullptr;
	float4* dPost = nullptr;
	uint32_t* dHsPost = nullptr;
	int32_t* dPrev = nullptr;
	uint4 *dCache = nullptr, *dCacheIn = nullptr;
	float *dXA = nullptr, *dXB = nullptr, *dX0A = nullptr, *dX0B = nullptr;
	DevManifold *dMan = nullptr, *dPrevMan = nullptr;
	int rc = B3G_OK;
	auto step = [&](cudaError_t e) {
		if (rc == B3G_OK && e != cudaSuccess)
			rc = fail(c, B3G_E_CUDA, "b3g_collide_pairs: %s", cudaGetErrorString(e));
	};
	step(dalloc(&dA, n));
	step(dalloc(&dB, n));
	step(dalloc(&dState, n));
	step(dalloc(&dPrevState, n));
	step(dalloc(&dList, n));
	step(dalloc(&dCount, BK_COUNT));
	step(dalloc(&dStatus, 1));
	step(dalloc(&dPrev, n));
	step(dalloc(&dCache, n));
	step(dalloc(&dCacheIn, n));
	step(dalloc(&dXA, 7 * (size_t)n));
	step(dalloc(&dXB, 7 * (size_t)n));
	step(dalloc(&dX0A, 7 * (size_t)n));
	step(dalloc(&dX0B, 7 * (size_t)n));
	step(dalloc(&dMan, n));
	step(dalloc(&dPrevMan, 1));
	step(dalloc(&dMiss, n));
	step(dalloc(&dMissCount, 4));
	step(dalloc(&dPost, 2 * (size_t)n));
	step(dalloc(&dHsPost, n));
	if (rc == B3G_OK)
	{
		std::vector<int32_t> prev(n);
		std::vector<uint4> cin(n);
		for (uint32_t i = 0; i < n; ++i)
		{
			prev[i] = (int32_t)i;
			cin[i] = cache4 ? make_uint4(cache4[4 * i], cache4[4 * i + 1], cache4[4 * i + 2], cache4[4 * i + 3])
							: make_uint4(0, 1, 0, 0);
		}
		step(cudaMemcpy(dA, fixA, 4 * n, cudaMemcpyHostToDevice));
		step(cudaMemcpy(dB, fixB, 4 * n, cudaMemcpyHostToDevice));
		step(cudaMemcpy(dXA, xfA, 28 * (size_t)n, cudaMemcpyHostToDevice));
		step(cudaMemcpy(dXB, xfB, 28 * (size_t)n, cudaMemcpyHostToDevice));
		step(cudaMemcpy(dX0A, xf0A ? xf0A : xfA, 28 * (size_t)n, cudaMemcpyHostToDevice));
		step(cudaMemcpy(dX0B, xf0B ? xf0B : xfB, 28 * (size_t)n, cudaMemcpyHostToDevice));
		step(cudaMemcpy(dPrev, prev.data(), 4 * n, cudaMemcpyHostToDevice));
		step(cudaMemcpy(dCacheIn, cin.data(), 16 * (size_t)n, cudaMemcpyHostToDevice));
		step(cudaMemset(dPrevState, 0, 4 * n));
		step(cudaMemset(dStatus, 0, 4));
		step(cudaMemset(dMissCount, 0, 16));
	}
	if (rc == B3G_OK)
	{
		NPArgs a;
		a.S = c->scene;
		a.pairA = dA;
		a.pairB = dB;
		a.cstate = dState;
		a.cache = dCache;
		a.man = dMan;
		a.prevState = dPrevState; // manifold count 0: no warm start
		a.prevCache = dCacheIn;
		a.prevMan = dPrevMan;
		a.prevIndex = dPrev;
		a.status = dStatus;
		a.warmStarting = 0;
		a.convexCache = (c->cfg.flags & B3G_FLAG_CONVEX_CACHE) ? 1 : 0;
		a.impN = a.impT = a.impM = nullptr;
		a.exA = dXA;
		a.exB = dXB;
		a.ex0A = dX0A;
		a.ex0B = dX0B;
		a.missList = dMiss;
		a.missCount = dMissCount;
		a.hcPost = dPost;
		a.hcPostCount = dMissCount + 1;
		a.hcPostCap = n;
		a.hsPost = dHsPost;
		a.hsPostCount = dMissCount + 3;
		a.extraCur = nullptr;
		a.extraPrev = nullptr;
		std::vector<uint32_t> flat(n), counts(BK_COUNT, 0);
		std::vector<uint32_t> offs(BK_COUNT, 0);
		uint32_t o = 0;
		for (int b = 0; b < BK_COUNT; ++b)
		{
			offs[b] = o;
			counts[b] = (uint32_t)lists[b].size();
			for (uint32_t v : lists[b])
				flat[o++] = v;
		}
		step(cudaMemcpy(dList, flat.data(), 4 * n, cudaMemcpyHostToDevice));
		step(cudaMemcpy(dCount, counts.data(), 4 * BK_COUNT, cudaMemcpyHostToDevice));
		if (rc == B3G_OK)
		{
			// One launch per bucket with the list offset by the bucket start.
			for (int b = 0; b < BK_COUNT; ++b)
			{
				if (!counts[b])
					continue;
				if (b == BK_HULLS)
				{
					launch_hulls(a, dList + offs[b], dCount + b, c->maxUniqueEdges, c->tune, c->stream);
				}
				else if (b == BK_HULL_TRIANGLE)
				{
					launch_hull_triangles(a, dList + offs[b], dCount + b, c->maxUniqueEdges, c->tune, c->stream);
				}
				else
				{
					// launch_convex_buckets indexes lists by bucket * cap; give it a
					// view where only bucket b is non-empty.
					std::vector<uint32_t> one(BK_COUNT, 0);
					one[b] = counts[b];
					uint32_t* dOne = nullptr;
					step(dalloc(&dOne, BK_COUNT));
					step(cudaMemcpy(dOne, one.data(), 4 * BK_COUNT, cudaMemcpyHostToDevice));
					launch_convex_buckets(a, dList + offs[b] - (size_t)b * n, dOne, n, c->tune, c->stream);
					step(cudaStreamSynchronize(c->stream));
					dfree(dOne);
				}
			}
			step(cudaStreamSynchronize(c->stream));
			step(cudaGetLastError());
		}
		if (rc == B3G_OK)
		{
			step(cudaMemcpy(manifolds, dMan, sizeof(DevManifold) * n, cudaMemcpyDeviceToHost));
			if (cache4)
			{
				std::vector<uint4> cout(n);
				step(cudaMemcpy(cout.data(), dCache, 16 * (size_t)n, cudaMemcpyDeviceToHost));
				for (uint32_t i = 0; i < n; ++i)
				{
					cache4[4 * i + 0] = cout[i].x;
					cache4[4 * i + 1] = cout[i].y;
					cache4[4 * i + 2] = cout[i].z;
					cache4[4 * i + 3] = cout[i].w;
				}
			}
		}
	}
	dfree(dA);
	dfree(dB);
	dfree(dState);
	dfree(dPrevState);
	dfree(dList);
	dfree(dCount);
	dfree(dStatus);
	dfree(dPrev);
	dfree(dCache);
	dfree(dCacheIn);
	dfree(dXA);
	dfree(dXB);
	dfree(dX0A);
	dfree(dX0B);
	dfree(dMan);
	dfree(dPrevMan);
	dfree(dMiss);
	dfree(dMissCount);
	dfree(dPost);
	dfree(dHsPost);
	return rc;
}

// ---------------------------------------------------------------------------
// Launch shapes and the autotuner.

size_t hull_sat_smem(int warps, uint32_t maxUE);

namespace {

const uint32_t kBlocksPerSM[] = {1, 2, 4, 8, 16};
const uint32_t kSatWarps[] = {2, 4, 8};
const uint32_t kSatBlocks[] = {1, 2, 4, 8};
const uint32_t kTraverse[] = {64, 128, 256};

template <size_t N>
bool one_of(const uint32_t (&set)[N], uint32_t v)
{
	for (size_t i = 0; i < N; ++i)
		if (set[i] == v)
			return true;
	return false;
}

bool sat_fits(const b3g_ctx* c, uint32_t warps)
{
	int optin = 0;
	cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
	return hull_sat_smem((int)warps, c->maxUniqueEdges) <= (size_t)optin;
}

} // namespace

extern "C" int b3g_set_tuning(b3g_ctx* c, const uint32_t* t)
{
	if (!c || !t)
		return fail(c, B3G_E_INVALID, "b3g_set_tuning: null argument");
	for (int k = 0; k < B3G_CONVEX_KERNELS; ++k)
		if (!one_of(kBlocksPerSM, t[B3G_TUNE_CONVEX + k]))
			return fail(c, B3G_E_INVALID, "tuning[%d] = %u: not a candidate", B3G_TUNE_CONVEX + k, t[k]);
	if (!one_of(kBlocksPerSM, t[B3G_TUNE_PROBE]) || !one_of(kSatWarps, t[B3G_TUNE_SAT_WARPS]) ||
		!one_of(kSatBlocks, t[B3G_TUNE_SAT_BLOCKS]) || !one_of(kTraverse, t[B3G_TUNE_TRAVERSE]))
		return fail(c, B3G_E_INVALID, "b3g_set_tuning: value outside the candidate sets");
	CK(cudaSetDevice(c->device));
	if (!sat_fits(c, t[B3G_TUNE_SAT_WARPS]))
		return fail(c, B3G_E_INVALID, "b3g_set_tuning: %u SAT warps need more shared memory than a block has",
			t[B3G_TUNE_SAT_WARPS]);
	CK(cudaDeviceSynchronize());
	destroy_graphs(c);
	for (int k = 0; k < B3G_TUNE_COUNT; ++k)
		c->tune.v[k] = t[k];
	return B3G_OK;
}

extern "C" int b3g_set_walk_limit(b3g_ctx* c, uint32_t maxNodes)
{
	if (!c)
		return B3G_E_INVALID;
	CK(cudaSetDevice(c->device));
	CK(cudaDeviceSynchronize());
	destroy_graphs(c); // captured passes hold the old limit
	c->walkLimit = maxNodes;
	return B3G_OK;
}

extern "C" int b3g_set_tree_rebuild_interval(b3g_ctx* c, uint32_t passes)
{
	if (!c)
		return B3G_E_INVALID;
	if (passes == 0)
		return fail(c, B3G_E_INVALID, "b3g_set_tree_rebuild_interval: the interval is at least 1 pass");
	CK(cudaSetDevice(c->device));
	CK(cudaDeviceSynchronize());
	destroy_graphs(c); // captured passes hold the old interval
	c->treeInterval = passes;
	c->treeForce = true;
	return B3G_OK;
}

extern "C" int b3g_get_tuning(b3g_ctx* c, uint32_t* t)
{
	if (!c || !t)
		return fail(c, B3G_E_INVALID, "b3g_get_tuning: null argument");
	for (int k = 0; k < B3G_TUNE_COUNT; ++k)
		t[k] = c->tune.v[k];
	return B3G_OK;
}

// Coordinate search over the launch shapes, each kernel timed alone on the
// last pass's data. A candidate replaces the current shape only when it is at
// least 3 % faster, so timing noise does not flip between equal shapes.
extern "C" int b3g_autotune(b3g_ctx* c, uint32_t reps, void* stream, uint32_t* out)
{
	if (!c)
		return B3G_E_INVALID;
	if (!c->havePass)
		return fail(c, B3G_E_STATE, "b3g_autotune: needs a pass first");
	if (reps == 0)
		reps = 10;
	CK(cudaSetDevice(c->device));
	cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
	CK(cudaDeviceSynchronize());
	uint32_t h[CTR_COUNT];
	CK(cudaMemcpy(h, c->buf.counters, sizeof(h), cudaMemcpyDeviceToHost));
	Buffers& B = c->buf;
	const uint32_t cap = c->cfg.max_contacts;
	// The narrowphase re-runs see exactly what the pass saw.
	const bool loaded = c->impulsesLoaded;
	c->impulsesLoaded = c->lastPassImpulses;
	NPArgs a = make_np_args(c);
	c->impulsesLoaded = loaded;
	cudaEvent_t e0, e1;
	CK(cudaEventCreate(&e0));
	CK(cudaEventCreate(&e1));
	int rc = B3G_OK;
	auto timeit = [&](auto&& body) -> float {
		body(); // warm-up
		cudaEventRecord(e0, s);
		for (uint32_t r = 0; r < reps; ++r)
			body();
		cudaEventRecord(e1, s);
		float ms = 0.0f;
		if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
			rc = B3G_E_CUDA;
		return ms;
	};
	auto pick = [&](uint32_t& slot, const uint32_t* cands, size_t nc, auto&& run) {
		float best = timeit(run);
		uint32_t bestV = slot;
		const uint32_t start = slot;
		for (size_t i = 0; i < nc && rc == B3G_OK; ++i)
		{
			if (cands[i] == start)
				continue;
			slot = cands[i];
			float ms = timeit(run);
			if (ms < 0.97f * best)
			{
				best = ms;
				bestV = cands[i];
			}
		}
		slot = bestV;
	};
	static const uint32_t convexBucket[B3G_CONVEX_KERNELS] = {BK_SPHERES, BK_CAPSULE_SPHERE, BK_CAPSULES,
		BK_TRIANGLE_SPHERE, BK_TRIANGLE_CAPSULE, BK_HULL_SPHERE, BK_HULL_CAPSULE, BK_SENSOR, BK_INACTIVE};
	for (int k = 0; k < B3G_CONVEX_KERNELS && rc == B3G_OK; ++k)
	{
		if (h[CTR_BUCKET0 + convexBucket[k]] == 0)
			continue;
		pick(c->tune.v[B3G_TUNE_CONVEX + k], kBlocksPerSM, 5,
			[&] { launch_convex_one(k, a, B.bucketList, B.counters + CTR_BUCKET0, cap, c->tune, s); });
	}
	const uint32_t* hullList = B.bucketList + (size_t)BK_HULLS * cap;
	const uint32_t* hullCount = B.counters + CTR_BUCKET0 + BK_HULLS;
	auto probe = [&] {
		cudaMemsetAsync(B.counters + CTR_HULL_MISS, 0, sizeof(uint32_t), s);
		launch_hulls_probe(a, hullList, hullCount, c->tune, s);
	};
	if (h[CTR_BUCKET0 + BK_HULLS] && rc == B3G_OK)
	{
		pick(c->tune.v[B3G_TUNE_PROBE], kBlocksPerSM, 5, probe);
		// The SAT kernel rewrites the caches the probe reads back: each run
		// is probe + SAT, so every run starts from the pass's inputs.
		uint32_t warps[3];
		size_t nw = 0;
		for (uint32_t w : kSatWarps)
			if (sat_fits(c, w))
				warps[nw++] = w;
		auto probeSat = [&] {
			probe();
			launch_hulls_sat(a, c->maxUniqueEdges, c->tune, s);
		};
		pick(c->tune.v[B3G_TUNE_SAT_WARPS], warps, nw, probeSat);
		pick(c->tune.v[B3G_TUNE_SAT_BLOCKS], kSatBlocks, 4, probeSat);
		probeSat();
	}
	if (rc == B3G_OK)
		pick(c->tune.v[B3G_TUNE_TRAVERSE], kTraverse, 3, [&] { launch_traverse(c, s); });
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	CK(cudaStreamSynchronize(s));
	CK(cudaGetLastError());
	if (rc != B3G_OK)
		return fail(c, rc, "b3g_autotune: timing failed");
	destroy_graphs(c);
	if (out)
		for (int k = 0; k < B3G_TUNE_COUNT; ++k)
			out[k] = c->tune.v[k];
	return B3G_OK;
}

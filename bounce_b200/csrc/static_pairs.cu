// Broadphase pair search that allocates nothing (b3g_find_pairs_static in
// include/b3g.h).
//
// Some callers cannot allocate device memory: an engine that hands every byte
// of GPU memory to its own arena, code running while a CUDA graph is being
// captured (cudaMalloc is not capturable), or a host thread that must not
// block on the allocator. This entry point serves them: its scratch is the
// file-scope array below, sized for B3G_STATIC_MAX_PROXIES proxies; the
// caller passes the fat AABBs and the output buffers, all in device memory.
//
// Algorithm (a variant of the pipeline's pair search, same closed overlap
// test b3TestOverlap, aabb.h:347-367): one block sorts the proxies by
// lower x (bitonic sort in shared memory), one thread per proxy sweeps
// forward while the next lower x does not pass its upper x and counts the
// y/z overlaps, a block scan turns counts into offsets, and the sweep runs
// again to write each pair (min index, max index).
//
// The array is shared by every call on a device and keeps the last call's
// contents; the counters that must start at zero are cleared by each call.
// Calls that overlap on the GPU (two streams, no ordering) race on it.

#include <mutex>

#include "b3g_internal.cuh"

namespace {

constexpr uint32_t SP_MAX = B3G_STATIC_MAX_PROXIES;
constexpr int SP_SORT_THREADS = 1024;

struct StaticPairScratch
{
	unsigned long long sorted[SP_MAX]; // (orderable lower x << 32) | proxy, ascending
	uint32_t offset[SP_MAX];           // pairs per sorted proxy, then exclusive offsets
	uint32_t total;                    // pairs found
	uint32_t pad[63];
};

static __device__ __align__(256) StaticPairScratch g_staticPairScratch;

__device__ __forceinline__ uint32_t orderable(float f)
{
	uint32_t u = __float_as_uint(f);
	return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// One block: load keys into shared memory, bitonic sort, store. Padding keys
// (all ones) sort last.
__global__ void __launch_bounds__(SP_SORT_THREADS) k_sp_sort(const float* aabbs, uint32_t n,
	StaticPairScratch* sc)
{
	extern __shared__ unsigned long long keys[];
	uint32_t m = 1;
	while (m < n)
		m <<= 1;
	for (uint32_t i = threadIdx.x; i < m; i += blockDim.x)
		keys[i] = i < n ? ((unsigned long long)orderable(aabbs[6 * (size_t)i]) << 32) | i : ~0ull;
	if (threadIdx.x == 0)
		sc->total = 0;
	__syncthreads();
	for (uint32_t k = 2; k <= m; k <<= 1)
	{
		for (uint32_t j = k >> 1; j > 0; j >>= 1)
		{
			for (uint32_t i = threadIdx.x; i < m; i += blockDim.x)
			{
				uint32_t p = i ^ j;
				if (p > i)
				{
					unsigned long long a = keys[i], b = keys[p];
					bool up = (i & k) == 0;
					if ((a > b) == up)
					{
						keys[i] = b;
						keys[p] = a;
					}
				}
			}
			__syncthreads();
		}
	}
	for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
		sc->sorted[i] = keys[i];
}

// Sweep from sorted position s: WRITE = false counts, true writes pairs.
template <bool WRITE>
__global__ void k_sp_sweep(const float* aabbs, uint32_t n, StaticPairScratch* sc, uint32_t* pairs,
	uint32_t capacity)
{
	uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n)
		return;
	uint32_t a = (uint32_t)(sc->sorted[s] & 0xFFFFFFFFu);
	const float* A = aabbs + 6 * (size_t)a;
	float ahx = A[3], aly = A[1], ahy = A[4], alz = A[2], ahz = A[5];
	uint32_t count = 0;
	uint32_t base = WRITE ? sc->offset[s] : 0;
	for (uint32_t t = s + 1; t < n; ++t)
	{
		uint32_t b = (uint32_t)(sc->sorted[t] & 0xFFFFFFFFu);
		const float* Bb = aabbs + 6 * (size_t)b;
		if (Bb[0] > ahx)
			break; // sorted by lower x: no later proxy overlaps in x
		if (ahy < Bb[1] || aly > Bb[4] || ahz < Bb[2] || alz > Bb[5])
			continue;
		if (WRITE)
		{
			uint32_t slot = base + count;
			if (slot < capacity)
			{
				pairs[2 * (size_t)slot + 0] = min(a, b);
				pairs[2 * (size_t)slot + 1] = max(a, b);
			}
		}
		++count;
	}
	if (!WRITE)
		sc->offset[s] = count;
}

// One block: exclusive scan of the counts, total to sc->total and *count.
__global__ void __launch_bounds__(1024) k_sp_scan(uint32_t n, StaticPairScratch* sc, uint32_t* countOut)
{
	__shared__ uint32_t part[1024];
	uint32_t per = (n + blockDim.x - 1) / blockDim.x;
	uint32_t beg = threadIdx.x * per, end = min(beg + per, n);
	uint32_t sum = 0;
	for (uint32_t i = beg; i < end; ++i)
		sum += sc->offset[i];
	part[threadIdx.x] = sum;
	__syncthreads();
	for (uint32_t off = 1; off < blockDim.x; off <<= 1)
	{
		uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
		__syncthreads();
		part[threadIdx.x] += v;
		__syncthreads();
	}
	uint32_t run = part[threadIdx.x] - sum;
	for (uint32_t i = beg; i < end; ++i)
	{
		uint32_t v = sc->offset[i];
		sc->offset[i] = run;
		run += v;
	}
	if (threadIdx.x == blockDim.x - 1)
	{
		sc->total = part[threadIdx.x];
		*countOut = part[threadIdx.x];
	}
}

// Per-device address of g_staticPairScratch. The host name of a __device__
// variable is only a stand-in, so the address is fetched with
// cudaGetSymbolAddress once per device, with that device current.
std::mutex g_spMutex;
StaticPairScratch* g_spAddr[64] = {};

} // namespace

extern "C" int b3g_find_pairs_static(const float* aabbs, uint32_t n, uint32_t* pairs, uint32_t capacity,
	uint32_t* count, void* stream)
{
	if (n > SP_MAX)
		return B3G_E_CAPACITY;
	if (!count || (n && (!aabbs || (capacity && !pairs))))
		return B3G_E_INVALID;
	// An error left pending by earlier work on this thread is not this call's:
	// leave it for its owner to read and run nothing. Past this check, a
	// launch error belongs to the launch just made.
	if (cudaPeekAtLastError() != cudaSuccess)
		return B3G_E_CUDA;
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
		return B3G_E_CUDA;
	StaticPairScratch* sc = nullptr;
	{
		std::lock_guard<std::mutex> lock(g_spMutex);
		if (!g_spAddr[dev])
		{
			void* p = nullptr;
			if (cudaGetSymbolAddress(&p, g_staticPairScratch) != cudaSuccess || !p)
				return B3G_E_CUDA;
			g_spAddr[dev] = (StaticPairScratch*)p;
		}
		sc = g_spAddr[dev];
	}
	cudaStream_t s = (cudaStream_t)stream;
	if (n < 2)
	{
		if (cudaMemsetAsync(count, 0, sizeof(uint32_t), s) != cudaSuccess)
			return B3G_E_CUDA;
		return B3G_OK;
	}
	uint32_t m = 1;
	while (m < n)
		m <<= 1;
	size_t smem = sizeof(unsigned long long) * m;
	if (smem > 48 * 1024 &&
		cudaFuncSetAttribute(k_sp_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
		return B3G_E_CUDA;
	k_sp_sort<<<1, SP_SORT_THREADS, smem, s>>>(aabbs, n, sc);
	if (cudaGetLastError() != cudaSuccess)
		return B3G_E_CUDA;
	k_sp_sweep<false><<<(n + 127) / 128, 128, 0, s>>>(aabbs, n, sc, pairs, capacity);
	if (cudaGetLastError() != cudaSuccess)
		return B3G_E_CUDA;
	k_sp_scan<<<1, 1024, 0, s>>>(n, sc, count);
	if (cudaGetLastError() != cudaSuccess)
		return B3G_E_CUDA;
	k_sp_sweep<true><<<(n + 127) / 128, 128, 0, s>>>(aabbs, n, sc, pairs, capacity);
	if (cudaGetLastError() != cudaSuccess)
		return B3G_E_CUDA;
	return B3G_OK;
}

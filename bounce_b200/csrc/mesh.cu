// Triangle meshes: b3Mesh upload (adjacency and static tree built on the
// host), the mesh fixtures' broadphase AABBs, and the mesh contacts' midphase
// and clustering (b3MeshContact, mesh_contact.cpp).
//
// Per pass, for every contact with a mesh fixture:
//  k_mesh_sync    b3MeshContact::SynchronizeFixture / MoveAABB (or the
//                 constructor's AABB for a new contact): the other shape's fat
//                 AABB in mesh space (mesh_contact.cpp:26-231); then the
//                 number of tree triangles it overlaps (b3StaticTree::QueryAABB)
//  scan + k_mesh_emit
//                 (contact, triangle) work items in the order the reference's
//                 query reports them (FindPairs / Report, :233-297)
//  evaluate       one work item = one b3Manifold of the child triangle
//                 (b3MeshShape::GetChildTriangle + b3CollideTriangleAndSphere /
//                 AndCapsule / b3CollideHullAndTriangle), points tagged with the
//                 triangle (narrow_convex.cu, narrow_hulls.cu)
//  k_mesh_cluster b3ClusterSolver::Run (cluster.cpp:202-585): k-means of the
//                 points' normals into at most 3 clusters, each reduced to at
//                 most 4 points; then b3Contact::Update's warm start over the
//                 previous manifolds (contact.cpp:424-446)

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "collide_common.cuh"

// ---------------------------------------------------------------------------
// Host: adjacency and static tree.

namespace {

struct HBox
{
	float lo[3], hi[3];
};

inline float center(const HBox& b, int axis) { return 0.5f * (b.lo[axis] + b.hi[axis]); }

// b3Mesh::BuildAdjacency (mesh.cpp:36-119): for each open edge of triangle i,
// the first later triangle with the same edge (either orientation) gives the
// wing vertices of both. An edge map replaces the quadratic search; it keeps
// each edge's users in triangle order, so the partner found is the same.
void build_adjacency(const uint32_t* tri, uint32_t T, std::vector<uint32_t>& wing)
{
	wing.assign(3 * (size_t)T, B3G_NULL);
	std::unordered_map<unsigned long long, std::vector<uint32_t>> users; // edge -> 3 * t + j
	users.reserve(3 * (size_t)T);
	for (uint32_t t = 0; t < T; ++t)
		for (uint32_t j = 0; j < 3; ++j)
		{
			uint32_t a = tri[3 * t + j], b = tri[3 * t + (j + 1) % 3];
			unsigned long long key = ((unsigned long long)std::min(a, b) << 32) | std::max(a, b);
			users[key].push_back(3 * t + j);
		}
	for (uint32_t i = 0; i < T; ++i)
		for (uint32_t j1 = 0; j1 < 3; ++j1)
		{
			if (wing[3 * i + j1] != B3G_NULL)
				continue;
			uint32_t k1 = j1 + 1 < 3 ? j1 + 1 : 0;
			uint32_t a = tri[3 * i + j1], b = tri[3 * i + k1];
			unsigned long long key = ((unsigned long long)std::min(a, b) << 32) | std::max(a, b);
			const std::vector<uint32_t>& u = users[key];
			for (uint32_t e : u)
			{
				uint32_t t2 = e / 3, j2 = e % 3;
				if (t2 <= i)
					continue;
				uint32_t k2 = j2 + 1 < 3 ? j2 + 1 : 0;
				uint32_t k3 = k1 + 1 < 3 ? k1 + 1 : 0;
				uint32_t k4 = k2 + 1 < 3 ? k2 + 1 : 0;
				wing[3 * t2 + j2] = tri[3 * i + k3];
				wing[3 * i + j1] = tri[3 * t2 + k4];
				break;
			}
		}
}

// b3StaticTree::Build (static_tree.cpp:22-167): top-down, nodes numbered in
// creation order (a node before its children, child1's subtree first); a
// node's triangles are sorted along its box's longest axis by centre
// (std::sort, as the reference) and split at the first centre past the box
// centre, or at the median when that leaves one side empty.
struct TreeBuilder
{
	const std::vector<HBox>& boxes;
	std::vector<HBox> nodeBox;
	std::vector<uint32_t> child1, child2; // child2 holds the triangle of a leaf

	explicit TreeBuilder(const std::vector<HBox>& b) : boxes(b) {}

	uint32_t build(uint32_t* idx, uint32_t count)
	{
		uint32_t id = (uint32_t)nodeBox.size();
		nodeBox.push_back(HBox());
		child1.push_back(B3G_NULL);
		child2.push_back(B3G_NULL);
		if (count <= 1)
		{
			nodeBox[id] = boxes[idx[0]];
			child1[id] = B3G_NULL;
			child2[id] = idx[0];
			return id;
		}
		HBox box = boxes[idx[0]];
		for (uint32_t i = 1; i < count; ++i)
			for (int k = 0; k < 3; ++k)
			{
				const HBox& b = boxes[idx[i]];
				box.lo[k] = b.lo[k] < box.lo[k] ? b.lo[k] : box.lo[k];
				box.hi[k] = box.hi[k] > b.hi[k] ? box.hi[k] : b.hi[k];
			}
		nodeBox[id] = box;
		// b3AABB::GetLongestAxis: the first largest extent
		float d[3] = {box.hi[0] - box.lo[0], box.hi[1] - box.lo[1], box.hi[2] - box.lo[2]};
		int axis = 0;
		float mx = d[0];
		if (d[1] > mx)
		{
			mx = d[1];
			axis = 1;
		}
		if (d[2] > mx)
			axis = 2;
		const std::vector<HBox>& bx = boxes;
		std::sort(idx, idx + count, [&](uint32_t i1, uint32_t i2) { return center(bx[i1], axis) < center(bx[i2], axis); });
		float split = center(box, axis);
		uint32_t k = 0;
		while (k < count && !(center(boxes[idx[k]], axis) > split))
			++k;
		if (k == 0 || k == count)
			k = count / 2;
		uint32_t c1 = build(idx, k);
		uint32_t c2 = build(idx + k, count - k);
		child1[id] = c1;
		child2[id] = c2;
		return id;
	}
};

float4 bits_w(const float* xyz, uint32_t w)
{
	float f;
	std::memcpy(&f, &w, 4);
	return make_float4(xyz[0], xyz[1], xyz[2], f);
}

int mesh_fail(b3g_ctx* c, int code, const char* msg)
{
	if (c)
		c->err = msg;
	return code;
}

template <class T>
cudaError_t mesh_alloc(T** p, size_t count)
{
	return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
}

template <class T>
void mesh_free(T*& p)
{
	if (p)
		cudaFree((void*)p);
	p = nullptr;
}

} // namespace

void free_mesh(b3g_ctx* c)
{
	mesh_free(c->dMeshes);
	mesh_free(c->dMeshVerts);
	mesh_free(c->dMeshTris);
	mesh_free(c->dMeshWings);
	mesh_free(c->dMeshNodes);
	Buffers& B = c->buf;
	for (int k = 0; k < 2; ++k)
	{
		mesh_free(B.meshAABB[k]);
		mesh_free(B.extraMan[k]);
	}
	mesh_free(B.meshCount);
	mesh_free(B.meshPairC);
	mesh_free(B.meshPairT);
	mesh_free(B.meshPairMan);
	mesh_free(B.meshObs);
	mesh_free(B.meshPoly);
	mesh_free(B.meshImpulses);
	B.meshPairCap = 0;
	c->nMeshes = 0;
	c->hMeshes.clear();
}

extern "C" int b3g_set_meshes(b3g_ctx* c, uint32_t nm, const uint32_t* desc, const float* verts,
	const uint32_t* tris, uint32_t maxTrianglePairs)
{
	if (!c || (nm && (!desc || !verts || !tris)))
		return mesh_fail(c, B3G_E_INVALID, "b3g_set_meshes: null argument");
	if (cudaSetDevice(c->device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
		return mesh_fail(c, B3G_E_CUDA, "b3g_set_meshes: device");
	free_mesh(c);
	std::vector<MeshDesc> md(nm);
	std::vector<float4> hv, nodes;
	std::vector<uint4> ht, hw;
	for (uint32_t m = 0; m < nm; ++m)
	{
		const uint32_t vOff = desc[4 * m], vCnt = desc[4 * m + 1], tOff = desc[4 * m + 2], tCnt = desc[4 * m + 3];
		if (vCnt == 0 || tCnt == 0)
			return mesh_fail(c, B3G_E_INVALID, "b3g_set_meshes: empty mesh");
		const uint32_t* tri = tris + 3 * (size_t)tOff;
		for (uint32_t i = 0; i < 3 * tCnt; ++i)
			if (tri[i] >= vCnt)
				return mesh_fail(c, B3G_E_INVALID, "b3g_set_meshes: triangle vertex out of range");
		const float* v = verts + 3 * (size_t)vOff;
		std::vector<uint32_t> wing;
		build_adjacency(tri, tCnt, wing);
		// b3Mesh::GetTriangleAABB (mesh.h:93-108): the vertices' box grown by
		// B3_LINEAR_SLOP.
		std::vector<HBox> boxes(tCnt);
		for (uint32_t t = 0; t < tCnt; ++t)
		{
			const float* a = v + 3 * tri[3 * t];
			const float* b = v + 3 * tri[3 * t + 1];
			const float* cc = v + 3 * tri[3 * t + 2];
			for (int k = 0; k < 3; ++k)
			{
				float mn = b[k] < cc[k] ? b[k] : cc[k];
				mn = a[k] < mn ? a[k] : mn;
				float mx = b[k] > cc[k] ? b[k] : cc[k];
				mx = a[k] > mx ? a[k] : mx;
				boxes[t].lo[k] = mn - B3G_LINEAR_SLOP;
				boxes[t].hi[k] = mx + B3G_LINEAR_SLOP;
			}
		}
		TreeBuilder tb(boxes);
		std::vector<uint32_t> idx(tCnt);
		for (uint32_t t = 0; t < tCnt; ++t)
			idx[t] = t;
		uint32_t root = tb.build(idx.data(), tCnt);
		md[m].vOff = (uint32_t)hv.size();
		md[m].vCnt = vCnt;
		md[m].tOff = (uint32_t)ht.size();
		md[m].tCnt = tCnt;
		md[m].nOff = (uint32_t)(nodes.size() / 2);
		md[m].nCnt = (uint32_t)tb.nodeBox.size();
		md[m].root = root;
		md[m].pad = 0;
		for (uint32_t i = 0; i < vCnt; ++i)
			hv.push_back(make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.0f));
		for (uint32_t t = 0; t < tCnt; ++t)
		{
			ht.push_back(make_uint4(tri[3 * t], tri[3 * t + 1], tri[3 * t + 2], 0));
			hw.push_back(make_uint4(wing[3 * t], wing[3 * t + 1], wing[3 * t + 2], 0));
		}
		for (size_t n = 0; n < tb.nodeBox.size(); ++n)
		{
			nodes.push_back(bits_w(tb.nodeBox[n].lo, tb.child1[n]));
			nodes.push_back(bits_w(tb.nodeBox[n].hi, tb.child2[n]));
		}
	}
	bool ok = true;
	auto up = [&](auto** dst, const auto& src) {
		if (!ok)
			return;
		ok = mesh_alloc(dst, src.size()) == cudaSuccess &&
			(src.empty() ||
				cudaMemcpy(*dst, src.data(), sizeof(src[0]) * src.size(), cudaMemcpyHostToDevice) == cudaSuccess);
	};
	up(&c->dMeshes, md);
	up(&c->dMeshVerts, hv);
	up(&c->dMeshTris, ht);
	up(&c->dMeshWings, hw);
	up(&c->dMeshNodes, nodes);
	// Per-contact mesh state and the work-item buffers.
	Buffers& B = c->buf;
	const size_t C = c->cfg.max_contacts;
	if (nm)
	{
		B.meshPairCap = maxTrianglePairs ? maxTrianglePairs : (uint32_t)std::min<size_t>(4 * C, 0x7FFFFFFF);
		for (int k = 0; k < 2 && ok; ++k)
		{
			ok = mesh_alloc(&B.meshAABB[k], 2 * C) == cudaSuccess && mesh_alloc(&B.extraMan[k], 2 * C) == cudaSuccess;
			if (ok)
				ok = cudaMemset(B.extraMan[k], 0, sizeof(DevManifold) * 2 * C) == cudaSuccess;
		}
		ok = ok && mesh_alloc(&B.meshCount, C + 1) == cudaSuccess && mesh_alloc(&B.meshPairC, B.meshPairCap) == cudaSuccess &&
			mesh_alloc(&B.meshPairT, B.meshPairCap) == cudaSuccess &&
			mesh_alloc(&B.meshPairMan, B.meshPairCap) == cudaSuccess &&
			mesh_alloc(&B.meshObs, 3 * 4 * (size_t)B.meshPairCap) == cudaSuccess &&
			mesh_alloc(&B.meshPoly, 4 * (size_t)B.meshPairCap) == cudaSuccess &&
			mesh_alloc(&B.meshImpulses, 14 * C) == cudaSuccess;
	}
	if (!ok)
	{
		free_mesh(c);
		return mesh_fail(c, B3G_E_CUDA, "b3g_set_meshes: device allocation failed");
	}
	c->nMeshes = nm;
	c->hMeshes = md;
	c->scene.meshes = c->dMeshes;
	c->scene.meshVerts = c->dMeshVerts;
	c->scene.meshTris = c->dMeshTris;
	c->scene.meshWings = c->dMeshWings;
	c->scene.meshNodes = c->dMeshNodes;
	c->creationPass = true;
	c->havePass = false;
	return B3G_OK;
}

extern "C" int b3g_mesh_wings(b3g_ctx* c, uint32_t m, uint32_t* out, uint32_t capacity)
{
	if (!c || !out)
		return mesh_fail(c, B3G_E_INVALID, "b3g_mesh_wings: null argument");
	if (m >= c->nMeshes)
		return mesh_fail(c, B3G_E_INVALID, "b3g_mesh_wings: no such mesh");
	const MeshDesc& d = c->hMeshes[m];
	uint32_t n = std::min(d.tCnt, capacity);
	std::vector<uint4> w(n);
	if (n && cudaMemcpy(w.data(), c->dMeshWings + d.tOff, sizeof(uint4) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
		return mesh_fail(c, B3G_E_CUDA, "b3g_mesh_wings: copy");
	for (uint32_t i = 0; i < n; ++i)
	{
		out[3 * i] = w[i].x;
		out[3 * i + 1] = w[i].y;
		out[3 * i + 2] = w[i].z;
	}
	return (int)n;
}

// ---------------------------------------------------------------------------
// Device.

namespace {

__device__ __forceinline__ bool is_mesh(const DevScene& S, uint32_t f) { return S.fixType[f] == B3G_SHAPE_MESH; }

__device__ __forceinline__ V3 mesh_scale(const DevScene& S, uint32_t f)
{
	float4 p = S.fixParams[3 * f];
	return V3{p.x, p.y, p.z};
}

// b3MeshContact::MoveAABB (mesh_contact.cpp:175-231): false when the box
// stays inside the old fat box.
__device__ __forceinline__ bool move_aabb(AABB& fat, const AABB& aabb, V3 d)
{
	if (aabb_contains(fat, aabb))
		return false;
	AABB f = aabb;
	aabb_extend(f, B3G_AABB_EXTENSION);
	if (d.x < 0.0f)
		f.lo.x += B3G_AABB_MULTIPLIER * d.x;
	else
		f.hi.x += B3G_AABB_MULTIPLIER * d.x;
	if (d.y < 0.0f)
		f.lo.y += B3G_AABB_MULTIPLIER * d.y;
	else
		f.hi.y += B3G_AABB_MULTIPLIER * d.y;
	if (d.z < 0.0f)
		f.lo.z += B3G_AABB_MULTIPLIER * d.z;
	else
		f.hi.z += B3G_AABB_MULTIPLIER * d.z;
	fat = f;
	return true;
}

// Broadphase AABB of each mesh fixture on a creation pass:
// b3MeshShape::ComputeAABB (mesh_shape.cpp:46-53) over every vertex, then the
// CreateProxy fattening. Min / max are exact, so the block reduction order
// does not matter.
__global__ void k_mesh_fat(DevScene S, Buffers B, const uint32_t* meshFix)
{
	__shared__ float red[6][256];
	const uint32_t f = meshFix[blockIdx.x];
	const MeshDesc md = S.meshes[S.fixHull[f]];
	const XF xf = load_xf(S.bodyState + 17 * (size_t)S.fixBody[f]);
	const V3 sc = mesh_scale(S, f);
	float lo[3] = {B3G_MAX_SCALAR, B3G_MAX_SCALAR, B3G_MAX_SCALAR};
	float hi[3] = {-B3G_MAX_SCALAR, -B3G_MAX_SCALAR, -B3G_MAX_SCALAR};
	for (uint32_t i = threadIdx.x; i < md.vCnt; i += blockDim.x)
	{
		float4 w = S.meshVerts[md.vOff + i];
		V3 p = xmul(xf, vmul(sc, V3{w.x, w.y, w.z}));
		lo[0] = fminr(lo[0], p.x), lo[1] = fminr(lo[1], p.y), lo[2] = fminr(lo[2], p.z);
		hi[0] = fmaxr(hi[0], p.x), hi[1] = fmaxr(hi[1], p.y), hi[2] = fmaxr(hi[2], p.z);
	}
	for (int k = 0; k < 3; ++k)
	{
		red[k][threadIdx.x] = lo[k];
		red[3 + k][threadIdx.x] = hi[k];
	}
	__syncthreads();
	for (uint32_t off = blockDim.x / 2; off > 0; off >>= 1)
	{
		if (threadIdx.x < off)
			for (int k = 0; k < 3; ++k)
			{
				red[k][threadIdx.x] = fminr(red[k][threadIdx.x], red[k][threadIdx.x + off]);
				red[3 + k][threadIdx.x] = fmaxr(red[3 + k][threadIdx.x], red[3 + k][threadIdx.x + off]);
			}
		__syncthreads();
	}
	if (threadIdx.x == 0)
	{
		AABB a;
		a.lo = V3{red[0][0], red[1][0], red[2][0]};
		a.hi = V3{red[3][0], red[4][0], red[5][0]};
		aabb_extend(a, S.fixParams[3 * f].w);
		aabb_extend(a, B3G_AABB_EXTENSION);
		B.fatLo[f] = make_float4(a.lo.x, a.lo.y, a.lo.z, 0.0f);
		B.fatHi[f] = make_float4(a.hi.x, a.hi.y, a.hi.z, 0.0f);
		B.moved[f] = 1;
	}
}

// The other shape's fat AABB in mesh space, and its triangle count.
__global__ void k_mesh_sync(DevScene S, Buffers B, uint32_t cur, uint32_t cap)
{
	uint32_t n = min(B.counters[CTR_PAIRS], cap);
	uint32_t prevBuf = cur ^ 1u;
	for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
	{
		uint32_t fa = B.pairA[cur][c], fb = B.pairB[cur][c];
		bool meshA = is_mesh(S, fa);
		if (!meshA && !is_mesh(S, fb))
		{
			B.meshCount[c] = 0;
			continue;
		}
		uint32_t mf = meshA ? fa : fb, of = meshA ? fb : fa;
		uint32_t mb = S.fixBody[mf], ob = S.fixBody[of];
		XF xfM = body_xf(S, mb), xfO = body_xf(S, ob);
		V3 sc = mesh_scale(S, mf);
		V3 inv = V3{1.0f / sc.x, 1.0f / sc.y, 1.0f / sc.z};
		int32_t prev = B.prevIndex[c];
		AABB fat;
		if (prev < 0)
		{
			// b3MeshContact::b3MeshContact (mesh_contact.cpp:28-92)
			AABB a, unused;
			compute_aabbs(S, of, xmult(xfM, xfO), xfO, false, a, unused);
			fat = aabb_scaled(a, inv);
			aabb_extend(fat, B3G_AABB_EXTENSION);
		}
		else
		{
			// b3MeshContact::SynchronizeFixture (mesh_contact.cpp:100-173)
			float4 l = B.meshAABB[prevBuf][2 * (size_t)prev], h = B.meshAABB[prevBuf][2 * (size_t)prev + 1];
			fat.lo = V3{l.x, l.y, l.z};
			fat.hi = V3{h.x, h.y, h.z};
			const float* st = S.bodyState + 17 * (size_t)ob;
			XF xfO0;
			xfO0.q = Q4{V3{st[10], st[11], st[12]}, st[13]};
			xfO0.p = V3{st[7], st[8], st[9]} - rot(xfO0.q, V3{st[14], st[15], st[16]});
			AABB a1, a2;
			compute_aabbs(S, of, xmult(xfM, xfO0), xmult(xfM, xfO), true, a1, a2);
			a1 = aabb_scaled(a1, inv);
			a2 = aabb_scaled(a2, inv);
			AABB a;
			a.lo = vmin(a1.lo, a2.lo);
			a.hi = vmax(a1.hi, a2.hi);
			move_aabb(fat, a, aabb_center(a2) - aabb_center(a1));
		}
		B.meshAABB[cur][2 * (size_t)c] = make_float4(fat.lo.x, fat.lo.y, fat.lo.z, 0.0f);
		B.meshAABB[cur][2 * (size_t)c + 1] = make_float4(fat.hi.x, fat.hi.y, fat.hi.z, 0.0f);
		// Triangles of every mesh contact, active or not: a wake-up later in
		// the pass may activate it.
		uint32_t count = 0;
		const MeshDesc md = S.meshes[S.fixHull[mf]];
		if (!mesh_query(S, md, fat, [&](uint32_t) { ++count; }))
			atomicOr(&B.counters[CTR_STATUS], B3G_ST_POLY_OVERFLOW);
		B.meshCount[c] = count;
	}
}

// Work items in query order, from the exclusive offsets.
__global__ void k_mesh_emit(DevScene S, Buffers B, uint32_t cur, uint32_t cap)
{
	uint32_t n = min(B.counters[CTR_PAIRS], cap);
	uint32_t total = B.counters[CTR_MESH_PAIRS];
	for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
	{
		uint32_t off = B.meshCount[c];
		uint32_t end = c + 1 < n ? B.meshCount[c + 1] : total;
		if (end == off)
			continue;
		uint32_t fa = B.pairA[cur][c], fb = B.pairB[cur][c];
		uint32_t mf = is_mesh(S, fa) ? fa : fb;
		float4 l = B.meshAABB[cur][2 * (size_t)c], h = B.meshAABB[cur][2 * (size_t)c + 1];
		AABB fat;
		fat.lo = V3{l.x, l.y, l.z};
		fat.hi = V3{h.x, h.y, h.z};
		const MeshDesc md = S.meshes[S.fixHull[mf]];
		uint32_t k = off;
		mesh_query(S, md, fat, [&](uint32_t t) {
			if (k < end && k < B.meshPairCap)
			{
				B.meshPairC[k] = c;
				B.meshPairT[k] = t;
			}
			++k;
		});
	}
}

__global__ void k_mesh_overflow(Buffers B)
{
	if (B.counters[CTR_MESH_PAIRS] > B.meshPairCap)
		atomicOr(&B.counters[CTR_STATUS], B3G_ST_POLY_OVERFLOW);
}

// ---------------------------------------------------------------------------
// b3ClusterSolver (cluster.cpp:202-585), one thread per mesh contact.

constexpr uint32_t MAX_CLUSTERS = 3;

// One observation in global scratch (three float4): a contact's work items
// [off, end) have at most 4 * (end - off) points, so its observations fit in
// the slots from 4 * off on.
struct Obs
{
	V3 normal; // b3Observation::point: the point's world normal
	float separation;
	V3 point;      // b3WorldManifoldPoint::point
	uint32_t item; // work item (the triangle's manifold)
	uint32_t index; // point in that manifold
	uint32_t cluster;
	uint32_t pad[2];
};
static_assert(sizeof(Obs) == 48, "three float4 per observation");
static_assert(sizeof(CV) == 16, "one float4 per polygon vertex");

__device__ __forceinline__ float dist2(V3 a, V3 b)
{
	V3 d = a - b;
	return (d.x * d.x + d.y * d.y) + d.z * d.z;
}

// b3ClusterSolver::FindCluster: the first nearest centroid.
__device__ __forceinline__ uint32_t find_cluster(const V3* cent, uint32_t nc, V3 p)
{
	uint32_t best = 0;
	float bestValue = B3G_MAX_SCALAR;
	for (uint32_t i = 0; i < nc; ++i)
	{
		float m = dist2(p, cent[i]);
		if (m < bestValue)
		{
			bestValue = m;
			best = i;
		}
	}
	return best;
}

// b3ClusterSolver::AddCluster: merge into the nearest centroid within 0.05.
__device__ __forceinline__ void add_cluster(V3* cent, uint32_t& nc, V3 c)
{
	if (nc == 0)
	{
		cent[nc++] = c;
		return;
	}
	uint32_t b = find_cluster(cent, nc, c);
	const float kTol = 0.05f;
	if (dist2(c, cent[b]) <= kTol * kTol)
	{
		cent[b] = cent[b] + c;
		normalize_inplace(cent[b]);
		return;
	}
	cent[nc++] = c;
}

__global__ void k_mesh_cluster(NPArgs a, Buffers B, DevManifold* extraCur, const DevManifold* extraPrev)
{
	uint32_t n = *a.listCount;
	uint32_t total = min(B.counters[CTR_MESH_PAIRS], B.meshPairCap);
	uint32_t nc = min(B.counters[CTR_PAIRS], (uint32_t)0xFFFFFFFFu);
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = a.list[t];
		uint32_t off = B.meshCount[c];
		uint32_t end = c + 1 < nc ? B.meshCount[c + 1] : B.counters[CTR_MESH_PAIRS];
		off = min(off, total);
		end = min(end, total);
		uint32_t fa = a.pairA[c], fb = a.pairB[c];
		XF xfA = body_xf(a.S, a.S.fixBody[fa]), xfB = body_xf(a.S, a.S.fixBody[fb]);
		DevManifold& m0 = a.man[c];
		DevManifold* out[3] = {&m0, extraCur + 2 * (size_t)c, extraCur + 2 * (size_t)c + 1};
		int32_t prev = a.prevIndex[c];
		uint32_t begun = prev < 0 ? 1u : 0u;
		bool sensor = ((a.S.fixFlags[fa] | a.S.fixFlags[fb]) & B3G_FIXTURE_SENSOR) != 0;
		if (sensor)
		{
			// b3MeshContact::TestOverlap: any triangle overlapping (the work
			// items carry the overlap in pointCount).
			uint32_t touching = 0;
			for (uint32_t i = off; i < end; ++i)
				touching |= B.meshPairMan[i].pointCount ? 1u : 0u;
			man_clear(m0);
			a.cstate[c] = touching | (begun << 16);
			a.cache[c] = make_uint4(B3G_NULL, B3G_NULL, B3G_NULL, B3G_NULL);
			continue;
		}
		// b3Shape::m_radius of both shapes (mesh: the fixture's radius)
		auto radius = [&](uint32_t f) -> float {
			float4 p0 = a.S.fixParams[3 * f], p1 = a.S.fixParams[3 * f + 1], p2 = a.S.fixParams[3 * f + 2];
			switch (a.S.fixType[f])
			{
			case B3G_SHAPE_SPHERE:
				return p0.w;
			case B3G_SHAPE_CAPSULE:
				return p1.z;
			case B3G_SHAPE_TRIANGLE:
				return p2.y;
			case B3G_SHAPE_MESH:
				return p0.w;
			default:
				return p0.x;
			}
		};
		const float rA = radius(fa), rB = radius(fb);
		// Observations: every point of every triangle manifold, in order.
		Obs* obs = reinterpret_cast<Obs*>(B.meshObs) + 4 * (size_t)off;
		CV* poly = reinterpret_cast<CV*>(B.meshPoly) + 4 * (size_t)off;
		uint32_t no = 0;
		for (uint32_t i = off; i < end; ++i)
		{
			const DevManifold& pm = B.meshPairMan[i];
			for (uint32_t j = 0; j < pm.pointCount && j < 4; ++j)
			{
				const DevPoint& p = pm.points[j];
				// b3WorldManifoldPoint::Initialize (collision.cpp:64-76)
				V3 nA = rot(xfA.q, V3{p.n[0], p.n[1], p.n[2]});
				V3 cA = xmul(xfA, V3{p.p1[0], p.p1[1], p.p1[2]});
				V3 cB = xmul(xfB, V3{p.p2[0], p.p2[1], p.p2[2]});
				V3 pA = cA + rA * nA;
				V3 pB = cB - rB * nA;
				Obs& o = obs[no++];
				o.point = 0.5f * (pA + pB);
				o.normal = nA;
				o.separation = (dot(cB - cA, nA) - rA) - rB;
				o.item = i;
				o.index = j;
				o.cluster = B3G_NULL;
			}
		}
		// InitializeClusters (cluster.cpp:207-333)
		V3 cent[MAX_CLUSTERS];
		uint32_t ncl = 0;
		if (no <= MAX_CLUSTERS)
		{
			for (uint32_t i = 0; i < no; ++i)
				add_cluster(cent, ncl, obs[i].normal);
		}
		else
		{
			// Observation 0 starts the first cluster; chosen1 the second.
			uint32_t chosen1 = B3G_NULL;
			add_cluster(cent, ncl, obs[0].normal);
			{
				V3 A = cent[0];
				uint32_t index = 0;
				float mx = -B3G_MAX_SCALAR;
				for (uint32_t i = 1; i < no; ++i)
				{
					float dd = dist2(A, obs[i].normal);
					if (dd > mx)
					{
						mx = dd;
						index = i;
					}
				}
				add_cluster(cent, ncl, obs[index].normal);
				chosen1 = index;
			}
			if (ncl == 1)
			{
				V3 A = cent[0];
				uint32_t index = 0;
				float mx = -B3G_MAX_SCALAR;
				for (uint32_t i = 1; i < no; ++i)
				{
					if (i == chosen1)
						continue;
					float dd = dist2(A, obs[i].normal);
					if (dd > mx)
					{
						mx = dd;
						index = i;
					}
				}
				add_cluster(cent, ncl, obs[index].normal);
			}
			else
			{
				V3 A = cent[0], Bc = cent[1];
				uint32_t index = 0;
				float mx = -B3G_MAX_SCALAR;
				for (uint32_t i = 1; i < no; ++i)
				{
					if (i == chosen1)
						continue;
					V3 C = obs[i].normal;
					V3 Q = closest_on_segment(C, A, Bc);
					float dd = dist2(C, Q);
					if (dd > mx)
					{
						mx = dd;
						index = i;
					}
				}
				add_cluster(cent, ncl, obs[index].normal);
			}
		}
		// k-means, 10 iterations (cluster.cpp:391-429)
		for (uint32_t iter = 0; iter < 10; ++iter)
		{
			for (uint32_t i = 0; i < no; ++i)
				obs[i].cluster = find_cluster(cent, ncl, obs[i].normal);
			for (uint32_t k = 0; k < ncl; ++k)
			{
				V3 sum = V3{0.0f, 0.0f, 0.0f};
				uint32_t cnt = 0;
				for (uint32_t i = 0; i < no; ++i)
					if (obs[i].cluster == k)
					{
						sum = sum + obs[i].normal;
						++cnt;
					}
				if (cnt > 0)
				{
					float s = 1.0f / (float)cnt; // b3Vec3::operator/= scales by the reciprocal
					cent[k] = s * sum;
				}
			}
		}
		// Empty clusters removed, the others renumbered in order (:431-455).
		uint32_t used = 0;
		for (uint32_t k = 0; k < ncl; ++k)
		{
			uint32_t cnt = 0;
			for (uint32_t i = 0; i < no; ++i)
				cnt += obs[i].cluster == k ? 1u : 0u;
			if (cnt > 0)
			{
				for (uint32_t i = 0; i < no; ++i)
					if (obs[i].cluster == k)
						obs[i].cluster = used;
				cent[used++] = cent[k];
			}
		}
		// One manifold per cluster (:458-585)
		uint32_t numOut = 0;
		for (uint32_t k = 0; k < used; ++k)
		{
			uint32_t np = 0;
			V3 normal = V3{0.0f, 0.0f, 0.0f};
			for (uint32_t j = 0; j < no; ++j)
			{
				if (obs[j].cluster != k)
					continue;
				poly[np].pos = obs[j].point;
				poly[np].clipIndex = j;
				++np;
				normal = normal + obs[j].normal;
			}
			if (np == 0)
				continue;
			normalize_inplace(normal);
			DevManifold& m = *out[numOut++];
			uint32_t minIndex = 0;
			float minSep = B3G_MAX_SCALAR;
			for (uint32_t j = 0; j < np; ++j)
			{
				float sep = obs[poly[j].clipIndex].separation;
				if (sep < minSep)
				{
					minIndex = j;
					minSep = sep;
				}
				poly[j].pos = poly[j].pos + sep * normal;
			}
			CV quad[4];
			uint32_t nq = reduce_polygon(quad, poly, np, normal, minIndex);
			// b3Manifold::Initialize, then the chosen points copied whole
			m.pointCount = nq;
			m.tangentImpulse[0] = m.tangentImpulse[1] = 0.0f;
			m.motorImpulse = m.motorSpeed = m.tangentSpeed1 = m.tangentSpeed2 = 0.0f;
			for (uint32_t j = 0; j < nq; ++j)
			{
				const Obs& o = obs[quad[j].clipIndex];
				m.points[j] = B.meshPairMan[o.item].points[o.index];
			}
		}
		for (uint32_t k = numOut; k < 3; ++k)
			man_clear(*out[k]);
		// b3Contact::Update's warm start: every new manifold against every
		// old one, in order (contact.cpp:424-446).
		uint32_t oldCount = prev >= 0 ? ((a.prevState[prev] >> 8) & 0xFFu) : 0u;
		if (a.warmStarting && oldCount > 0)
		{
			for (uint32_t i = 0; i < numOut; ++i)
			{
				DevManifold& m2 = *out[i];
				for (uint32_t j = 0; j < oldCount && j < 3; ++j)
				{
					const DevManifold& m1 = j == 0 ? a.prevMan[prev] : extraPrev[2 * (size_t)prev + j - 1];
					bool host = j == 0 && a.impN;
					m2.tangentImpulse[0] = host ? a.impT[2 * prev] : m1.tangentImpulse[0];
					m2.tangentImpulse[1] = host ? a.impT[2 * prev + 1] : m1.tangentImpulse[1];
					m2.motorImpulse = host ? a.impM[prev] : m1.motorImpulse;
					for (uint32_t pi = 0; pi < m2.pointCount; ++pi)
					{
						DevPoint& p1 = m2.points[pi];
						for (uint32_t pj = 0; pj < m1.pointCount; ++pj)
						{
							const DevPoint& p2 = m1.points[pj];
							if (p2.triangleKey == p1.triangleKey && p2.key[0] == p1.key[0] && p2.key[1] == p1.key[1] &&
								p2.key[2] == p1.key[2] && p2.key[3] == p1.key[3])
							{
								p1.normalImpulse = host ? a.impN[4 * prev + pj] : p2.normalImpulse;
								p1.persisting = 1;
								break;
							}
						}
					}
				}
			}
		}
		uint32_t touching = numOut > 0 ? 1u : 0u;
		a.cstate[c] = touching | (numOut << 8) | (begun << 16);
		a.cache[c] = make_uint4(B3G_NULL, B3G_NULL, B3G_NULL, B3G_NULL);
	}
}

} // namespace

void launch_mesh_fat(b3g_ctx* c, cudaStream_t s)
{
	if (c->nMeshFix)
		k_mesh_fat<<<c->nMeshFix, 256, 0, s>>>(c->scene, c->buf, c->dMeshFix);
}

void launch_mesh_prepare(b3g_ctx* c, cudaStream_t s)
{
	if (!c->nMeshFix)
		return;
	Buffers& B = c->buf;
	const uint32_t cap = c->cfg.max_contacts, cur = c->cur;
	k_mesh_sync<<<persistent_blocks(4), 128, 0, s>>>(c->scene, B, cur, cap);
	scan_exclusive_device(B.meshCount, B.counters + CTR_PAIRS, cap, B.scanAux, B.counters + CTR_MESH_PAIRS,
		B.counters + CTR_STATUS, s);
	k_mesh_overflow<<<1, 1, 0, s>>>(B);
	k_mesh_emit<<<persistent_blocks(4), 128, 0, s>>>(c->scene, B, cur, cap);
}

void launch_mesh_collide(b3g_ctx* c, const uint32_t* list, const uint32_t* count, cudaStream_t s)
{
	if (!c->nMeshFix)
		return;
	Buffers& B = c->buf;
	NPArgs a = make_np_args(c);
	launch_mesh_items_convex(a, B, s);
	launch_mesh_items_hull(a, B, c->maxUniqueEdges, c->tune, s);
	a.list = list;
	a.listCount = count;
	const uint32_t cur = c->cur;
	k_mesh_cluster<<<persistent_blocks(2), 64, 0, s>>>(a, B, B.extraMan[cur], B.extraMan[cur ^ 1u]);
}

uint32_t mesh_launches(const b3g_ctx* c)
{
	if (!c->nMeshFix)
		return 0;
	// sync, scan, overflow, emit; two evaluation kernels, cluster
	return 1 + 1 + 1 + 1 + 2 + 1;
}

// Warp-per-pair hull-hull narrowphase: b3CollideHulls with the feature cache
// (collide_hulls.cpp:355-534) and without it (collide_hulls.cpp:189-264).
//
// The 32 lanes of a warp share one contact. The separating-axis queries are
// spread over the lanes: face queries (sat.cpp:33-58) put faces on lanes and
// loop over the other hull's vertices for the support point; the edge query
// (sat.cpp:111-174) flattens the (edge1, edge2) double loop onto lanes after
// the per-edge data (both endpoints, edge vector and length, the two adjacent
// face normals of the Gauss map) is precomputed into shared memory. Every
// argmax is reduced with warp shuffles on (value, flattened index), keeping
// the larger value and, on equal values, the lower index - which is exactly
// the first maximum the reference's sequential "if (s > max)" loops select.
// The serial remainder (incident face clipping, polygon reduction, the cache
// decision tree) runs on lane 0.

#include "collide_common.cuh"

namespace {


struct EdgeRec
{
	float4 P; // xyz endpoint, w = |E|
	float4 E; // xyz edge vector
	float4 U; // xyz normal of the edge's face
	float4 V; // xyz normal of the twin's face
};

__device__ __forceinline__ V3 f3(float4 a) { return V3{a.x, a.y, a.z}; }

// First-maximum reduction across the warp on (value, index).
__device__ __forceinline__ void warp_argmax(float& v, uint32_t& idx)
{
	for (int o = 16; o > 0; o >>= 1)
	{
		float ov = __shfl_xor_sync(0xffffffffu, v, o);
		uint32_t oi = __shfl_xor_sync(0xffffffffu, idx, o);
		if (ov > v || (ov == v && oi < idx))
		{
			v = ov;
			idx = oi;
		}
	}
}

// b3QueryFaceSeparation(hull, hull) (sat.cpp:33-58).
__device__ void warp_query_faces(const XF& xf1, const HullRef& h1, const XF& xf2, const HullRef& h2,
	uint32_t lane, uint32_t& index, float& sep)
{
	XF xf = xmult(xf2, xf1);
	float best = -B3G_MAX_SCALAR;
	uint32_t bi = 0xFFFFFFFFu;
	for (uint32_t i = lane; i < h1.fCnt; i += 32)
	{
		PL plane = pmul(xf, hp(h1, i));
		V3 d = -plane.n;
		uint32_t si = 0;
		float sp = dot(d, hv(h2, 0));
		for (uint32_t k = 1; k < h2.vCnt; ++k)
		{
			float proj = dot(d, hv(h2, k));
			if (proj > sp)
			{
				si = k;
				sp = proj;
			}
		}
		float s = pdist(hv(h2, si), plane);
		if (s > best)
		{
			best = s;
			bi = i;
		}
	}
	warp_argmax(best, bi);
	index = bi == 0xFFFFFFFFu ? 0u : bi;
	sep = best;
}

// b3IsMinkowskiFace (sat.cpp:60-71).
__device__ __forceinline__ bool is_minkowski_face(V3 A, V3 B, V3 BxA, V3 C, V3 D, V3 DxC)
{
	float ADC = dot(A, DxC);
	float BDC = dot(B, DxC);
	float CBA = dot(C, BxA);
	float DBA = dot(D, BxA);
	return CBA * DBA < 0.0f && ADC * BDC < 0.0f && CBA * BDC > 0.0f;
}

// b3Project(P1, Q1, E1, P2, E2, C1) (sat.cpp:73-109); L1 = |E1|, L2 = |E2|.
__device__ __forceinline__ float project_edges(V3 P1, V3 E1, float L1, V3 P2, V3 E2, float L2, V3 C1)
{
	if (L1 < B3G_LINEAR_SLOP)
		return -B3G_MAX_SCALAR;
	if (L2 < B3G_LINEAR_SLOP)
		return -B3G_MAX_SCALAR;
	const float kTol = 0.005f;
	V3 E1_x_E2 = cross(E1, E2);
	float L = len(E1_x_E2);
	if (L < (kTol * L1) * L2)
		return -B3G_MAX_SCALAR;
	V3 N = (1.0f / L) * E1_x_E2;
	if (dot(N, P1 - C1) < 0.0f)
		N = -N;
	return dot(N, P2 - P1);
}

__device__ __forceinline__ void edge_rec_1(EdgeRec& r, const XF& xf, const HullRef& h1, uint32_t i)
{
	uint4 e1 = h1.e[i], t1 = h1.e[i + 1];
	V3 P1 = xmul(xf, hv(h1, e1.x));
	V3 Q1 = xmul(xf, hv(h1, t1.x));
	V3 E1 = Q1 - P1;
	V3 U1 = rot(xf.q, hp(h1, e1.y).n);
	V3 V1 = rot(xf.q, hp(h1, t1.y).n);
	r.P = make_float4(P1.x, P1.y, P1.z, len(E1));
	r.E = make_float4(E1.x, E1.y, E1.z, 0.0f);
	r.U = make_float4(U1.x, U1.y, U1.z, 0.0f);
	r.V = make_float4(V1.x, V1.y, V1.z, 0.0f);
}

__device__ __forceinline__ void edge_rec_2(EdgeRec& r, const HullRef& h2, uint32_t j)
{
	uint4 e2 = h2.e[j], t2 = h2.e[j + 1];
	V3 P2 = hv(h2, e2.x);
	V3 Q2 = hv(h2, t2.x);
	V3 E2 = Q2 - P2;
	V3 U2 = hp(h2, e2.y).n;
	V3 V2 = hp(h2, t2.y).n;
	r.P = make_float4(P2.x, P2.y, P2.z, len(E2));
	r.E = make_float4(E2.x, E2.y, E2.z, 0.0f);
	r.U = make_float4(U2.x, U2.y, U2.z, 0.0f);
	r.V = make_float4(V2.x, V2.y, V2.z, 0.0f);
}

__device__ __forceinline__ float edge_pair_sep(const EdgeRec& a, const EdgeRec& b, V3 C1)
{
	V3 U1 = f3(a.U), V1 = f3(a.V), E1 = f3(a.E);
	V3 U2 = f3(b.U), V2 = f3(b.V), E2 = f3(b.E);
	if (!is_minkowski_face(U1, V1, -E1, -U2, -V2, -E2))
		return -INFINITY; // not a Minkowski face: never a candidate
	return project_edges(f3(a.P), E1, a.P.w, f3(b.P), E2, b.P.w, C1);
}

// Hulls with fewer unique edges than this on both sides share the pairs out
// flat over the lanes (both edge sets staged); otherwise the larger set sits
// on the lanes and only the smaller one is staged.
constexpr uint32_t SAT_FLAT_EDGES = 48;

// Edge records of shared memory one warp needs (maxUE: the most unique
// edges of any hull): both sets of a flat query (at most 2 maxUE, and at
// most 2 (SAT_FLAT_EDGES - 1)), or the smaller set of a broadcast one (at
// most maxUE).
__host__ __device__ __forceinline__ uint32_t sat_warp_recs(uint32_t maxUE)
{
	if (maxUE < SAT_FLAT_EDGES)
		return 2 * maxUE;
	return maxUE > 2 * (SAT_FLAT_EDGES - 1) ? maxUE : 2 * (SAT_FLAT_EDGES - 1);
}

// b3QueryEdgeSeparation(hull, hull) (sat.cpp:111-174). recs holds
// sat_warp_recs(maxUE) records.
__device__ void warp_query_edges(const XF& xf1, const HullRef& h1, const XF& xf2, const HullRef& h2,
	uint32_t lane, EdgeRec* recs, uint32_t maxUE, uint32_t& index1, uint32_t& index2, float& sep)
{
	XF xf = xmult(xf2, xf1);
	V3 C1 = xmul(xf, h1.centroid);
	uint32_t n1 = h1.eCnt / 2, n2 = h2.eCnt / 2;
	const bool flat = n1 < SAT_FLAT_EDGES && n2 < SAT_FLAT_EDGES;
	EdgeRec* r1 = recs;
	EdgeRec* r2 = recs + (flat ? n1 : 0);
	bool staged = n1 <= maxUE && n2 <= maxUE;
	if (staged && flat)
	{
		for (uint32_t i = lane; i < n1; i += 32)
			edge_rec_1(r1[i], xf, h1, 2 * i);
		for (uint32_t j = lane; j < n2; j += 32)
			edge_rec_2(r2[j], h2, 2 * j);
		__syncwarp();
	}
	float best = -B3G_MAX_SCALAR;
	uint32_t bk = 0xFFFFFFFFu;
	uint32_t total = n1 * n2;
	// Each lane keeps the first maximum in k = i n2 + j among the pairs it
	// tests (larger value, or equal value and smaller k; nothing at or below
	// the start value, as the serial loop's strict test), and warp_argmax
	// picks the first maximum over the lanes: the serial loop's answer,
	// whatever pairs a lane is given.
	auto keep = [&](float s, uint32_t k) {
		if (s > best || (s == best && bk != 0xFFFFFFFFu && k < bk))
		{
			best = s;
			bk = k;
		}
	};
	if (staged && !flat)
	{
		// Larger hull's edges on the lanes, held in registers; the other
		// hull's edges staged and read by all lanes at once (shared-memory
		// broadcast).
		const bool rows1 = n1 >= n2;
		const uint32_t nl = rows1 ? n1 : n2, nb = rows1 ? n2 : n1;
		EdgeRec* rb = recs;
		for (uint32_t b = lane; b < nb; b += 32)
		{
			if (rows1)
				edge_rec_2(rb[b], h2, 2 * b);
			else
				edge_rec_1(rb[b], xf, h1, 2 * b);
		}
		__syncwarp();
		for (uint32_t base = 0; base < nl; base += 32)
		{
			const uint32_t l = base + lane;
			const bool valid = l < nl;
			EdgeRec mine;
			const uint32_t le = 2 * (valid ? l : 0);
			if (rows1)
				edge_rec_1(mine, xf, h1, le);
			else
				edge_rec_2(mine, h2, le);
			for (uint32_t b = 0; b < nb; ++b)
			{
				const EdgeRec other = rb[b];
				if (!valid)
					continue;
				const uint32_t i = rows1 ? l : b, j = rows1 ? b : l;
				keep(rows1 ? edge_pair_sep(mine, other, C1) : edge_pair_sep(other, mine, C1), i * n2 + j);
			}
		}
	}
	else
	{
		// (i, j) of k = i n2 + j, stepped without a division per pair.
		uint32_t i = n2 ? lane / n2 : 0u, j = lane - i * n2;
		for (uint32_t k = lane; k < total; k += 32, j += 32)
		{
			while (j >= n2)
			{
				j -= n2;
				++i;
			}
			float s;
			if (staged)
			{
				s = edge_pair_sep(r1[i], r2[j], C1);
			}
			else
			{
				EdgeRec a, b;
				edge_rec_1(a, xf, h1, 2 * i);
				edge_rec_2(b, h2, 2 * j);
				s = edge_pair_sep(a, b, C1);
			}
			keep(s, k);
		}
	}
	warp_argmax(best, bk);
	if (bk == 0xFFFFFFFFu)
	{
		index1 = 0;
		index2 = 0;
	}
	else
	{
		index1 = 2 * (bk / n2);
		index2 = 2 * (bk % n2);
	}
	sep = best;
	__syncwarp();
}

// b3BuildEdgeContact (collide_hulls.cpp:30-73).
__device__ void build_edge_contact(DevManifold& m, const XF& xf1, uint32_t index1, const HullRef& h1,
	const XF& xf2, uint32_t index2, const HullRef& h2)
{
	uint4 e1 = h1.e[index1], t1 = h1.e[index1 + 1];
	V3 C1 = xmul(xf1, h1.centroid);
	V3 P1 = xmul(xf1, hv(h1, e1.x));
	V3 Q1 = xmul(xf1, hv(h1, t1.x));
	V3 E1 = Q1 - P1;
	uint4 e2 = h2.e[index2], t2 = h2.e[index2 + 1];
	V3 P2 = xmul(xf2, hv(h2, e2.x));
	V3 Q2 = xmul(xf2, hv(h2, t2.x));
	V3 E2 = Q2 - P2;
	V3 N = cross(E1, E2);
	normalize_inplace(N);
	if (dot(N, P1 - C1) < 0.0f)
		N = -N;
	V3 point1, point2;
	closest_on_segments(point1, point2, P1, Q1, P2, Q2);
	m.pointCount = 1;
	set_point(m.points[0], rotc(xf1.q, N), xmult(xf1, point1), xmult(xf2, point2));
	set_id(m.points[0], mkpair(index1, index1 + 1, index2, index2 + 1));
	m.points[0].edgeContact = 1;
}

// b3BuildFaceContact (collide_hulls.cpp:75-187). Runs on one lane.
__device__ void build_face_contact(DevManifold& m, const XF& xf1, uint32_t index1, const HullRef& h1, float r1,
	const XF& xf2, const HullRef& h2, float r2, bool flipNormal, uint32_t* status)
{
	float totalRadius = r1 + r2;
	PL localPlane1 = hp(h1, index1);
	PL plane1 = pmul(xf1, localPlane1);
	V3 normal1 = rotc(xf2.q, plane1.n);
	uint32_t index2 = hull_support_face(h2, -normal1);
	Poly pa, pb;
	if (!build_polygon(pa, xf2, index2, h2))
	{
		atomicOr(status, B3G_ST_POLY_OVERFLOW);
		return;
	}
	bool ok;
	Poly* clip = clip_polygon_to_face_side_planes(pa, pb, xf1, totalRadius, index1, h1, ok);
	if (!ok)
	{
		atomicOr(status, B3G_ST_POLY_OVERFLOW);
		return;
	}
	if (clip->n == 0)
		return;
	CV poly1[B3G_MAX_POLY];
	uint32_t n1 = 0;
	uint32_t minIndex = 0;
	float minSep = B3G_MAX_SCALAR;
	for (uint32_t i = 0; i < clip->n; ++i)
	{
		V3 p = clip->v[i].pos;
		float s = pdist(p, plane1);
		if (s <= totalRadius)
		{
			if (s < minSep)
			{
				minIndex = n1;
				minSep = s;
			}
			poly1[n1].pos = pclosest(p, plane1);
			poly1[n1].clipIndex = i;
			++n1;
		}
	}
	if (n1 == 0)
		return;
	V3 normal = plane1.n;
	V3 oriented = flipNormal ? -normal : normal;
	CV red[4];
	uint32_t cnt = reduce_polygon(red, poly1, n1, oriented, minIndex);
	for (uint32_t i = 0; i < cnt; ++i)
	{
		const ClipV& v2 = clip->v[red[i].clipIndex];
		V3 v1 = pclosest(v2.pos, plane1);
		DevPoint& mp = m.points[i];
		if (flipNormal)
		{
			set_point(mp, rotc(xf2.q, oriented), xmult(xf2, v2.pos), xmult(xf1, v1));
			set_id(mp, mkpair(v2.pair.inEdge2, v2.pair.outEdge2, v2.pair.inEdge1, v2.pair.outEdge1));
		}
		else
		{
			set_point(mp, rotc(xf1.q, oriented), xmult(xf1, v1), xmult(xf2, v2.pos));
			set_id(mp, v2.pair);
		}
		mp.edgeContact = 0;
	}
	m.pointCount = cnt;
}

// Shared-memory buffers of one warp for warp_build_face_contact: two clip
// polygons (ping-pong) and the kept points of the reference face.
struct WarpClip
{
	ClipV a[B3G_MAX_POLY];
	ClipV b[B3G_MAX_POLY];
	CV kept[B3G_MAX_POLY];
};

// Shared memory of one warp in the hull kernels: the edge records of the edge
// query, then (the query done) the clip buffers of the face contact.
__host__ __device__ __forceinline__ size_t sat_warp_bytes(uint32_t maxUE)
{
	size_t recs = (size_t)sat_warp_recs(maxUE) * sizeof(EdgeRec);
	return recs > sizeof(WarpClip) ? recs : sizeof(WarpClip);
}

// Exclusive prefix sum of v over the warp; *total receives the sum.
__device__ __forceinline__ uint32_t warp_excl_scan(uint32_t v, uint32_t lane, uint32_t& total)
{
	uint32_t x = v;
	for (int o = 1; o < 32; o <<= 1)
	{
		uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
		if (lane >= (uint32_t)o)
			x += y;
	}
	total = __shfl_sync(0xffffffffu, x, 31);
	return x - v;
}

// b3ClipPolygonToPlane (clip.cpp:101-150) on the warp: vertex i (lanes take i
// and i + 32) emits what the sequential loop emits at step i — v2, the
// intersection, or both — at the place a prefix sum of the emit counts gives,
// so out holds the sequential loop's polygon, same values, same order. d1 of
// step i is the distance of vertex i - 1 (n - 1 for step 0), the value the
// loop carries over. Returns the new vertex count, or B3G_MAX_POLY + 1 when
// the polygon would outgrow the buffer (the loop fails there too).
__device__ uint32_t warp_clip_polygon_to_plane(ClipV* out, const ClipV* in, uint32_t n, PL plane, uint32_t edge,
	uint32_t lane)
{
	uint32_t base = 0;
	for (uint32_t i0 = 0; i0 < n; i0 += 32)
	{
		const uint32_t i = i0 + lane;
		uint32_t cnt = 0;
		ClipV v1, v2;
		float d1 = 0.0f, d2 = 0.0f;
		if (i < n)
		{
			v2 = in[i];
			v1 = in[i == 0 ? n - 1 : i - 1];
			d2 = pdist(v2.pos, plane);
			d1 = pdist(v1.pos, plane);
			if (d1 <= 0.0f && d2 <= 0.0f)
				cnt = 1;
			else if (d1 <= 0.0f && d2 > 0.0f)
				cnt = 1;
			else if (d1 > 0.0f && d2 <= 0.0f)
				cnt = 2;
		}
		uint32_t total;
		const uint32_t o = base + warp_excl_scan(cnt, lane, total);
		base += total;
		// Writes past the buffer are skipped; the count reports the overflow.
		if (cnt != 0 && o + cnt <= B3G_MAX_POLY)
		{
			if (d1 <= 0.0f && d2 <= 0.0f)
				out[o] = v2;
			else if (d1 <= 0.0f && d2 > 0.0f)
			{
				float fraction = d1 / (d1 - d2);
				out[o].pos = v1.pos + fraction * (v2.pos - v1.pos);
				out[o].pair = mkpair(edge, B3G_NULL_EDGE, v1.pair.outEdge2, B3G_NULL_EDGE);
			}
			else
			{
				float fraction = d1 / (d1 - d2);
				out[o].pos = v1.pos + fraction * (v2.pos - v1.pos);
				out[o].pair = mkpair(B3G_NULL_EDGE, edge, B3G_NULL_EDGE, v2.pair.inEdge2);
				out[o + 1] = v2;
			}
		}
	}
	__syncwarp();
	return base > B3G_MAX_POLY ? B3G_MAX_POLY + 1 : base;
}

// b3BuildFaceContact (collide_hulls.cpp:75-187) on the warp, with W in
// shared memory: the incident polygon (lane 0 walks the face loop), the
// clipping against the reference face's side planes (warp_clip_polygon_to_
// plane), the kept points and the deepest of them (first minimum: smaller
// separation, on ties the earlier point), then the reduction to four points
// and the manifold on lane 0. Same operations and order as build_face_contact;
// returns the point count on every lane.
__device__ __noinline__ uint32_t warp_build_face_contact(DevManifold& m, const XF& xf1, uint32_t index1, const HullRef& h1,
	float r1, const XF& xf2, const HullRef& h2, float r2, bool flipNormal, uint32_t* status, uint32_t lane,
	WarpClip& W)
{
	float totalRadius = r1 + r2;
	PL localPlane1 = hp(h1, index1);
	PL plane1 = pmul(xf1, localPlane1);
	V3 normal1 = rotc(xf2.q, plane1.n);
	uint32_t index2 = hull_support_face(h2, -normal1);
	uint32_t n = 0;
	if (lane == 0)
	{
		uint32_t begin = h2.f[index2];
		uint32_t edge = begin;
		do
		{
			if (n >= B3G_MAX_POLY)
			{
				n = B3G_MAX_POLY + 1;
				break;
			}
			ClipV& cv = W.a[n++];
			cv.pos = xmul(xf2, hv(h2, he_origin(h2, edge)));
			cv.pair = mkpair(B3G_NULL_EDGE, B3G_NULL_EDGE, he_prev(h2, edge), edge);
			edge = he_next(h2, edge);
		} while (edge != begin);
	}
	n = __shfl_sync(0xffffffffu, n, 0);
	__syncwarp();
	bool ok = n <= B3G_MAX_POLY;
	ClipV* in = W.a;
	ClipV* out = W.b;
	if (ok)
	{
		uint32_t begin = h1.f[index1];
		uint32_t edge = begin;
		uint32_t guard = 0;
		do
		{
			if (++guard > h1.eCnt)
			{
				ok = false;
				break;
			}
			PL plane = hull_edge_side_plane(h1, edge);
			plane.d += totalRadius;
			PL cp = pmul(xf1, plane);
			uint32_t nn = warp_clip_polygon_to_plane(out, in, n, cp, edge, lane);
			if (nn > B3G_MAX_POLY)
			{
				ok = false;
				break;
			}
			ClipV* t = in;
			in = out;
			out = t;
			n = nn;
			if (n == 0)
				break;
			edge = he_next(h1, edge);
		} while (edge != begin);
	}
	if (!ok)
	{
		if (lane == 0)
			atomicOr(status, B3G_ST_POLY_OVERFLOW);
		return 0;
	}
	if (n == 0)
		return 0;
	// Kept points (separation within the radius), projected on the reference
	// plane, in order; the first of the smallest separation.
	uint32_t base = 0;
	float bestS = B3G_MAX_SCALAR;
	uint32_t bestK = 0xFFFFFFFFu;
	for (uint32_t i0 = 0; i0 < n; i0 += 32)
	{
		const uint32_t i = i0 + lane;
		bool keep = false;
		V3 p{0.0f, 0.0f, 0.0f};
		float sep = 0.0f;
		if (i < n)
		{
			p = in[i].pos;
			sep = pdist(p, plane1);
			keep = sep <= totalRadius;
		}
		uint32_t total;
		const uint32_t k = base + warp_excl_scan(keep ? 1u : 0u, lane, total);
		if (keep)
		{
			W.kept[k].pos = pclosest(p, plane1);
			W.kept[k].clipIndex = i;
			if (sep < bestS || (sep == bestS && k < bestK))
			{
				bestS = sep;
				bestK = k;
			}
		}
		base += total;
	}
	const uint32_t n1 = base;
	if (n1 == 0)
		return 0;
	for (int o = 16; o > 0; o >>= 1)
	{
		float os = __shfl_xor_sync(0xffffffffu, bestS, o);
		uint32_t ok2 = __shfl_xor_sync(0xffffffffu, bestK, o);
		if (os < bestS || (os == bestS && ok2 < bestK))
		{
			bestS = os;
			bestK = ok2;
		}
	}
	__syncwarp();
	uint32_t cnt = 0;
	if (lane == 0)
	{
		V3 normal = plane1.n;
		V3 oriented = flipNormal ? -normal : normal;
		CV red[4];
		cnt = reduce_polygon(red, W.kept, n1, oriented, bestK);
		for (uint32_t i = 0; i < cnt; ++i)
		{
			const ClipV& v2 = in[red[i].clipIndex];
			V3 v1 = pclosest(v2.pos, plane1);
			DevPoint& mp = m.points[i];
			if (flipNormal)
			{
				set_point(mp, rotc(xf2.q, oriented), xmult(xf2, v2.pos), xmult(xf1, v1));
				set_id(mp, mkpair(v2.pair.inEdge2, v2.pair.outEdge2, v2.pair.inEdge1, v2.pair.outEdge1));
			}
			else
			{
				set_point(mp, rotc(xf1.q, oriented), xmult(xf1, v1), xmult(xf2, v2.pos));
				set_id(mp, v2.pair);
			}
			mp.edgeContact = 0;
		}
		m.pointCount = cnt;
	}
	cnt = __shfl_sync(0xffffffffu, cnt, 0);
	__syncwarp();
	return cnt;
}

// b3RebuildEdgeContact (collide_hulls.cpp:266-321).
__device__ void rebuild_edge_contact(DevManifold& m, const XF& xf1, uint32_t index1, const HullRef& h1,
	const XF& xf2, uint32_t index2, const HullRef& h2)
{
	uint4 e1 = h1.e[index1], t1 = h1.e[index1 + 1];
	V3 C1 = xmul(xf1, h1.centroid);
	V3 P1 = xmul(xf1, hv(h1, e1.x));
	V3 Q1 = xmul(xf1, hv(h1, t1.x));
	V3 E1 = Q1 - P1;
	uint4 e2 = h2.e[index2], t2 = h2.e[index2 + 1];
	V3 P2 = xmul(xf2, hv(h2, e2.x));
	V3 Q2 = xmul(xf2, hv(h2, t2.x));
	V3 E2 = Q2 - P2;
	V3 point1, point2;
	closest_on_segments(point1, point2, P1, Q1, P2, Q2);
	float w1[3], w2[3];
	barycentric_segment(w1, P2, Q2, point1);
	barycentric_segment(w2, P1, Q1, point2);
	if (w1[1] > 0.0f && w1[1] <= w1[2] && w2[1] > 0.0f && w2[1] <= w2[2])
	{
		V3 N = cross(E1, E2);
		normalize_inplace(N);
		if (dot(N, P1 - C1) < 0.0f)
			N = -N;
		m.pointCount = 1;
		set_point(m.points[0], rotc(xf1.q, N), xmult(xf1, point1), xmult(xf2, point2));
		set_id(m.points[0], mkpair(index1, index1 + 1, index2, index2 + 1));
		m.points[0].edgeContact = 1;
	}
}

// b3RebuildFaceContact (collide_hulls.cpp:323-353).
__device__ void rebuild_face_contact(DevManifold& m, const XF& xf1, uint32_t index1, const HullRef& h1, float r1,
	const XF& xf2, const HullRef& h2, float r2, bool flipNormal, const XF& xf01, const XF& xf02,
	uint32_t* status)
{
	Q4 q01 = xf01.q, q1 = xf1.q;
	Q4 q02 = xf02.q, q2 = xf2.q;
	Q4 dq0 = qmul(conj(q01), q02);
	Q4 dq = qmul(conj(q1), q2);
	Q4 q = qmul(conj(dq0), dq);
	const float kCosTol = 0.995f;
	if (fabsr(q.s) > kCosTol)
		build_face_contact(m, xf1, index1, h1, r1, xf2, h2, r2, flipNormal, status);
}

enum
{
	CT_EMPTY = 0,
	CT_SEPARATION = 1,
	CT_OVERLAP = 2
};
enum
{
	FT_EDGES = 0,
	FT_FACE1 = 1,
	FT_FACE2 = 2
};

// b3FeatureCache::ReadEdges (sat.cpp:226-281).
__device__ uint32_t read_edges(const XF& xf1, const HullRef& h1, const XF& xf2, const HullRef& h2, uint32_t i,
	uint32_t j, float totalRadius)
{
	XF xf = xmult(xf2, xf1);
	V3 C1 = xmul(xf, h1.centroid);
	EdgeRec a, b;
	edge_rec_1(a, xf, h1, i);
	edge_rec_2(b, h2, j);
	V3 U1 = f3(a.U), V1 = f3(a.V), E1 = f3(a.E);
	V3 U2 = f3(b.U), V2 = f3(b.V), E2 = f3(b.E);
	if (is_minkowski_face(U1, V1, -E1, -U2, -V2, -E2))
	{
		float s = project_edges(f3(a.P), E1, a.P.w, f3(b.P), E2, b.P.w, C1);
		return s > totalRadius ? CT_SEPARATION : CT_OVERLAP;
	}
	return CT_EMPTY;
}

struct HullCtx
{
	XF xf1, xf2, xf01, xf02;
	HullRef h1, h2;
	float r1, r2;
	EdgeRec* recs;
	uint32_t maxUE;
	uint32_t* status;
	WarpClip* clip; // the warp's shared clip buffers
};

// Lane 0 builds, the warp learns the point count.
// Face contact on the warp (H.clip: the warp's shared clip buffers); every
// lane learns the point count.
__device__ uint32_t face_contact_all(DevManifold& m, const HullCtx& H, bool flip, uint32_t index, uint32_t lane)
{
	if (flip)
		return warp_build_face_contact(m, H.xf2, index, H.h2, H.r2, H.xf1, H.h1, H.r1, true, H.status, lane, *H.clip);
	return warp_build_face_contact(m, H.xf1, index, H.h1, H.r1, H.xf2, H.h2, H.r2, false, H.status, lane, *H.clip);
}

// b3CollideHulls without cache (collide_hulls.cpp:189-264).
__device__ void collide_hulls_nocache(DevManifold& m, const HullCtx& H, uint32_t lane)
{
	float totalRadius = H.r1 + H.r2;
	uint32_t fi1, fi2, ei1, ei2;
	float fs1, fs2, es;
	warp_query_faces(H.xf1, H.h1, H.xf2, H.h2, lane, fi1, fs1);
	if (fs1 > totalRadius)
		return;
	warp_query_faces(H.xf2, H.h2, H.xf1, H.h1, lane, fi2, fs2);
	if (fs2 > totalRadius)
		return;
	warp_query_edges(H.xf1, H.h1, H.xf2, H.h2, lane, H.recs, H.maxUE, ei1, ei2, es);
	if (es > totalRadius)
		return;
	const float kRelEdgeTol = 0.90f;
	const float kRelFaceTol = 0.98f;
	const float kAbsTol = 0.5f * B3G_LINEAR_SLOP;
	uint32_t pc;
	if (es > kRelEdgeTol * fmaxr(fs1, fs2) + kAbsTol)
	{
		if (lane == 0)
			build_edge_contact(m, H.xf1, ei1, H.h1, H.xf2, ei2, H.h2);
		pc = 1;
	}
	else if (fs2 > kRelFaceTol * fs1 + kAbsTol)
		pc = face_contact_all(m, H, true, fi2, lane);
	else
		pc = face_contact_all(m, H, false, fi1, lane);
	if (pc > 0)
		return;
	if (es > fmaxr(fs1, fs2))
	{
		if (lane == 0)
			build_edge_contact(m, H.xf1, ei1, H.h1, H.xf2, ei2, H.h2);
	}
	else if (fs2 > fs1)
		face_contact_all(m, H, true, fi2, lane);
	else
		face_contact_all(m, H, false, fi1, lane);
}

// Thread-level b3FeatureCache::ReadFace (sat.cpp:209-224).
__device__ uint32_t read_face_thread(const XF& xf1, const HullRef& h1, const XF& xf2, const HullRef& h2,
	uint32_t index1, float totalRadius)
{
	XF xf = xmult(xf2, xf1);
	PL plane = pmul(xf, hp(h1, index1));
	uint32_t si = hull_support_vertex(h2, -plane.n);
	float s = pdist(hv(h2, si), plane);
	return s > totalRadius ? CT_SEPARATION : CT_OVERLAP;
}

// The cache half of b3CollideHullsCache (collide_hulls.cpp:367-415), one
// thread per contact: b3FeatureCache::ReadState (sat.cpp:178-207), then the
// separation hit, or the overlap hit that rebuilds the cached edge or face
// contact. Returns true when the contact is finished; otherwise the cache is
// flushed (cacheType = empty, the feature fields as ReadState left them) and
// the contact needs the SAT. The face rebuild clips on this thread: the
// polygons are small (3 or 4 vertices on these hulls), and a warp per rebuild
// measured slower than the threads that do it here.
__device__ bool probe_cache(DevManifold& m, const HullCtx& H, uint4& cache)
{
	float totalRadius = H.r1 + H.r2;
	uint32_t state0 = cache.x;
	if (cache.x == CT_EMPTY)
	{
		cache.x = CT_SEPARATION;
		cache.y = FT_FACE1;
		cache.z = 0;
		cache.w = 0;
	}
	// A face of either hull is read by one call with the hulls in the face's
	// order, so the lanes of a warp with face caches of hull 1 and of hull 2
	// run it together rather than one group after the other.
	const bool face = cache.y == FT_FACE1 || cache.y == FT_FACE2;
	const bool f2 = cache.y == FT_FACE2;
	const XF xa = f2 ? H.xf2 : H.xf1, xb = f2 ? H.xf1 : H.xf2;
	const HullRef ha = f2 ? H.h2 : H.h1, hb = f2 ? H.h1 : H.h2;
	uint32_t state1;
	if (cache.y == FT_EDGES)
		state1 = read_edges(H.xf1, H.h1, H.xf2, H.h2, cache.z, cache.w, totalRadius);
	else if (face)
		state1 = read_face_thread(xa, ha, xb, hb, cache.z, totalRadius);
	else
		state1 = CT_EMPTY;
	if (state0 == CT_SEPARATION && state1 == CT_SEPARATION)
		return true; // separation cache hit
	if (state0 == CT_OVERLAP && state1 == CT_OVERLAP)
	{
		if (cache.y == FT_EDGES)
			rebuild_edge_contact(m, H.xf1, cache.z, H.h1, H.xf2, cache.w, H.h2);
		else if (face)
			rebuild_face_contact(m, xa, cache.z, ha, f2 ? H.r2 : H.r1, xb, hb, f2 ? H.r1 : H.r2, f2,
				f2 ? H.xf02 : H.xf01, f2 ? H.xf01 : H.xf02, H.status);
		if (m.pointCount > 0)
			return true; // overlap cache hit
	}
	cache.x = CT_EMPTY;
	return false;
}

// Warp-aggregated append of c to a list (the calling lanes of the warp).
__device__ __forceinline__ void warp_append(uint32_t* list, uint32_t* count, uint32_t c)
{
	uint32_t mask = __activemask();
	uint32_t lane = threadIdx.x & 31;
	uint32_t leader = __ffs(mask) - 1;
	uint32_t base = 0;
	if (lane == leader)
		base = atomicAdd(count, (uint32_t)__popc(mask));
	base = __shfl_sync(mask, base, leader);
	list[base + __popc(mask & ((1u << lane) - 1u))] = c;
}

// The SAT half of b3CollideHullsCache (collide_hulls.cpp:417-515), one warp
// per contact. cache is uniform across the warp; m is written by lane 0.
__device__ void sat_after_miss(DevManifold& m, const HullCtx& H, uint4& cache, uint32_t lane)
{
	float totalRadius = H.r1 + H.r2;
	uint32_t fi1, fi2, ei1, ei2;
	float fs1, fs2, es;
	warp_query_faces(H.xf1, H.h1, H.xf2, H.h2, lane, fi1, fs1);
	if (fs1 > totalRadius)
	{
		cache = make_uint4(CT_SEPARATION, FT_FACE1, fi1, fi1);
		return;
	}
	warp_query_faces(H.xf2, H.h2, H.xf1, H.h1, lane, fi2, fs2);
	if (fs2 > totalRadius)
	{
		cache = make_uint4(CT_SEPARATION, FT_FACE2, fi2, fi2);
		return;
	}
	warp_query_edges(H.xf1, H.h1, H.xf2, H.h2, lane, H.recs, H.maxUE, ei1, ei2, es);
	if (es > totalRadius)
	{
		cache = make_uint4(CT_SEPARATION, FT_EDGES, ei1, ei2);
		return;
	}
	const float kRelEdgeTol = 0.90f;
	const float kRelFaceTol = 0.98f;
	const float kAbsTol = 0.5f * B3G_LINEAR_SLOP;
	if (es > kRelEdgeTol * fmaxr(fs1, fs2) + kAbsTol)
	{
		if (lane == 0)
			build_edge_contact(m, H.xf1, ei1, H.h1, H.xf2, ei2, H.h2);
		cache = make_uint4(CT_OVERLAP, FT_EDGES, ei1, ei2);
		return;
	}
	if (fs2 > kRelFaceTol * fs1 + kAbsTol)
	{
		if (face_contact_all(m, H, true, fi2, lane) > 0)
		{
			cache = make_uint4(CT_OVERLAP, FT_FACE2, fi2, fi2);
			return;
		}
	}
	else
	{
		if (face_contact_all(m, H, false, fi1, lane) > 0)
		{
			cache = make_uint4(CT_OVERLAP, FT_FACE1, fi1, fi1);
			return;
		}
	}
	// Heuristic failed. Fallback.
	if (es > fmaxr(fs1, fs2))
	{
		if (lane == 0)
			build_edge_contact(m, H.xf1, ei1, H.h1, H.xf2, ei2, H.h2);
		cache = make_uint4(CT_OVERLAP, FT_EDGES, ei1, ei2);
		return;
	}
	if (fs2 > fs1)
	{
		if (face_contact_all(m, H, true, fi2, lane) > 0)
			cache = make_uint4(CT_OVERLAP, FT_FACE2, fi2, fi2);
	}
	else
	{
		if (face_contact_all(m, H, false, fi1, lane) > 0)
			cache = make_uint4(CT_OVERLAP, FT_FACE1, fi1, fi1);
	}
}

__device__ __forceinline__ void load_hull_ctx(const NPArgs& a, uint32_t c, HullCtx& H)
{
	uint32_t fa = a.pairA[c], fb = a.pairB[c];
	uint32_t ba = a.S.fixBody[fa], bb = a.S.fixBody[fb];
	H.xf1 = a.exA ? load_xf7(a.exA + 7 * (size_t)c) : body_xf(a.S, ba);
	H.xf2 = a.exB ? load_xf7(a.exB + 7 * (size_t)c) : body_xf(a.S, bb);
	H.xf01 = a.ex0A ? load_xf7(a.ex0A + 7 * (size_t)c) : body_xf0(a.S, ba);
	H.xf02 = a.ex0B ? load_xf7(a.ex0B + 7 * (size_t)c) : body_xf0(a.S, bb);
	H.h1 = hull_ref(a.S, a.S.fixHull[fa]);
	H.h2 = hull_ref(a.S, a.S.fixHull[fb]);
	H.r1 = a.S.fixParams[3 * fa].x;
	H.r2 = a.S.fixParams[3 * fb].x;
	H.status = a.status;
	H.recs = nullptr;
	H.maxUE = 0;
	H.clip = nullptr;
}

// Pass 1: one thread per hull-hull contact reads its feature cache.
__global__ void __launch_bounds__(128) k_hulls_probe(NPArgs a)
{
	uint32_t n = *a.listCount;
	for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		uint32_t c = a.list[t];
		int32_t prev = a.prevIndex[c];
		uint4 cache = prev >= 0 ? a.prevCache[prev] : make_uint4(CT_EMPTY, FT_FACE1, 0, 0);
		DevManifold& m = a.man[c];
		man_clear(m);
		bool done = false;
		if (a.convexCache)
		{
			HullCtx H;
			load_hull_ctx(a, c, H);
			done = probe_cache(m, H, cache);
		}
		a.cache[c] = cache;
		if (done)
			finish_convex(a, c, m);
		else
			warp_append(a.missList, a.missCount, c);
	}
}

// Bulk copies from global into shared memory (the TMA engine without a
// tensor map: cp.async.bulk, 16-byte aligned addresses, sizes multiples of 16
// bytes) that complete on a shared-memory barrier. Sources are this GPU's
// own memory; no multicast.
__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
	return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t arrivals)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(arrivals) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
				 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t phase)
{
	uint32_t done;
	asm volatile("{\n\t.reg .pred p;\n\t"
				 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
				 "selp.u32 %0, 1, 0, p;\n\t}"
				 : "=r"(done)
				 : "r"(smem_addr(bar)), "r"(phase)
				 : "memory");
	return done != 0;
}
__device__ __forceinline__ void bulk_to_shared(void* dst, const void* src, uint32_t bytes, unsigned long long* bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
					 smem_addr(dst)),
				 "l"(src), "r"(bytes), "r"(smem_addr(bar))
				 : "memory");
}

// Bytes of one warp's staging area: vertices, planes and half-edges of two
// hulls of the scene's largest sizes.
__host__ __device__ __forceinline__ size_t sat_stage_bytes(uint32_t maxV, uint32_t maxF, uint32_t maxE)
{
	return 2 * 16 * ((size_t)maxV + maxF + maxE);
}

// Waits at most STAGE_SPIN polls for the barrier's phase; every lane polls.
constexpr uint32_t STAGE_SPIN = 1u << 22;
__device__ __forceinline__ bool stage_wait(unsigned long long* bar, uint32_t phase)
{
	for (uint32_t k = 0; k < STAGE_SPIN; ++k)
		if (mbar_try_wait(bar, phase))
			return true;
	return false;
}

// Pass 2: one warp per contact the cache did not resolve (W warps per block).
// With STAGE, each pair's hull vertices, planes and half-edges are brought
// into the warp's shared memory by bulk copies (lane 0 issues six, the warp
// waits on its barrier), and the face and edge queries and the face contact
// read them there instead of from global memory, where every lane's loop
// over the other hull's vertices waited on each load. Shared memory per block:
// W barriers (16-byte rounded), then per warp its query / clip area
// (sat_warp_bytes), then per warp its staging area (sat_stage_bytes).
template <int W, bool STAGE>
__global__ void __launch_bounds__(W * 32) k_hulls_sat(NPArgs a, uint32_t maxUE)
{
	extern __shared__ float4 smem[];
	const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const size_t barBytes = STAGE ? ((W * 8 + 15) & ~15) : 0;
	char* base = reinterpret_cast<char*>(smem) + barBytes;
	char* wsm = base + (size_t)warp * sat_warp_bytes(maxUE);
	EdgeRec* recs = reinterpret_cast<EdgeRec*>(wsm);
	unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem) + warp;
	const size_t stageBytes = sat_stage_bytes(a.S.hullMaxV, a.S.hullMaxF, a.S.hullMaxE);
	char* stage = base + (size_t)W * sat_warp_bytes(maxUE) + (size_t)warp * stageBytes;
	uint32_t phase = 0;
	if (STAGE)
	{
		if (lane == 0)
		{
			mbar_init(bar, 1);
			asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
		}
		__syncwarp();
	}
	uint32_t n = *a.missCount;
	uint32_t gw = blockIdx.x * W + warp;
	uint32_t nw = gridDim.x * W;
	for (uint32_t t = gw; t < n; t += nw)
	{
		uint32_t c = a.missList[t];
		HullCtx H;
		load_hull_ctx(a, c, H);
		H.recs = recs;
		H.clip = reinterpret_cast<WarpClip*>(wsm);
		H.maxUE = maxUE;
		if (STAGE)
		{
			float4* v1 = reinterpret_cast<float4*>(stage);
			float4* p1 = v1 + H.h1.vCnt;
			uint4* e1 = reinterpret_cast<uint4*>(p1 + H.h1.fCnt);
			float4* v2 = reinterpret_cast<float4*>(e1 + H.h1.eCnt);
			float4* p2 = v2 + H.h2.vCnt;
			uint4* e2 = reinterpret_cast<uint4*>(p2 + H.h2.fCnt);
			if (lane == 0)
			{
				// The warp's reads of the previous pair (generic proxy) come
				// before these writes (async proxy).
				asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
				const uint32_t bytes = 16u * (H.h1.vCnt + H.h1.fCnt + H.h1.eCnt + H.h2.vCnt + H.h2.fCnt + H.h2.eCnt);
				mbar_arrive_expect_tx(bar, bytes);
				bulk_to_shared(v1, H.h1.v, 16u * H.h1.vCnt, bar);
				bulk_to_shared(p1, H.h1.p, 16u * H.h1.fCnt, bar);
				bulk_to_shared(e1, H.h1.e, 16u * H.h1.eCnt, bar);
				bulk_to_shared(v2, H.h2.v, 16u * H.h2.vCnt, bar);
				bulk_to_shared(p2, H.h2.p, 16u * H.h2.fCnt, bar);
				bulk_to_shared(e2, H.h2.e, 16u * H.h2.eCnt, bar);
			}
			const bool ok = stage_wait(bar, phase);
			if (!__all_sync(0xffffffffu, ok))
			{
				// The copies did not land in time: report it, wait (bounded)
				// for them before the shared memory goes away, and stop.
				if (lane == 0)
					atomicOr(a.status, B3G_ST_WAIT_TIMEOUT);
				stage_wait(bar, phase);
				return;
			}
			phase ^= 1u;
			H.h1.v = v1;
			H.h1.p = p1;
			H.h1.e = e1;
			H.h2.v = v2;
			H.h2.p = p2;
			H.h2.e = e2;
		}
		uint4 cache = a.cache[c];
		DevManifold& m = a.man[c];
		if (a.convexCache)
			sat_after_miss(m, H, cache, lane);
		else
			collide_hulls_nocache(m, H, lane);
		__syncwarp();
		if (lane == 0)
		{
			finish_convex(a, c, m);
			a.cache[c] = cache;
		}
		__syncwarp();
	}
}

// b3CollideHullAndTriangle (collide_hull_triangle.cpp:24-124) after the
// hull-hull SAT: points on a triangle edge that has a coplanar wing take the
// triangle's face normal (oriented from the hull to the triangle) so bodies
// slide over mesh edges. Lane 0 only.
__device__ void triangle_wing_normals(DevManifold& m, const float4 w4[3], const XF& xf1, const HullRef& h1,
	const XF& xf2, const HullRef& h2)
{
	PL plane2 = pmul(xf2, hp(h2, 0));
	V3 centroid1 = xmul(xf1, h1.centroid);
	V3 centroid2 = xmul(xf2, h2.centroid);
	for (uint32_t i = 0; i < m.pointCount; ++i)
	{
		DevPoint& mp = m.points[i];
		uint32_t inEdge2 = mp.key[2], outEdge2 = mp.key[3];
		uint32_t e2;
		if (mp.edgeContact)
			e2 = inEdge2;
		else
		{
			e2 = inEdge2 == B3G_NULL_EDGE ? outEdge2 : inEdge2;
			if (e2 == B3G_NULL_EDGE)
				continue;
		}
		uint32_t edgeIndex = e2 >> 1; // half-edges 2k, 2k + 1 lie on triangle edge k
		if (edgeIndex > 2 || w4[edgeIndex].w == 0.0f)
			continue;
		uint32_t ev1 = edgeIndex;
		uint32_t ev2 = edgeIndex + 1 < 3 ? edgeIndex + 1 : 0;
		V3 A = V3{w4[edgeIndex].x, w4[edgeIndex].y, w4[edgeIndex].z};
		V3 B = hv(h2, ev2);
		V3 C = hv(h2, ev1);
		V3 center = ((A + B) + C) / 3.0f;
		float distance = pdist(center, hp(h2, 0));
		const float kCoplanarTol = 0.005f;
		if (distance > -kCoplanarTol && distance < kCoplanarTol)
		{
			V3 localN1 = V3{mp.n[0], mp.n[1], mp.n[2]};
			V3 localC1 = V3{mp.p1[0], mp.p1[1], mp.p1[2]};
			V3 localC2 = V3{mp.p2[0], mp.p2[1], mp.p2[2]};
			V3 n1 = rot(xf1.q, localN1);
			V3 c1 = xmul(xf1, localC1);
			V3 c2 = xmul(xf2, localC2);
			float sep = dot(c2 - c1, n1);
			V3 n = plane2.n;
			if (dot(n, centroid2 - centroid1) < 0.0f)
				n = -n;
			V3 nc1 = c2 - sep * n;
			V3 ln = rotc(xf1.q, n);
			V3 lp = xmult(xf1, nc1);
			mp.n[0] = ln.x, mp.n[1] = ln.y, mp.n[2] = ln.z;
			mp.p1[0] = lp.x, mp.p1[1] = lp.y, mp.p1[2] = lp.z;
		}
	}
}

// Hull (A) against triangle (B): one warp per contact, the full SAT of
// b3CollideHulls without a feature cache (b3HullAndTriangleContact keeps
// none), on the triangle's two-faced hull.
template <int W>
__global__ void __launch_bounds__(W * 32) k_hull_triangle(NPArgs a, uint32_t maxUE)
{
	extern __shared__ float4 smem[];
	const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	char* wsm = reinterpret_cast<char*>(smem) + (size_t)warp * sat_warp_bytes(maxUE);
	EdgeRec* recs = reinterpret_cast<EdgeRec*>(wsm);
	uint32_t n = *a.listCount;
	for (uint32_t t = blockIdx.x * W + warp; t < n; t += gridDim.x * W)
	{
		uint32_t c = a.list[t];
		uint32_t fa = a.pairA[c], fb = a.pairB[c];
		HullCtx H;
		H.xf1 = a.exA ? load_xf7(a.exA + 7 * (size_t)c) : body_xf(a.S, a.S.fixBody[fa]);
		H.xf2 = a.exB ? load_xf7(a.exB + 7 * (size_t)c) : body_xf(a.S, a.S.fixBody[fb]);
		H.h1 = hull_ref(a.S, a.S.fixHull[fa]);
		H.h2 = tri_ref(a.S, fb);
		H.r1 = a.S.fixParams[3 * fa].x;
		H.r2 = a.S.fixParams[3 * fb + 2].y;
		H.status = a.status;
		H.recs = recs;
		H.clip = reinterpret_cast<WarpClip*>(wsm);
		H.maxUE = maxUE;
		DevManifold& m = a.man[c];
		if (lane == 0)
			man_clear(m);
		__syncwarp();
		collide_hulls_nocache(m, H, lane);
		__syncwarp();
		if (lane == 0)
		{
			float4 w4[3];
			for (int k = 0; k < 3; ++k)
				w4[k] = a.S.fixWing[3 * (size_t)fb + k];
			triangle_wing_normals(m, w4, H.xf1, H.h1, H.xf2, H.h2);
			finish_convex(a, c, m);
			a.cache[c] = make_uint4(B3G_NULL, B3G_NULL, B3G_NULL, B3G_NULL);
		}
		__syncwarp();
	}
}

// Mesh work items of hull-mesh contacts (hull A, mesh B): one warp per
// triangle, b3CollideHullAndTriangle on the child triangle
// (hull_mesh_contact.cpp:42-50), points tagged with the triangle. Sensor
// contacts record the triangle's overlap in pointCount.
template <int W>
__global__ void __launch_bounds__(W * 32) k_mesh_items_hull(NPArgs a, Buffers B, uint32_t maxUE)
{
	extern __shared__ float4 smem[];
	const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	char* wsm = reinterpret_cast<char*>(smem) + (size_t)warp * sat_warp_bytes(maxUE);
	EdgeRec* recs = reinterpret_cast<EdgeRec*>(wsm);
	uint32_t n = min(B.counters[CTR_MESH_PAIRS], B.meshPairCap);
	for (uint32_t i = blockIdx.x * W + warp; i < n; i += gridDim.x * W)
	{
		uint32_t c = B.meshPairC[i], t = B.meshPairT[i];
		uint32_t fa = a.pairA[c], fb = a.pairB[c];
		if (a.S.fixType[fa] != B3G_SHAPE_HULL || a.S.fixType[fb] != B3G_SHAPE_MESH)
			continue;
		MeshTri tri;
		mesh_triangle(a.S, fb, t, tri);
		HullCtx H;
		H.xf1 = body_xf(a.S, a.S.fixBody[fa]);
		H.xf2 = body_xf(a.S, a.S.fixBody[fb]);
		H.h1 = hull_ref(a.S, a.S.fixHull[fa]);
		H.h2 = mesh_tri_ref(tri);
		H.r1 = a.S.fixParams[3 * fa].x;
		H.r2 = tri.radius;
		H.status = a.status;
		H.recs = recs;
		H.clip = reinterpret_cast<WarpClip*>(wsm);
		H.maxUE = maxUE;
		DevManifold& m = B.meshPairMan[i];
		if (lane == 0)
			man_clear(m);
		__syncwarp();
		if ((a.S.fixFlags[fa] | a.S.fixFlags[fb]) & B3G_FIXTURE_SENSOR)
		{
			if (lane == 0)
			{
				GProxy pb;
				pb.gv = nullptr;
				pb.lv[0] = tri.v[0];
				pb.lv[1] = tri.v[1];
				pb.lv[2] = tri.v[2];
				pb.count = 3;
				pb.radius = tri.radius;
				GProxy pa;
				pa.gv = H.h1.v;
				pa.count = H.h1.vCnt;
				pa.radius = H.r1;
				GJKOut q = gjk(H.xf1, pa, H.xf2, pb, true);
				m.pointCount = q.distance <= 10.0f * B3G_EPSILON ? 1u : 0u;
			}
			__syncwarp();
			continue;
		}
		collide_hulls_nocache(m, H, lane);
		__syncwarp();
		if (lane == 0)
		{
			triangle_wing_normals(m, tri.wing, H.xf1, H.h1, H.xf2, H.h2);
			for (uint32_t j = 0; j < m.pointCount; ++j)
				m.points[j].triangleKey = t;
		}
		__syncwarp();
	}
}

} // namespace

void launch_hulls_sat(const NPArgs& a, uint32_t maxUE, const Tune& tune, cudaStream_t s);
size_t hull_sat_smem(int warps, uint32_t maxUE);

// Hull-triangle contacts (bucket BK_HULL_TRIANGLE), with the SAT kernel's
// warps per block.
void launch_hull_triangles(const NPArgs& base, const uint32_t* list, const uint32_t* count, uint32_t maxUE,
	const Tune& tune, cudaStream_t s)
{
	NPArgs a = base;
	a.list = list;
	a.listCount = count;
	uint32_t ue = maxUE > 3 ? maxUE : 3;
	const int bps = (int)tune.v[B3G_TUNE_SAT_BLOCKS];
	size_t smem;
	switch (tune.v[B3G_TUNE_SAT_WARPS])
	{
	case 2:
		smem = hull_sat_smem(2, ue);
		if (smem > 48 * 1024)
			cudaFuncSetAttribute(k_hull_triangle<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		k_hull_triangle<2><<<persistent_blocks(bps), 64, smem, s>>>(a, ue);
		break;
	case 8:
		smem = hull_sat_smem(8, ue);
		if (smem > 48 * 1024)
			cudaFuncSetAttribute(k_hull_triangle<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		k_hull_triangle<8><<<persistent_blocks(bps), 256, smem, s>>>(a, ue);
		break;
	default:
		smem = hull_sat_smem(4, ue);
		if (smem > 48 * 1024)
			cudaFuncSetAttribute(k_hull_triangle<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		k_hull_triangle<4><<<persistent_blocks(bps), 128, smem, s>>>(a, ue);
		break;
	}
}

template <int W, bool STAGE>
void launch_sat_kernel(const NPArgs& a, uint32_t maxUE, int blocksPerSM, size_t smem, cudaStream_t s)
{
	static size_t configured = 0;
	if (smem > 48 * 1024 && smem > configured)
	{
		cudaFuncSetAttribute(k_hulls_sat<W, STAGE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		configured = smem;
	}
	k_hulls_sat<W, STAGE><<<persistent_blocks(blocksPerSM), W * 32, smem, s>>>(a, maxUE);
}

// The staged kernel when its shared memory fits a block, else the kernel
// that reads the hulls from global memory.
template <int W>
void launch_sat(const NPArgs& a, uint32_t maxUE, int blocksPerSM, cudaStream_t s)
{
	const size_t plain = (size_t)W * sat_warp_bytes(maxUE);
	const size_t staged = ((W * 8 + 15) & ~(size_t)15) + plain +
		(size_t)W * sat_stage_bytes(a.S.hullMaxV, a.S.hullMaxF, a.S.hullMaxE);
	static int optin = -1;
	if (optin < 0)
	{
		int dev = 0;
		cudaGetDevice(&dev);
		if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
			optin = 48 * 1024;
	}
	if (staged <= (size_t)optin && a.S.hullMaxV > 0)
		launch_sat_kernel<W, true>(a, maxUE, blocksPerSM, staged, s);
	else
		launch_sat_kernel<W, false>(a, maxUE, blocksPerSM, plain, s);
}

void launch_hulls(const NPArgs& base, const uint32_t* list, const uint32_t* count, uint32_t maxUE, const Tune& tune,
	cudaStream_t s)
{
	NPArgs a = base;
	a.list = list;
	a.listCount = count;
	launch_hulls_probe(a, a.list, a.listCount, tune, s);
	launch_hulls_sat(a, maxUE, tune, s);
}

void launch_hulls_sat(const NPArgs& a, uint32_t maxUE, const Tune& tune, cudaStream_t s)
{
	const int bps = (int)tune.v[B3G_TUNE_SAT_BLOCKS];
	switch (tune.v[B3G_TUNE_SAT_WARPS])
	{
	case 2:
		launch_sat<2>(a, maxUE, bps, s);
		break;
	case 8:
		launch_sat<8>(a, maxUE, bps, s);
		break;
	default:
		launch_sat<4>(a, maxUE, bps, s);
		break;
	}
}

void launch_hulls_probe(const NPArgs& base, const uint32_t* list, const uint32_t* count, const Tune& tune,
	cudaStream_t s)
{
	NPArgs a = base;
	a.list = list;
	a.listCount = count;
	k_hulls_probe<<<persistent_blocks((int)tune.v[B3G_TUNE_PROBE]), 128, 0, s>>>(a);
}

// Dynamic shared memory of the SAT kernel with `warps` warps per block.
size_t hull_sat_smem(int warps, uint32_t maxUE)
{
	return (size_t)warps * sat_warp_bytes(maxUE);
}

void launch_mesh_items_hull(const NPArgs& a, const Buffers& B, uint32_t maxUE, const Tune& tune, cudaStream_t s)
{
	uint32_t ue = maxUE > 3 ? maxUE : 3;
	size_t smem = hull_sat_smem(4, ue);
	if (smem > 48 * 1024)
		cudaFuncSetAttribute(k_mesh_items_hull<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	k_mesh_items_hull<4><<<persistent_blocks((int)tune.v[B3G_TUNE_SAT_BLOCKS]), 128, smem, s>>>(a, B, ue);
}

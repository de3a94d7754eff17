// Host-side convex hull construction (scene input, not on the per-step path).
//
// Incremental hull in double precision: start from a non-degenerate
// tetrahedron, add points one at a time, delete the faces a point sees and
// fan new triangles from the horizon. The result is converted to the b3Hull
// half-edge layout (include/bounce/collision/geometry/hull.h:24-72): every
// undirected edge owns two consecutive half-edges 2k / 2k+1 that are each
// other's twin (the pairing b3QueryEdgeSeparation asserts, sat.cpp:131),
// face loops are counter-clockwise seen from outside, and each face plane is
// computed in single precision from its first three vertices with the
// reference's b3Plane(A, B, C) formula (plane.h:43-48).

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/b3g_hull.h"

namespace {

struct V3
{
	double x, y, z;
};

inline V3 sub(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 cross(const V3& a, const V3& b)
{
	return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double len(const V3& a) { return std::sqrt(dot(a, a)); }

struct Tri
{
	int v[3];
	V3 n;
	double d;
	bool alive;
};

Tri make_tri(const std::vector<V3>& p, int a, int b, int c)
{
	Tri t;
	t.v[0] = a;
	t.v[1] = b;
	t.v[2] = c;
	V3 n = cross(sub(p[b], p[a]), sub(p[c], p[a]));
	double l = len(n);
	if (l > 0)
	{
		n.x /= l;
		n.y /= l;
		n.z /= l;
	}
	t.n = n;
	t.d = dot(n, p[a]);
	t.alive = true;
	return t;
}

// Face loops (vertex index lists, CCW from outside) -> b3Hull arrays.
int emit(const std::vector<V3>& pts, const std::vector<std::vector<int>>& loops, float* verts,
	uint32_t* edges, uint32_t* faces, float* planes, float* centroid, uint32_t* counts)
{
	// Compact the used vertices in first-use order.
	std::vector<int> remap(pts.size(), -1);
	int nv = 0;
	for (const auto& L : loops)
		for (int v : L)
			if (remap[v] < 0)
				remap[v] = nv++;
	std::vector<float> fv(3 * nv);
	for (size_t i = 0; i < pts.size(); ++i)
	{
		if (remap[i] < 0)
			continue;
		fv[3 * remap[i] + 0] = (float)pts[i].x;
		fv[3 * remap[i] + 1] = (float)pts[i].y;
		fv[3 * remap[i] + 2] = (float)pts[i].z;
	}

	// Half-edges: one pair per undirected edge, allocated on first sight.
	struct HE
	{
		uint32_t origin, twin, face, prev, next;
	};
	std::vector<HE> he;
	std::vector<long long> keys; // directed key a*65536+b -> index in he
	std::vector<uint32_t> keyIndex;
	auto find = [&](int a, int b) -> int {
		long long k = (long long)a * 65536 + b;
		for (size_t i = 0; i < keys.size(); ++i)
			if (keys[i] == k)
				return (int)keyIndex[i];
		return -1;
	};
	std::vector<uint32_t> faceFirst(loops.size());
	for (size_t f = 0; f < loops.size(); ++f)
	{
		const auto& L = loops[f];
		int m = (int)L.size();
		std::vector<uint32_t> ids(m);
		for (int i = 0; i < m; ++i)
		{
			int a = remap[L[i]], b = remap[L[(i + 1) % m]];
			int idx = find(a, b);
			if (idx < 0)
			{
				uint32_t base = (uint32_t)he.size();
				he.push_back({(uint32_t)a, base + 1, 0, 0, 0});
				he.push_back({(uint32_t)b, base, 0, 0, 0});
				keys.push_back((long long)a * 65536 + b);
				keyIndex.push_back(base);
				keys.push_back((long long)b * 65536 + a);
				keyIndex.push_back(base + 1);
				idx = (int)base;
			}
			ids[i] = (uint32_t)idx;
		}
		for (int i = 0; i < m; ++i)
		{
			HE& e = he[ids[i]];
			e.face = (uint32_t)f;
			e.next = ids[(i + 1) % m];
			e.prev = ids[(i + m - 1) % m];
		}
		faceFirst[f] = ids[0];
	}

	// Planes in single precision, b3Plane(A, B, C) of the first three vertices.
	for (size_t f = 0; f < loops.size(); ++f)
	{
		const auto& L = loops[f];
		const float* A = &fv[3 * remap[L[0]]];
		const float* B = &fv[3 * remap[L[1]]];
		const float* C = &fv[3 * remap[L[2]]];
		float e1x = B[0] - A[0], e1y = B[1] - A[1], e1z = B[2] - A[2];
		float e2x = C[0] - A[0], e2y = C[1] - A[1], e2z = C[2] - A[2];
		float nx = e1y * e2z - e1z * e2y;
		float ny = e1z * e2x - e1x * e2z;
		float nz = e1x * e2y - e1y * e2x;
		float l = std::sqrt(nx * nx + ny * ny + nz * nz);
		if (l > 1.1920928955078125e-7f)
		{
			float s = 1.0f / l;
			nx = s * nx;
			ny = s * ny;
			nz = s * nz;
		}
		planes[4 * f + 0] = nx;
		planes[4 * f + 1] = ny;
		planes[4 * f + 2] = nz;
		planes[4 * f + 3] = nx * A[0] + ny * A[1] + nz * A[2];
		faces[f] = faceFirst[f];
	}
	for (size_t i = 0; i < he.size(); ++i)
	{
		edges[5 * i + 0] = he[i].origin;
		edges[5 * i + 1] = he[i].twin;
		edges[5 * i + 2] = he[i].face;
		edges[5 * i + 3] = he[i].prev;
		edges[5 * i + 4] = he[i].next;
	}
	std::memcpy(verts, fv.data(), sizeof(float) * 3 * nv);

	// Volume centroid of the polyhedron (fan of tetrahedra from vertex 0).
	V3 o = {fv[0], fv[1], fv[2]};
	double vol = 0, cx = 0, cy = 0, cz = 0;
	for (const auto& L : loops)
	{
		for (size_t i = 1; i + 1 < L.size(); ++i)
		{
			V3 a = {fv[3 * remap[L[0]]], fv[3 * remap[L[0]] + 1], fv[3 * remap[L[0]] + 2]};
			V3 b = {fv[3 * remap[L[i]]], fv[3 * remap[L[i]] + 1], fv[3 * remap[L[i]] + 2]};
			V3 c = {fv[3 * remap[L[i + 1]]], fv[3 * remap[L[i + 1]] + 1], fv[3 * remap[L[i + 1]] + 2]};
			double v6 = dot(sub(a, o), cross(sub(b, o), sub(c, o)));
			vol += v6;
			cx += v6 * (o.x + a.x + b.x + c.x) / 4;
			cy += v6 * (o.y + a.y + b.y + c.y) / 4;
			cz += v6 * (o.z + a.z + b.z + c.z) / 4;
		}
	}
	if (vol > 0)
	{
		centroid[0] = (float)(cx / vol);
		centroid[1] = (float)(cy / vol);
		centroid[2] = (float)(cz / vol);
	}
	else
	{
		centroid[0] = centroid[1] = centroid[2] = 0;
	}
	counts[0] = (uint32_t)nv;
	counts[1] = (uint32_t)he.size();
	counts[2] = (uint32_t)loops.size();
	return 0;
}

} // namespace

extern "C" int b3g_hull_from_points(const float* points, uint32_t n, float* verts, uint32_t* edges,
	uint32_t* faces, float* planes, float* centroid, uint32_t* counts)
{
	if (n < 4 || n > B3G_HULL_MAX_POINTS)
		return -1;
	std::vector<V3> p(n);
	for (uint32_t i = 0; i < n; ++i)
		p[i] = {points[3 * i], points[3 * i + 1], points[3 * i + 2]};

	// Scale-aware tolerance.
	double ext = 0;
	for (const V3& q : p)
		ext = std::fmax(ext, std::fmax(std::fabs(q.x), std::fmax(std::fabs(q.y), std::fabs(q.z))));
	const double eps = 1e-9 * (ext > 0 ? ext : 1) * 8;

	// Initial tetrahedron.
	int i0 = 0, i1 = -1, i2 = -1, i3 = -1;
	double best = 0;
	for (uint32_t i = 1; i < n; ++i)
	{
		double d = len(sub(p[i], p[i0]));
		if (d > best)
		{
			best = d;
			i1 = (int)i;
		}
	}
	if (i1 < 0 || best <= eps)
		return -1;
	best = 0;
	for (uint32_t i = 0; i < n; ++i)
	{
		double d = len(cross(sub(p[i1], p[i0]), sub(p[i], p[i0])));
		if (d > best)
		{
			best = d;
			i2 = (int)i;
		}
	}
	if (i2 < 0 || best <= eps)
		return -1;
	V3 n012 = cross(sub(p[i1], p[i0]), sub(p[i2], p[i0]));
	best = 0;
	for (uint32_t i = 0; i < n; ++i)
	{
		double d = std::fabs(dot(n012, sub(p[i], p[i0])));
		if (d > best)
		{
			best = d;
			i3 = (int)i;
		}
	}
	if (i3 < 0 || best <= eps * len(n012))
		return -1;

	std::vector<Tri> tris;
	if (dot(n012, sub(p[i3], p[i0])) > 0)
	{
		// i3 above the plane of (i0, i1, i2): orient base downwards.
		tris.push_back(make_tri(p, i0, i2, i1));
		tris.push_back(make_tri(p, i0, i1, i3));
		tris.push_back(make_tri(p, i1, i2, i3));
		tris.push_back(make_tri(p, i2, i0, i3));
	}
	else
	{
		tris.push_back(make_tri(p, i0, i1, i2));
		tris.push_back(make_tri(p, i0, i3, i1));
		tris.push_back(make_tri(p, i1, i3, i2));
		tris.push_back(make_tri(p, i2, i3, i0));
	}

	std::vector<char> visible;
	for (uint32_t pi = 0; pi < n; ++pi)
	{
		if ((int)pi == i0 || (int)pi == i1 || (int)pi == i2 || (int)pi == i3)
			continue;
		visible.assign(tris.size(), 0);
		bool any = false;
		for (size_t t = 0; t < tris.size(); ++t)
		{
			if (!tris[t].alive)
				continue;
			if (dot(tris[t].n, p[pi]) - tris[t].d > eps)
			{
				visible[t] = 1;
				any = true;
			}
		}
		if (!any)
			continue;
		// Horizon: directed edges of visible faces whose reverse edge belongs
		// to a live non-visible face.
		std::vector<std::pair<int, int>> horizon;
		for (size_t t = 0; t < tris.size(); ++t)
		{
			if (!visible[t])
				continue;
			for (int k = 0; k < 3; ++k)
			{
				int a = tris[t].v[k], b = tris[t].v[(k + 1) % 3];
				bool reverseVisible = false;
				for (size_t u = 0; u < tris.size(); ++u)
				{
					if (!tris[u].alive || !visible[u])
						continue;
					for (int m = 0; m < 3; ++m)
						if (tris[u].v[m] == b && tris[u].v[(m + 1) % 3] == a)
							reverseVisible = true;
				}
				if (!reverseVisible)
					horizon.push_back({a, b});
			}
		}
		for (size_t t = 0; t < tris.size(); ++t)
			if (visible[t])
				tris[t].alive = false;
		for (const auto& e : horizon)
			tris.push_back(make_tri(p, e.first, e.second, (int)pi));
	}

	std::vector<std::vector<int>> loops;
	for (const Tri& t : tris)
		if (t.alive)
			loops.push_back({t.v[0], t.v[1], t.v[2]});
	return emit(p, loops, verts, edges, faces, planes, centroid, counts);
}

extern "C" int b3g_hull_box(float ex, float ey, float ez, float* verts, uint32_t* edges,
	uint32_t* faces, float* planes, float* centroid, uint32_t* counts)
{
	std::vector<V3> p = {
		{-ex, -ey, -ez}, {ex, -ey, -ez}, {ex, ey, -ez}, {-ex, ey, -ez},
		{-ex, -ey, ez}, {ex, -ey, ez}, {ex, ey, ez}, {-ex, ey, ez},
	};
	// Counter-clockwise seen from outside.
	std::vector<std::vector<int>> loops = {
		{0, 4, 7, 3}, // -x
		{1, 2, 6, 5}, // +x
		{0, 1, 5, 4}, // -y
		{3, 7, 6, 2}, // +y
		{0, 3, 2, 1}, // -z
		{4, 5, 6, 7}, // +z
	};
	int rc = emit(p, loops, verts, edges, faces, planes, centroid, counts);
	centroid[0] = centroid[1] = centroid[2] = 0;
	return rc;
}

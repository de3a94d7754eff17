/*
 * CPU restatement of the reference's broadphase front end, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: compiled into oracle/_ref/librestate.so by
 * oracle/Makefile and called by tests/ as a second, independent checker of
 * the fat-AABB update and the contact set; never linked by the product.
 * Pinned against the golden fixtures of tests/golden (generated by running
 * the reference itself) in tests/test_golden.py.
 *
 * Restated functions (reference file:line):
 *   quaternion rotate                     include/bounce/common/math/quat.h:270-274
 *   transform * vector                    include/bounce/common/math/transform.h:66-69
 *   b3Shape::ComputeAABB (sphere, capsule, triangle, hull)
 *       src/bounce/collision/shapes/sphere_shape.cpp:51-57, capsule_shape.cpp:124-131,
 *       triangle_shape.cpp:59-67, hull_shape.cpp:160-164, aabb.h:53-62
 *   b3Body::SynchronizeFixtures           src/bounce/dynamics/body.cpp:216-238
 *   b3Fixture::Synchronize                src/bounce/dynamics/fixture.cpp:120-132
 *   b3DynamicTree::CreateProxy / MoveProxy src/bounce/collision/trees/dynamic_tree.cpp:108-207
 *   b3TestOverlap                         include/bounce/collision/geometry/aabb.h:347-367
 *   AddPair filters + b3Contact::Create order
 *       src/bounce/dynamics/contact_manager.cpp:98-160, body.cpp:240-263,
 *       src/bounce/dynamics/contacts/contact.cpp:253-322, broad_phase.cpp:341-342
 *
 * Built with -ffp-contract=off so every float operation rounds separately,
 * in the order written, as in the reference.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define EXT 0.2f   /* B3_AABB_EXTENSION, common.h:73 */
#define MULT 2.0f  /* B3_AABB_MULTIPLIER, common.h:78 */

typedef struct { float x, y, z; } v3;
typedef struct { v3 v; float s; } q4;

static v3 add(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static v3 sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3 scl(float s, v3 a) { v3 r = {s * a.x, s * a.y, s * a.z}; return r; }
static v3 crs(v3 a, v3 b)
{
	v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
	return r;
}
static float mn(float a, float b) { return a < b ? a : b; }
static float mx(float a, float b) { return a > b ? a : b; }
static v3 vmn(v3 a, v3 b) { v3 r = {mn(a.x, b.x), mn(a.y, b.y), mn(a.z, b.z)}; return r; }
static v3 vmx(v3 a, v3 b) { v3 r = {mx(a.x, b.x), mx(a.y, b.y), mx(a.z, b.z)}; return r; }

/* v + s*t + qv x t, t = 2 (qv x v) */
static v3 rotate(q4 q, v3 v)
{
	v3 t = scl(2.0f, crs(q.v, v));
	return add(add(v, scl(q.s, t)), crs(q.v, t));
}

typedef struct { v3 p; q4 q; } xf;
static v3 xmul(xf T, v3 v) { return add(rotate(T.q, v), T.p); }

typedef struct { v3 lo, hi; } box;

/* ComputeAABB for one transform. params: 12 floats; hull vertices: 3 floats each. */
static box shape_aabb(uint32_t type, const float* p, const float* hv, uint32_t hn, xf T)
{
	box b;
	if (type == 0)
	{
		v3 c = {p[0], p[1], p[2]};
		v3 r = {p[3], p[3], p[3]};
		c = xmul(T, c);
		b.lo = sub(c, r);
		b.hi = add(c, r);
	}
	else if (type == 1)
	{
		v3 a = {p[0], p[1], p[2]}, c = {p[3], p[4], p[5]};
		v3 r = {p[6], p[6], p[6]};
		a = xmul(T, a);
		c = xmul(T, c);
		b.lo = sub(vmn(a, c), r);
		b.hi = add(vmx(a, c), r);
	}
	else if (type == 2)
	{
		/* The reference ignores the transform for triangles. */
		v3 a = {p[0], p[1], p[2]}, c = {p[3], p[4], p[5]}, d = {p[6], p[7], p[8]};
		v3 r = {p[9], p[9], p[9]};
		b.lo = sub(vmn(a, vmn(c, d)), r);
		b.hi = add(vmx(a, vmx(c, d)), r);
	}
	else
	{
		v3 v0 = {hv[0], hv[1], hv[2]};
		b.lo = b.hi = xmul(T, v0);
		for (uint32_t i = 1; i < hn; ++i)
		{
			v3 v = {hv[3 * i], hv[3 * i + 1], hv[3 * i + 2]};
			v = xmul(T, v);
			b.lo = vmn(b.lo, v);
			b.hi = vmx(b.hi, v);
		}
		float r = p[0];
		b.lo.x -= r; b.lo.y -= r; b.lo.z -= r;
		b.hi.x += r; b.hi.y += r; b.hi.z += r;
	}
	return b;
}

static int contains(box a, box b)
{
	return a.lo.x <= b.lo.x && a.lo.y <= b.lo.y && a.lo.z <= b.lo.z &&
		b.hi.x <= a.hi.x && b.hi.y <= a.hi.y && b.hi.z <= a.hi.z;
}

/*
 * Fat-AABB update of every fixture. state: 17 floats per body (xf.p, xf.q,
 * worldCenter0, orientation0, localCenter). fat: 6 floats per fixture (in:
 * previous, out: new). moved: 1 if re-inserted (or created).
 * creation != 0: b3DynamicTree::CreateProxy; otherwise bodies that are
 * asleep or static are not synchronised (world.cpp:427-442).
 */
void rs_sync(int creation, uint32_t nf, const uint32_t* fixBody, const uint32_t* fixType, const uint32_t* fixHull,
	const float* params, const uint32_t* bodyType, const uint8_t* awake, const float* state, const uint32_t* hullDesc,
	const float* hullVerts, float* fat, uint8_t* moved)
{
	for (uint32_t i = 0; i < nf; ++i)
	{
		uint32_t b = fixBody[i];
		const float* s = state + 17 * (size_t)b;
		xf T1 = {{s[0], s[1], s[2]}, {{s[3], s[4], s[5]}, s[6]}};
		const float* p = params + 12 * (size_t)i;
		const float* hv = 0;
		uint32_t hn = 0;
		if (fixType[i] == 3)
		{
			const uint32_t* d = hullDesc + 6 * (size_t)fixHull[i];
			hv = hullVerts + 3 * (size_t)d[0];
			hn = d[1];
		}
		float* f = fat + 6 * (size_t)i;
		if (creation)
		{
			box a = shape_aabb(fixType[i], p, hv, hn, T1);
			f[0] = a.lo.x - EXT; f[1] = a.lo.y - EXT; f[2] = a.lo.z - EXT;
			f[3] = a.hi.x + EXT; f[4] = a.hi.y + EXT; f[5] = a.hi.z + EXT;
			moved[i] = 1;
			continue;
		}
		if (bodyType[b] == 0 || !awake[b])
		{
			moved[i] = 0;
			continue;
		}
		/* xf0 from the sweep start (body.cpp:222-224) */
		q4 q0 = {{s[10], s[11], s[12]}, s[13]};
		v3 c0 = {s[7], s[8], s[9]}, lc = {s[14], s[15], s[16]};
		xf T0 = {sub(c0, rotate(q0, lc)), q0};
		box a1 = shape_aabb(fixType[i], p, hv, hn, T0);
		box a2 = shape_aabb(fixType[i], p, hv, hn, T1);
		box aabb = {vmn(a1.lo, a2.lo), vmx(a1.hi, a2.hi)};
		v3 c1 = scl(0.5f, add(a1.lo, a1.hi)), c2 = scl(0.5f, add(a2.lo, a2.hi));
		v3 d = scl(MULT, sub(c2, c1));
		box fb = aabb;
		fb.lo.x -= EXT; fb.lo.y -= EXT; fb.lo.z -= EXT;
		fb.hi.x += EXT; fb.hi.y += EXT; fb.hi.z += EXT;
		if (d.x < 0.0f) fb.lo.x += d.x; else fb.hi.x += d.x;
		if (d.y < 0.0f) fb.lo.y += d.y; else fb.hi.y += d.y;
		if (d.z < 0.0f) fb.lo.z += d.z; else fb.hi.z += d.z;
		box tree = {{f[0], f[1], f[2]}, {f[3], f[4], f[5]}};
		if (contains(tree, aabb))
		{
			box huge = fb;
			float e = 4.0f * EXT;
			huge.lo.x -= e; huge.lo.y -= e; huge.lo.z -= e;
			huge.hi.x += e; huge.hi.y += e; huge.hi.z += e;
			if (contains(huge, tree))
			{
				moved[i] = 0;
				continue;
			}
		}
		f[0] = fb.lo.x; f[1] = fb.lo.y; f[2] = fb.lo.z;
		f[3] = fb.hi.x; f[4] = fb.hi.y; f[5] = fb.hi.z;
		moved[i] = 1;
	}
}

/* b3Contact::s_registers: registered type pairs and the primary order. */
static int registered(uint32_t a, uint32_t b)
{
	static const char reg[5][5] = {
		{1, 1, 1, 1, 1}, {1, 1, 1, 1, 1}, {1, 1, 0, 1, 0}, {1, 1, 1, 1, 1}, {1, 1, 0, 1, 0}};
	return reg[a][b];
}
static int primary(uint32_t a, uint32_t b)
{
	static const char pri[5][5] = {
		{1, 0, 0, 0, 0}, {1, 1, 0, 0, 0}, {1, 1, 0, 0, 0}, {1, 1, 1, 1, 1}, {1, 1, 0, 0, 0}};
	return pri[a][b];
}

/*
 * Contact set for the fat AABBs: every overlapping pair of fixtures of
 * different bodies with at least one dynamic body and a registered shape
 * pair, as (fixture A, fixture B) after the factory's A/B order. Returns the
 * number of contacts (records written up to cap).
 */
uint32_t rs_pairs(uint32_t nf, const float* fat, const uint32_t* fixBody, const uint32_t* bodyType,
	const uint32_t* fixType, const uint32_t* fixKey, uint32_t* out, uint32_t cap)
{
	uint32_t n = 0;
	for (uint32_t i = 0; i < nf; ++i)
	{
		const float* a = fat + 6 * (size_t)i;
		for (uint32_t j = i + 1; j < nf; ++j)
		{
			const float* b = fat + 6 * (size_t)j;
			if (a[3] < b[0] || a[0] > b[3] || a[4] < b[1] || a[1] > b[4] || a[5] < b[2] || a[2] > b[5])
				continue;
			if (fixBody[i] == fixBody[j])
				continue;
			if (bodyType[fixBody[i]] != 2 && bodyType[fixBody[j]] != 2)
				continue;
			if (!registered(fixType[i], fixType[j]))
				continue;
			uint32_t f1 = fixKey[i] < fixKey[j] ? i : j;
			uint32_t f2 = fixKey[i] < fixKey[j] ? j : i;
			if (!primary(fixType[f1], fixType[f2]))
			{
				uint32_t t = f1;
				f1 = f2;
				f2 = t;
			}
			if (n < cap)
			{
				out[2 * n] = f1;
				out[2 * n + 1] = f2;
			}
			++n;
		}
	}
	return n;
}

// Headless driver around the unmodified reference (Bounce) library.
//
// TEST INFRASTRUCTURE ONLY: this file is compiled together with the
// reference's own sources into oracle/_ref/libb3ref{32,64}.so. It is loaded by
// tests/, by __graft_entry__.smoke() as the checker and by bench.py's CPU
// baseline leg; the product never links or calls it.
//
// It builds a b3World from flat arrays (the same arrays the product's C ABI
// takes), drives the collision pass exactly as b3World::Step and the tail of
// b3World::Solve do, and dumps the contact list, manifolds and hull feature
// caches in a fixed record layout that tests compare against.
//
// Reference call sites mirrored here:
//   first pass   = b3World::Step with dt = 0  (src/bounce/dynamics/world.cpp:201-225)
//   later passes = "Find New Pairs" block     (world.cpp:424-449) followed by
//                  b3ContactManager::UpdateContacts (contact_manager.cpp:225-287)
// Bodies are moved kinematically between passes: the driver writes the sweep
// (worldCenter0/orientation0 = previous, worldCenter/orientation = current)
// and lets b3Body::SynchronizeTransform (body.h) derive m_xf, which is what
// b3Island::Solve leaves behind after integrating positions.

#include <algorithm>
#include <assert.h>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <float.h>
#include <new>
#include <stdarg.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <vector>

// The harness needs the engine's private state (sweeps, the contact manager,
// the per-body fixture sync). Access specifiers do not change layout.
#define private public
#define protected public
#include <bounce/bounce.h>
#include <bounce/dynamics/contacts/hull_contact.h>
#include <bounce/dynamics/contacts/mesh_contact.h>
#include <bounce/collision/sat/sat.h>
#include <bounce/dynamics/contacts/contact_solver.h>
#include <bounce/dynamics/time_step.h>
#include <bounce/collision/gjk/gjk_proxy.h>
#include <bounce/collision/time_of_impact.h>
#undef private
#undef protected

#define REF_API extern "C" __attribute__((visibility("default")))

// Runtime switch of the hull feature cache (collide_hulls.cpp:27).
extern bool b3_convexCache;

// ---------------------------------------------------------------------------
// Fixed dump records (doubles so the FP32 and FP64 builds share one layout).

struct DumpPoint
{
	double localNormal1[3];
	double localPoint1[3];
	double localPoint2[3];
	double normalImpulse;
	uint32_t triangleKey;
	uint32_t key[4];
	uint32_t persisting;
	uint32_t edgeContact;
	uint32_t pad;
};

struct DumpManifold
{
	uint32_t pointCount;
	uint32_t pad;
	double tangentImpulse[2];
	double motorImpulse;
	DumpPoint points[4];
};

struct DumpContact
{
	uint32_t fixtureA;
	uint32_t fixtureB;
	uint32_t flags;          // bit0 touching
	uint32_t manifoldCount;
	uint32_t cache[4];       // hull-hull feature cache: cacheType, featureType, index1, index2
	DumpManifold manifolds[3];
};

static void DumpM(DumpManifold* out, const b3Manifold& m)
{
	memset(out, 0, sizeof(DumpManifold));
	out->pointCount = m.pointCount;
	out->tangentImpulse[0] = m.tangentImpulse.x;
	out->tangentImpulse[1] = m.tangentImpulse.y;
	out->motorImpulse = m.motorImpulse;
	for (uint32 i = 0; i < m.pointCount && i < 4; ++i)
	{
		const b3ManifoldPoint& p = m.points[i];
		DumpPoint* q = out->points + i;
		for (int k = 0; k < 3; ++k)
		{
			q->localNormal1[k] = p.localNormal1[k];
			q->localPoint1[k] = p.localPoint1[k];
			q->localPoint2[k] = p.localPoint2[k];
		}
		q->normalImpulse = p.normalImpulse;
		q->triangleKey = p.id.triangleKey;
		q->key[0] = p.id.key.pair.inEdge1;
		q->key[1] = p.id.key.pair.outEdge1;
		q->key[2] = p.id.key.pair.inEdge2;
		q->key[3] = p.id.key.pair.outEdge2;
		q->persisting = p.persisting ? 1 : 0;
		q->edgeContact = p.edgeContact ? 1 : 0;
	}
}

// ---------------------------------------------------------------------------
// Hull pool: b3Hull views over flat arrays.
//   desc[6*h] = vertexOffset, vertexCount, edgeOffset, edgeCount, faceOffset, faceCount
//   edges: 5 u32 per half-edge (origin, twin, face, prev, next), hull-local
//   planes: 4 floats per face (normal xyz, offset)

struct HullPool
{
	std::vector<b3Hull> hulls;
	std::vector<b3Vec3> verts;
	std::vector<b3HalfEdge> edges;
	std::vector<b3Face> faces;
	std::vector<b3Plane> planes;
	// triangle meshes (b3Mesh owns its static tree, so it is not copied)
	std::vector<b3Mesh*> meshes;
	std::vector<std::vector<b3Vec3>*> meshVerts;
	std::vector<std::vector<b3MeshTriangle>*> meshTris;
	~HullPool()
	{
		for (size_t i = 0; i < meshes.size(); ++i)
		{
			delete meshes[i];
			delete meshVerts[i];
			delete meshTris[i];
		}
	}
};

// Triangle meshes: desc 4 u32 per mesh (vertex offset, vertex count, triangle
// offset, triangle count), vertices 3 floats, triangles 3 u32 (mesh-local
// vertex indices). Each mesh gets its static tree and adjacency as
// b3Mesh::BuildTree / BuildAdjacency build them.
REF_API void refh_add_meshes(void* p, uint32_t nm, const uint32_t* desc, const float* mv, const uint32_t* mt)
{
	HullPool* pool = (HullPool*)p;
	for (uint32_t m = 0; m < nm; ++m)
	{
		const uint32_t vOff = desc[4 * m], vCnt = desc[4 * m + 1], tOff = desc[4 * m + 2], tCnt = desc[4 * m + 3];
		std::vector<b3Vec3>* V = new std::vector<b3Vec3>(vCnt);
		std::vector<b3MeshTriangle>* T = new std::vector<b3MeshTriangle>(tCnt);
		for (uint32_t i = 0; i < vCnt; ++i)
			(*V)[i].Set(mv[3 * (vOff + i)], mv[3 * (vOff + i) + 1], mv[3 * (vOff + i) + 2]);
		for (uint32_t i = 0; i < tCnt; ++i)
		{
			(*T)[i].v1 = mt[3 * (tOff + i)];
			(*T)[i].v2 = mt[3 * (tOff + i) + 1];
			(*T)[i].v3 = mt[3 * (tOff + i) + 2];
		}
		b3Mesh* mesh = new b3Mesh();
		mesh->vertexCount = vCnt;
		mesh->vertices = V->data();
		mesh->triangleCount = tCnt;
		mesh->triangles = T->data();
		mesh->BuildTree();
		mesh->BuildAdjacency();
		pool->meshes.push_back(mesh);
		pool->meshVerts.push_back(V);
		pool->meshTris.push_back(T);
	}
}

// Wing vertices of every triangle of mesh m (3 u32 each; B3_NULL_VERTEX for
// an open edge), for checking the pipeline's adjacency.
REF_API void refh_mesh_wings(void* p, uint32_t m, uint32_t* out)
{
	const b3Mesh* mesh = ((HullPool*)p)->meshes[m];
	for (uint32_t i = 0; i < mesh->triangleCount; ++i)
	{
		out[3 * i] = mesh->triangles[i].u1;
		out[3 * i + 1] = mesh->triangles[i].u2;
		out[3 * i + 2] = mesh->triangles[i].u3;
	}
}

REF_API void* refh_create(uint32_t nh, const uint32_t* desc, const float* hv, const uint32_t* he,
	const uint32_t* hf, const float* hp, const float* hc)
{
	HullPool* pool = new HullPool;
	uint32_t nv = 0, ne = 0, nf = 0;
	for (uint32_t h = 0; h < nh; ++h)
	{
		nv = std::max(nv, desc[6 * h + 0] + desc[6 * h + 1]);
		ne = std::max(ne, desc[6 * h + 2] + desc[6 * h + 3]);
		nf = std::max(nf, desc[6 * h + 4] + desc[6 * h + 5]);
	}
	pool->verts.resize(nv);
	pool->edges.resize(ne);
	pool->faces.resize(nf);
	pool->planes.resize(nf);
	for (uint32_t i = 0; i < nv; ++i)
		pool->verts[i].Set(hv[3 * i + 0], hv[3 * i + 1], hv[3 * i + 2]);
	for (uint32_t i = 0; i < ne; ++i)
		pool->edges[i] = b3MakeEdge(he[5 * i + 0], he[5 * i + 1], he[5 * i + 2], he[5 * i + 3], he[5 * i + 4]);
	for (uint32_t i = 0; i < nf; ++i)
	{
		pool->faces[i].edge = hf[i];
		pool->planes[i].normal.Set(hp[4 * i + 0], hp[4 * i + 1], hp[4 * i + 2]);
		pool->planes[i].offset = hp[4 * i + 3];
	}
	pool->hulls.resize(nh);
	for (uint32_t h = 0; h < nh; ++h)
	{
		b3Hull& H = pool->hulls[h];
		H.centroid.Set(hc[3 * h + 0], hc[3 * h + 1], hc[3 * h + 2]);
		H.vertexCount = desc[6 * h + 1];
		H.vertices = pool->verts.data() + desc[6 * h + 0];
		H.edgeCount = desc[6 * h + 3];
		H.edges = pool->edges.data() + desc[6 * h + 2];
		H.faceCount = desc[6 * h + 5];
		H.faces = pool->faces.data() + desc[6 * h + 4];
		H.planes = pool->planes.data() + desc[6 * h + 4];
	}
	return pool;
}

REF_API void refh_destroy(void* p)
{
	delete (HullPool*)p;
}

// ---------------------------------------------------------------------------
// Shapes from fixture parameters.
//   type 0 sphere:   p[0..2] center, p[3] radius
//   type 1 capsule:  p[0..2] vertex1, p[3..5] vertex2, p[6] radius
//   type 2 triangle: p[0..8] vertices, p[9] radius
//   type 3 hull:     p[0] radius (B3_HULL_RADIUS when the shape keeps its default)

struct ShapeStore
{
	b3SphereShape sphere;
	b3CapsuleShape capsule;
	b3TriangleShape triangle;
	b3HullShape hull;
	b3MeshShape mesh;
};

// Wings of a triangle shape: 12 floats (e1, e2, e3 vertices, three flags).
static void SetWings(b3TriangleShape& t, const float* w)
{
	t.m_e1Vertex.Set(w[0], w[1], w[2]);
	t.m_e2Vertex.Set(w[3], w[4], w[5]);
	t.m_e3Vertex.Set(w[6], w[7], w[8]);
	t.m_hasE1Vertex = w[9] != 0.0f;
	t.m_hasE2Vertex = w[10] != 0.0f;
	t.m_hasE3Vertex = w[11] != 0.0f;
}

static const b3Shape* MakeShape(ShapeStore& s, uint32_t type, const float* p, uint32_t hullIndex, const HullPool* pool)
{
	switch (type)
	{
	case 0:
		s.sphere.m_center.Set(p[0], p[1], p[2]);
		s.sphere.m_radius = p[3];
		return &s.sphere;
	case 1:
		s.capsule.m_vertex1.Set(p[0], p[1], p[2]);
		s.capsule.m_vertex2.Set(p[3], p[4], p[5]);
		s.capsule.m_radius = p[6];
		return &s.capsule;
	case 2:
		s.triangle.Set(b3Vec3(p[0], p[1], p[2]), b3Vec3(p[3], p[4], p[5]), b3Vec3(p[6], p[7], p[8]));
		s.triangle.m_radius = p[9];
		return &s.triangle;
	case 3:
		s.hull.m_hull = &pool->hulls[hullIndex];
		s.hull.m_radius = p[0];
		return &s.hull;
	case 4:
		// mesh: p[0..2] scale; the radius stays B3_HULL_RADIUS
		s.mesh.m_mesh = pool->meshes[hullIndex];
		s.mesh.m_scale.Set(p[0], p[1], p[2]);
		return &s.mesh;
	default:
		return nullptr;
	}
}

// ---------------------------------------------------------------------------
// Time of impact and GJK shape cast, the reference's free functions on
// shapes built from fixture parameters (hulls from the pool).

// b3ShapeCast and its output are defined in gjk.cpp (gjk.cpp:930-942) without
// a header; declared here as they are defined there.
struct b3ShapeCastOutput
{
	scalar t;
	b3Vec3 point;
	b3Vec3 normal;
	uint32 iterations;
};
bool b3ShapeCast(b3ShapeCastOutput* output, const b3Transform& xf1, const b3GJKProxy& proxy1,
	const b3Transform& xf2, const b3GJKProxy& proxy2, const b3Vec3& translation2);

static void SetSweep(b3Sweep& w, const float* s)
{
	w.localCenter.Set(s[0], s[1], s[2]);
	w.orientation0.v.Set(s[3], s[4], s[5]);
	w.orientation0.s = s[6];
	w.worldCenter0.Set(s[7], s[8], s[9]);
	w.t0 = s[10];
	w.orientation.v.Set(s[11], s[12], s[13]);
	w.orientation.s = s[14];
	w.worldCenter.Set(s[15], s[16], s[17]);
}

static void PutTOI(uint32_t* o, const b3TOIOutput& r)
{
	float t = (float)r.t;
	o[0] = (uint32_t)r.state;
	memcpy(o + 1, &t, 4);
	o[2] = r.iterations;
	o[3] = 0;
}

// b3TimeOfImpact(const b3TOIInput&) per query (68 words, the b3g_toi_input
// layout); 4 words out each: state, t bits, iterations, 0.
REF_API void refh_toi(void* hullPool, uint32_t n, const float* q, uint32_t* out)
{
	const HullPool* pool = (const HullPool*)hullPool;
	for (uint32_t i = 0; i < n; ++i)
	{
		const float* r = q + 68 * (size_t)i;
		uint32_t w[4];
		memcpy(w, r, 16);
		ShapeStore sa, sb;
		const b3Shape* a = MakeShape(sa, w[0], r + 4, w[1], pool);
		const b3Shape* b = MakeShape(sb, w[2], r + 16, w[3], pool);
		b3TOIInput in;
		in.proxy1.Set(a, 0);
		in.proxy2.Set(b, 0);
		SetSweep(in.sweep1, r + 28);
		SetSweep(in.sweep2, r + 46);
		in.tMax = r[64];
		PutTOI(out + 4 * (size_t)i, b3TimeOfImpact(in));
	}
}

// b3TimeOfImpact(aabb1, d1, aabb2, d2) per query (18 floats).
REF_API void refh_toi_aabb(uint32_t n, const float* q, uint32_t* out)
{
	for (uint32_t i = 0; i < n; ++i)
	{
		const float* r = q + 18 * (size_t)i;
		b3AABB a, b;
		a.lowerBound.Set(r[0], r[1], r[2]);
		a.upperBound.Set(r[3], r[4], r[5]);
		b.lowerBound.Set(r[9], r[10], r[11]);
		b.upperBound.Set(r[12], r[13], r[14]);
		PutTOI(out + 4 * (size_t)i,
			b3TimeOfImpact(a, b3Vec3(r[6], r[7], r[8]), b, b3Vec3(r[15], r[16], r[17])));
	}
}

// b3ShapeCast per query (48 words, the b3g_gjk_cast_input layout); 9 words
// out each: hit, t, point, normal, iterations (zeros without a hit).
REF_API void refh_gjk_cast(void* hullPool, uint32_t n, const float* q, float* out)
{
	const HullPool* pool = (const HullPool*)hullPool;
	for (uint32_t i = 0; i < n; ++i)
	{
		const float* r = q + 48 * (size_t)i;
		uint32_t w[4];
		memcpy(w, r, 16);
		ShapeStore sa, sb;
		const b3Shape* a = MakeShape(sa, w[0], r + 4, w[1], pool);
		const b3Shape* b = MakeShape(sb, w[2], r + 16, w[3], pool);
		b3GJKProxy pa(a, 0), pb(b, 0);
		b3Transform xa, xb;
		xa.translation.Set(r[28], r[29], r[30]);
		xa.rotation.v.Set(r[31], r[32], r[33]);
		xa.rotation.s = r[34];
		xb.translation.Set(r[35], r[36], r[37]);
		xb.rotation.v.Set(r[38], r[39], r[40]);
		xb.rotation.s = r[41];
		b3ShapeCastOutput o;
		bool hit = b3ShapeCast(&o, xa, pa, xb, pb, b3Vec3(r[42], r[43], r[44]));
		float* d = out + 9 * (size_t)i;
		uint32_t h = hit ? 1u : 0u, it = o.iterations;
		memcpy(d, &h, 4);
		d[1] = hit ? (float)o.t : 0.0f;
		d[2] = hit ? (float)o.point.x : 0.0f;
		d[3] = hit ? (float)o.point.y : 0.0f;
		d[4] = hit ? (float)o.point.z : 0.0f;
		d[5] = hit ? (float)o.normal.x : 0.0f;
		d[6] = hit ? (float)o.normal.y : 0.0f;
		d[7] = hit ? (float)o.normal.z : 0.0f;
		memcpy(d + 8, &it, 4);
	}
}

// ---------------------------------------------------------------------------
// World.

// A seeded contact filter (b3ContactFilter, world_callbacks.h:131-138) for
// the filter tests: it rejects a fixture pair when a hash of (smaller index,
// larger index, salt) is 0 modulo `modulus` (0: accept every pair). While
// `log` is on it records the pairs it is asked about, in call order.
static bool filter_rejects(uint32_t ia, uint32_t ib, uint32_t modulus, uint32_t salt)
{
	if (modulus == 0)
		return false;
	uint32_t lo = ia < ib ? ia : ib, hi = ia < ib ? ib : ia;
	uint32_t h = lo * 2654435761u + hi * 40503u + salt * 97u;
	return ((h >> 8) % modulus) == 0;
}

struct HarnessFilter : b3ContactFilter
{
	uint32_t modulus = 0, salt = 0;
	bool log = false;
	std::vector<uint32_t> calls;
	bool ShouldCollide(b3Fixture* a, b3Fixture* b) override
	{
		uint32_t ia = (uint32_t)(uintptr_t)a->GetUserData(), ib = (uint32_t)(uintptr_t)b->GetUserData();
		if (log)
		{
			calls.push_back(ia);
			calls.push_back(ib);
		}
		return !filter_rejects(ia, ib, modulus, salt);
	}
};

struct RefWorld
{
	b3World* world;
	std::vector<b3Body*> bodies;
	std::vector<b3Fixture*> fixtures;
	const HullPool* pool;
	double tFind;
	double tUpdate;
	HarnessFilter* filter = nullptr;
};

// FindNewContacts with the filter's AddPair calls logged.
static void find_new_contacts(RefWorld* w)
{
	if (w->filter)
	{
		w->filter->calls.clear();
		w->filter->log = true;
	}
	w->world->m_contactManager.FindNewContacts();
	if (w->filter)
		w->filter->log = false;
}

static inline double Now()
{
	return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// body_pose: 7 floats per body (position xyz, quaternion xyzw)
// fix_flags: bit0 sensor
REF_API void* refw_create(void* hullPool, uint32_t nb, const uint32_t* bodyType, const float* bodyPose,
	uint32_t nf, const uint32_t* fixBody, const uint32_t* fixType, const uint32_t* fixHull,
	const float* fixParams, const uint32_t* fixFlags, uint32_t warmStarting)
{
	RefWorld* w = new RefWorld;
	w->pool = (const HullPool*)hullPool;
	w->world = new b3World();
	w->world->SetGravity(b3Vec3(0, 0, 0));
	w->world->SetSleeping(false);
	w->world->SetWarmStarting(warmStarting != 0);
	w->tFind = 0;
	w->tUpdate = 0;
	for (uint32_t i = 0; i < nb; ++i)
	{
		b3BodyDef bd;
		bd.type = (b3BodyType)bodyType[i];
		bd.position.Set(bodyPose[7 * i + 0], bodyPose[7 * i + 1], bodyPose[7 * i + 2]);
		bd.orientation.v.Set(bodyPose[7 * i + 3], bodyPose[7 * i + 4], bodyPose[7 * i + 5]);
		bd.orientation.s = bodyPose[7 * i + 6];
		bd.allowSleep = false;
		bd.awake = true;
		w->bodies.push_back(w->world->CreateBody(bd));
	}
	for (uint32_t i = 0; i < nf; ++i)
	{
		ShapeStore store;
		const b3Shape* shape = MakeShape(store, fixType[i], fixParams + 12 * i, fixHull[i], w->pool);
		b3FixtureDef fd;
		fd.shape = shape;
		fd.density = bodyType[fixBody[i]] == e_dynamicBody ? scalar(1) : scalar(0);
		fd.isSensor = (fixFlags[i] & 1) != 0;
		fd.userData = (void*)(uintptr_t)i;
		w->fixtures.push_back(w->bodies[fixBody[i]]->CreateFixture(fd));
	}
	return w;
}

// The device state a GPU contact manager keeps beside the world, in a build
// whose b3ContactManager is the shim of bounce_b200/shim (absent otherwise).
extern "C" void b3g_shim_release(b3ContactManager* cm) __attribute__((weak));

REF_API void refw_destroy(void* p)
{
	RefWorld* w = (RefWorld*)p;
	if (b3g_shim_release)
		b3g_shim_release(&w->world->m_contactManager);
	delete w->world;
	delete w->filter;
	delete w;
}

// A world for whole steps of b3World::Step (the solver, islands and sleep
// included): as refw_create, with gravity, sleeping allowed, and each body's
// linear and angular velocity (6 floats per body).
REF_API void* stepw_create(void* hullPool, uint32_t nb, const uint32_t* bodyType, const float* bodyPose,
	const float* bodyVel, uint32_t nf, const uint32_t* fixBody, const uint32_t* fixType, const uint32_t* fixHull,
	const float* fixParams, const uint32_t* fixFlags, const float* gravity)
{
	RefWorld* w = new RefWorld;
	w->pool = (const HullPool*)hullPool;
	w->world = new b3World();
	w->world->SetGravity(b3Vec3(gravity[0], gravity[1], gravity[2]));
	w->world->SetSleeping(true);
	w->world->SetWarmStarting(true);
	w->tFind = 0;
	w->tUpdate = 0;
	for (uint32_t i = 0; i < nb; ++i)
	{
		b3BodyDef bd;
		bd.type = (b3BodyType)bodyType[i];
		bd.position.Set(bodyPose[7 * i + 0], bodyPose[7 * i + 1], bodyPose[7 * i + 2]);
		bd.orientation.v.Set(bodyPose[7 * i + 3], bodyPose[7 * i + 4], bodyPose[7 * i + 5]);
		bd.orientation.s = bodyPose[7 * i + 6];
		if (bd.type != e_staticBody)
		{
			bd.linearVelocity.Set(bodyVel[6 * i + 0], bodyVel[6 * i + 1], bodyVel[6 * i + 2]);
			bd.angularVelocity.Set(bodyVel[6 * i + 3], bodyVel[6 * i + 4], bodyVel[6 * i + 5]);
		}
		w->bodies.push_back(w->world->CreateBody(bd));
	}
	for (uint32_t i = 0; i < nf; ++i)
	{
		ShapeStore store;
		const b3Shape* shape = MakeShape(store, fixType[i], fixParams + 12 * i, fixHull[i], w->pool);
		b3FixtureDef fd;
		fd.shape = shape;
		fd.density = bodyType[fixBody[i]] == e_dynamicBody ? scalar(1) : scalar(0);
		fd.isSensor = (fixFlags[i] & 1) != 0;
		fd.userData = (void*)(uintptr_t)i;
		w->fixtures.push_back(w->bodies[fixBody[i]]->CreateFixture(fd));
	}
	return w;
}

// One b3World::Step.
REF_API void stepw_step(void* p, float dt, uint32_t velocityIterations, uint32_t positionIterations)
{
	RefWorld* w = (RefWorld*)p;
	w->world->Step(dt, velocityIterations, positionIterations);
}

// Joints with collideConnected = false between body pairs (2 u32 each): a
// b3SphereJoint per pair, which b3Body::ShouldCollide finds in the bodies'
// joint lists (body.cpp:248-260). The collision pass never solves joints.
REF_API void refw_add_joints(void* p, uint32_t n, const uint32_t* pairs)
{
	RefWorld* w = (RefWorld*)p;
	for (uint32_t i = 0; i < n; ++i)
	{
		b3SphereJointDef jd;
		jd.bodyA = w->bodies[pairs[2 * i]];
		jd.bodyB = w->bodies[pairs[2 * i + 1]];
		jd.collideConnected = false;
		w->world->CreateJoint(jd);
	}
}

// Destroys every joint of the world.
REF_API void refw_clear_joints(void* p)
{
	RefWorld* w = (RefWorld*)p;
	while (w->world->GetJointList())
		w->world->DestroyJoint(w->world->GetJointList());
}

// Installs (modulus != 0) or removes the seeded contact filter.
REF_API void refw_set_filter(void* p, uint32_t modulus, uint32_t salt)
{
	RefWorld* w = (RefWorld*)p;
	if (!w->filter)
		w->filter = new HarnessFilter;
	w->filter->modulus = modulus;
	w->filter->salt = salt;
	w->world->SetContactFilter(modulus ? w->filter : nullptr);
}

// The pairs the filter was asked about by AddPair in the last pass, in call
// order (2 u32 each, fixture indices). Returns the number of pairs.
REF_API uint32_t refw_filter_calls(void* p, uint32_t* out, uint32_t capacity)
{
	RefWorld* w = (RefWorld*)p;
	if (!w->filter)
		return 0;
	uint32_t n = (uint32_t)(w->filter->calls.size() / 2);
	for (uint32_t i = 0; i < n && i < capacity; ++i)
	{
		out[2 * i] = w->filter->calls[2 * i];
		out[2 * i + 1] = w->filter->calls[2 * i + 1];
	}
	return n;
}

// The filter's rule, for callers that apply the same filter elsewhere.
REF_API uint32_t ref_filter_rejects(uint32_t ia, uint32_t ib, uint32_t modulus, uint32_t salt)
{
	return filter_rejects(ia, ib, modulus, salt) ? 1u : 0u;
}

// 17 floats per body: xf.translation(3), xf.rotation(xyzw 4), sweep.worldCenter0(3),
// sweep.orientation0(4), sweep.localCenter(3)
REF_API void refw_get_bodies(void* p, float* out)
{
	RefWorld* w = (RefWorld*)p;
	for (size_t i = 0; i < w->bodies.size(); ++i)
	{
		const b3Body* b = w->bodies[i];
		float* o = out + 17 * i;
		o[0] = (float)b->m_xf.translation.x; o[1] = (float)b->m_xf.translation.y; o[2] = (float)b->m_xf.translation.z;
		o[3] = (float)b->m_xf.rotation.v.x; o[4] = (float)b->m_xf.rotation.v.y; o[5] = (float)b->m_xf.rotation.v.z;
		o[6] = (float)b->m_xf.rotation.s;
		o[7] = (float)b->m_sweep.worldCenter0.x; o[8] = (float)b->m_sweep.worldCenter0.y; o[9] = (float)b->m_sweep.worldCenter0.z;
		o[10] = (float)b->m_sweep.orientation0.v.x; o[11] = (float)b->m_sweep.orientation0.v.y;
		o[12] = (float)b->m_sweep.orientation0.v.z; o[13] = (float)b->m_sweep.orientation0.s;
		o[14] = (float)b->m_sweep.localCenter.x; o[15] = (float)b->m_sweep.localCenter.y; o[16] = (float)b->m_sweep.localCenter.z;
	}
}

// 3 floats per body: the centre of mass in body frame. Sets each dynamic
// body's m_sweep.localCenter and its world centres from the current
// transform, as b3Body::ResetMass ends (body.cpp:370-372), so that a caller
// whose scene computed the centres itself drives the reference's sweeps with
// the same transforms. Mass and inertia stay as the reference computed them
// (the collision pass reads neither).
REF_API void refw_set_local_centers(void* p, const float* lc)
{
	RefWorld* w = (RefWorld*)p;
	for (size_t i = 0; i < w->bodies.size(); ++i)
	{
		b3Body* b = w->bodies[i];
		if (b->m_type != e_dynamicBody)
			continue;
		b->m_sweep.localCenter.Set(lc[3 * i + 0], lc[3 * i + 1], lc[3 * i + 2]);
		b->m_sweep.worldCenter = b3Mul(b->m_xf, b->m_sweep.localCenter);
		b->m_sweep.worldCenter0 = b->m_sweep.worldCenter;
	}
}

// 14 floats per body: worldCenter0(3), orientation0(4), worldCenter(3), orientation(4).
// Static bodies are skipped (their sweep never changes in the reference).
REF_API void refw_set_sweeps(void* p, const float* in)
{
	RefWorld* w = (RefWorld*)p;
	for (size_t i = 0; i < w->bodies.size(); ++i)
	{
		b3Body* b = w->bodies[i];
		if (b->m_type == e_staticBody)
			continue;
		const float* s = in + 14 * i;
		b->m_sweep.worldCenter0.Set(s[0], s[1], s[2]);
		b->m_sweep.orientation0.v.Set(s[3], s[4], s[5]);
		b->m_sweep.orientation0.s = s[6];
		b->m_sweep.worldCenter.Set(s[7], s[8], s[9]);
		b->m_sweep.orientation.v.Set(s[10], s[11], s[12]);
		b->m_sweep.orientation.s = s[13];
		b->SynchronizeTransform();
	}
}

// Awake flags per body (1 awake, 0 asleep).
REF_API void refw_set_awake(void* p, const uint8_t* awake)
{
	RefWorld* w = (RefWorld*)p;
	for (size_t i = 0; i < w->bodies.size(); ++i)
	{
		b3Body* b = w->bodies[i];
		if (awake[i])
			b->m_flags |= b3Body::e_awakeFlag;
		else
			b->m_flags &= ~b3Body::e_awakeFlag;
	}
}

REF_API void refw_set_convex_cache(uint32_t on)
{
	b3_convexCache = on != 0;
}

// The first collision pass of a fresh world: b3World::Step(0, ...) runs
// FindNewContacts (m_newContacts is set by CreateFixture) then UpdateContacts.
REF_API void refw_first_pass(void* p, double* times)
{
	RefWorld* w = (RefWorld*)p;
	double t0 = Now();
	if (w->world->m_newContacts)
	{
		find_new_contacts(w);
		w->world->m_newContacts = false;
	}
	double t1 = Now();
	w->world->m_contactManager.UpdateContacts();
	double t2 = Now();
	times[0] = t1 - t0;
	times[1] = t2 - t1;
}

// One later collision pass after the driver has moved the bodies: the
// "Find New Pairs" block of b3World::Solve, then the next step's UpdateContacts.
REF_API void refw_pass(void* p, double* times)
{
	RefWorld* w = (RefWorld*)p;
	b3World* world = w->world;
	double t0 = Now();
	for (b3Body* b = world->m_bodyList; b; b = b->m_next)
	{
		if (b->GetType() == e_staticBody)
			continue;
		if (!b->IsAwake())
			continue;
		b->SynchronizeFixtures();
	}
	world->m_contactManager.SynchronizeFixtures();
	find_new_contacts(w);
	double t1 = Now();
	world->m_contactManager.UpdateContacts();
	double t2 = Now();
	times[0] = t1 - t0;
	times[1] = t2 - t1;
}

// A pass in which some bodies fall asleep at the end of the solve that moved
// them (b3Island::Solve puts an island to sleep after integrating it,
// island.cpp:297-305, and b3World::Solve still synchronises its fixtures,
// world.cpp:424-449): the bodies flagged in `moved`
// are synchronised, pairs are found, then the awake flags become `awake` and
// UpdateContacts runs.
REF_API void refw_pass_sleep(void* p, const uint8_t* moved, const uint8_t* awake, double* times)
{
	RefWorld* w = (RefWorld*)p;
	b3World* world = w->world;
	double t0 = Now();
	for (size_t i = 0; i < w->bodies.size(); ++i)
	{
		b3Body* b = w->bodies[i];
		if (b->GetType() != e_staticBody && moved[i])
			b->SynchronizeFixtures();
	}
	world->m_contactManager.SynchronizeFixtures();
	find_new_contacts(w);
	refw_set_awake(p, awake);
	double t1 = Now();
	world->m_contactManager.UpdateContacts();
	double t2 = Now();
	times[0] = t1 - t0;
	times[1] = t2 - t1;
}

// Edge wings of triangle fixtures (12 floats per listed fixture).
REF_API void refw_set_triangle_wings(void* p, uint32_t n, const uint32_t* fixture, const float* wings)
{
	RefWorld* w = (RefWorld*)p;
	for (uint32_t i = 0; i < n; ++i)
	{
		b3Fixture* f = w->fixtures[fixture[i]];
		if (f->GetType() == b3Shape::e_triangle)
			SetWings(*(b3TriangleShape*)f->GetShape(), wings + 12 * (size_t)i);
	}
}

// Awake flags per body (1 awake, 0 asleep).
REF_API void refw_get_awake(void* p, uint8_t* out)
{
	RefWorld* w = (RefWorld*)p;
	for (size_t i = 0; i < w->bodies.size(); ++i)
		out[i] = w->bodies[i]->IsAwake() ? 1 : 0;
}

REF_API uint32_t refw_contact_count(void* p)
{
	return ((RefWorld*)p)->world->m_contactManager.m_contactCount;
}

REF_API uint32_t refw_touching_count(void* p, uint32_t* manifolds, uint32_t* points)
{
	RefWorld* w = (RefWorld*)p;
	uint32_t touching = 0, nm = 0, np = 0;
	for (b3Contact* c = w->world->m_contactManager.m_contactList; c; c = c->m_next)
	{
		if (c->IsTouching())
			++touching;
		for (uint32 i = 0; i < c->m_manifoldCount; ++i)
		{
			if (c->m_manifolds[i].pointCount > 0)
			{
				++nm;
				np += c->m_manifolds[i].pointCount;
			}
		}
	}
	if (manifolds) *manifolds = nm;
	if (points) *points = np;
	return touching;
}

// Fat AABBs of every fixture proxy, 6 floats each (lower xyz, upper xyz).
REF_API void refw_fat_aabbs(void* p, float* out)
{
	RefWorld* w = (RefWorld*)p;
	const b3BroadPhase& bp = w->world->m_contactManager.m_broadPhase;
	for (size_t i = 0; i < w->fixtures.size(); ++i)
	{
		const b3AABB& a = bp.GetFatAABB(w->fixtures[i]->m_proxyId);
		out[6 * i + 0] = (float)a.lowerBound.x; out[6 * i + 1] = (float)a.lowerBound.y; out[6 * i + 2] = (float)a.lowerBound.z;
		out[6 * i + 3] = (float)a.upperBound.x; out[6 * i + 4] = (float)a.upperBound.y; out[6 * i + 5] = (float)a.upperBound.z;
	}
}

REF_API void refw_proxy_ids(void* p, uint32_t* out)
{
	RefWorld* w = (RefWorld*)p;
	for (size_t i = 0; i < w->fixtures.size(); ++i)
		out[i] = w->fixtures[i]->m_proxyId;
}

static void DumpOne(DumpContact* d, const b3Contact* c)
{
	memset(d, 0, sizeof(DumpContact));
	d->fixtureA = (uint32_t)(uintptr_t)c->m_fixtureA->m_userData;
	d->fixtureB = (uint32_t)(uintptr_t)c->m_fixtureB->m_userData;
	d->flags = c->IsTouching() ? 1 : 0;
	d->manifoldCount = c->m_manifoldCount;
	d->cache[0] = d->cache[1] = d->cache[2] = d->cache[3] = 0xFFFFFFFFu;
	if (c->m_fixtureA->GetType() == b3Shape::e_hull && c->m_fixtureB->GetType() == b3Shape::e_hull)
	{
		const b3HullContact* hc = (const b3HullContact*)c;
		d->cache[0] = (uint32_t)hc->m_cache.cacheType;
		d->cache[1] = (uint32_t)hc->m_cache.featureType;
		d->cache[2] = hc->m_cache.index1;
		d->cache[3] = hc->m_cache.index2;
	}
	for (uint32 i = 0; i < c->m_manifoldCount && i < 3; ++i)
		DumpM(d->manifolds + i, c->m_manifolds[i]);
}

// Pairs in contact-list order: 3 u32 per contact (fixtureA, fixtureB, flags | manifoldCount << 8).
REF_API uint32_t refw_dump_pairs(void* p, uint32_t* out)
{
	RefWorld* w = (RefWorld*)p;
	uint32_t n = 0;
	for (b3Contact* c = w->world->m_contactManager.m_contactList; c; c = c->m_next, ++n)
	{
		out[3 * n + 0] = (uint32_t)(uintptr_t)c->m_fixtureA->m_userData;
		out[3 * n + 1] = (uint32_t)(uintptr_t)c->m_fixtureB->m_userData;
		out[3 * n + 2] = (c->IsTouching() ? 1u : 0u) | (c->m_manifoldCount << 8);
	}
	return n;
}

// Full records for contacts [start, start + count) of the contact list.
REF_API uint32_t refw_dump_contacts(void* p, uint32_t start, uint32_t count, void* out)
{
	RefWorld* w = (RefWorld*)p;
	uint32_t i = 0, n = 0;
	for (b3Contact* c = w->world->m_contactManager.m_contactList; c && n < count; c = c->m_next, ++i)
	{
		if (i < start)
			continue;
		DumpOne((DumpContact*)out + n, c);
		++n;
	}
	return n;
}

// Overwrite the warm-start state of every contact's manifolds (as the solver
// would leave it): per contact in list order, per manifold point, the normal
// impulse; per manifold the tangent and motor impulses. Records as dumped.
REF_API void refw_load_impulses(void* p, const void* in)
{
	RefWorld* w = (RefWorld*)p;
	const DumpContact* d = (const DumpContact*)in;
	for (b3Contact* c = w->world->m_contactManager.m_contactList; c; c = c->m_next, ++d)
	{
		for (uint32 i = 0; i < c->m_manifoldCount && i < 3; ++i)
		{
			b3Manifold& m = c->m_manifolds[i];
			m.tangentImpulse.x = (scalar)d->manifolds[i].tangentImpulse[0];
			m.tangentImpulse.y = (scalar)d->manifolds[i].tangentImpulse[1];
			m.motorImpulse = (scalar)d->manifolds[i].motorImpulse;
			for (uint32 k = 0; k < m.pointCount && k < 4; ++k)
				m.points[k].normalImpulse = (scalar)d->manifolds[i].points[k].normalImpulse;
		}
	}
}

// b3CollideHulls call and feature-cache hit counters (collide_hulls.cpp:28),
// read and reset.
extern uint32 b3_convexCalls, b3_convexCacheHits;
REF_API void refw_convex_stats(uint32_t* out)
{
	out[0] = b3_convexCalls;
	out[1] = b3_convexCacheHits;
	b3_convexCalls = 0;
	b3_convexCacheHits = 0;
}

// Each fixture's contact edges (b3Fixture::m_contactList) in list order:
// offsets (fixture count + 1) and the (fixtureA, fixtureB) of every edge's
// contact; returns the number of edges.
REF_API uint32_t refw_fixture_edges(void* p, uint32_t* offsets, uint32_t* pairs, uint32_t cap)
{
	RefWorld* w = (RefWorld*)p;
	uint32_t k = 0;
	for (size_t i = 0; i < w->fixtures.size(); ++i)
	{
		offsets[i] = k;
		for (b3ContactEdge* ce = w->fixtures[i]->m_contactList; ce; ce = ce->next, ++k)
		{
			if (k < cap)
			{
				pairs[2 * k] = (uint32_t)(uintptr_t)ce->contact->m_fixtureA->m_userData;
				pairs[2 * k + 1] = (uint32_t)(uintptr_t)ce->contact->m_fixtureB->m_userData;
			}
		}
	}
	offsets[w->fixtures.size()] = k;
	return k;
}

static inline void PutF(uint32_t* o, scalar x)
{
	float f = (float)x;
	memcpy(o, &f, 4);
}

static inline void PutV(uint32_t* o, const b3Vec3& v)
{
	PutF(o, v.x);
	PutF(o + 1, v.y);
	PutF(o + 2, v.z);
}

static inline void PutM(uint32_t* o, const b3Mat33& m)
{
	PutV(o, m.x);
	PutV(o + 3, m.y);
	PutV(o + 6, m.z);
}

// The reference's b3ContactSolver constructor and InitializeVelocityConstraints
// (contact_solver.cpp:28-149, :177-305) on this world's contacts: the listed
// contact-list positions (count of them) or, with list null, every touching
// contact without a sensor fixture, in list order (the filter of
// b3World::Solve, world.cpp:336-348). bodies: 28 floats per body (x, q, v, w,
// invMass, localCenter, I columns, pad) becoming b3Position / b3Velocity
// entries at island index = body index and the body's m_invMass and
// m_sweep.localCenter (restored afterwards); friction and restitution per
// fixture are set on the fixtures. Writes 32 words per constraint and 116
// per manifold (the records of include/b3g.h); tangents of manifolds without
// points, which the reference leaves unset, are written as zero. Returns the
// constraint count; *manifoldCount receives the manifold count and, when
// seconds is not null, *seconds the time of the constructor and
// InitializeVelocityConstraints alone.
REF_API uint32_t refw_contact_solver(void* p, uint32_t count, const uint32_t* list, const float* bodies,
	const float* friction, const float* restitution, float dtRatio, uint32_t warm, uint32_t* conOut,
	uint32_t* manOut, uint32_t* manifoldCount, double* seconds)
{
	RefWorld* w = (RefWorld*)p;
	std::vector<b3Contact*> all;
	for (b3Contact* c = w->world->m_contactManager.m_contactList; c; c = c->m_next)
		all.push_back(c);
	std::vector<b3Contact*> sel;
	std::vector<uint32_t> selIndex;
	if (list)
	{
		for (uint32_t i = 0; i < count; ++i)
		{
			sel.push_back(all[list[i]]);
			selIndex.push_back(list[i]);
		}
	}
	else
	{
		for (size_t i = 0; i < all.size(); ++i)
		{
			b3Contact* c = all[i];
			if (!c->IsTouching() || c->m_fixtureA->m_isSensor || c->m_fixtureB->m_isSensor)
				continue;
			sel.push_back(c);
			selIndex.push_back((uint32_t)i);
		}
	}
	for (size_t i = 0; i < w->fixtures.size(); ++i)
	{
		w->fixtures[i]->m_friction = friction[i];
		w->fixtures[i]->m_restitution = restitution[i];
	}
	const size_t nb = w->bodies.size();
	std::vector<b3Position> pos(nb);
	std::vector<b3Velocity> vel(nb);
	std::vector<scalar> savedMass(nb);
	std::vector<b3Vec3> savedCenter(nb);
	for (size_t i = 0; i < nb; ++i)
	{
		b3Body* b = w->bodies[i];
		const float* r = bodies + 28 * i;
		savedMass[i] = b->m_invMass;
		savedCenter[i] = b->m_sweep.localCenter;
		b->m_islandIndex = (uint32)i;
		b->m_invMass = r[13];
		b->m_sweep.localCenter.Set(r[14], r[15], r[16]);
		pos[i].x.Set(r[0], r[1], r[2]);
		pos[i].q.v.Set(r[3], r[4], r[5]);
		pos[i].q.s = r[6];
		pos[i].I = b3Mat33(b3Vec3(r[17], r[18], r[19]), b3Vec3(r[20], r[21], r[22]), b3Vec3(r[23], r[24], r[25]));
		vel[i].v.Set(r[7], r[8], r[9]);
		vel[i].w.Set(r[10], r[11], r[12]);
	}
	b3TimeStep step;
	step.dt = scalar(1) / scalar(60);
	step.inv_dt = scalar(60);
	step.dtRatio = dtRatio;
	step.velocityIterations = 8;
	step.positionIterations = 2;
	step.warmStarting = warm != 0;
	b3ContactSolverDef def;
	def.step = step;
	def.contacts = sel.data();
	def.count = (uint32)sel.size();
	def.positions = pos.data();
	def.velocities = vel.data();
	def.allocator = &w->world->m_stackAllocator;
	uint32_t mk = 0;
	{
		double t0 = Now();
		b3ContactSolver solver(&def);
		solver.InitializeVelocityConstraints();
		if (seconds)
			*seconds = Now() - t0;
		for (uint32_t i = 0; i < def.count; ++i)
		{
			const b3ContactVelocityConstraint& vc = solver.m_velocityConstraints[i];
			const b3ContactPositionConstraint& pc = solver.m_positionConstraints[i];
			uint32_t* o = conOut + 32 * (size_t)i;
			memset(o, 0, 128);
			o[0] = vc.indexA;
			o[1] = vc.indexB;
			o[2] = mk;
			o[3] = vc.manifoldCount;
			PutF(o + 4, vc.invMassA);
			PutF(o + 5, vc.invMassB);
			PutF(o + 6, vc.friction);
			PutF(o + 7, vc.restitution);
			PutM(o + 8, vc.invIA);
			PutM(o + 17, vc.invIB);
			PutF(o + 26, pc.radiusA);
			PutF(o + 27, pc.radiusB);
			o[28] = selIndex[i];
			for (uint32_t j = 0; j < vc.manifoldCount; ++j, ++mk)
			{
				const b3VelocityConstraintManifold& vm = vc.manifolds[j];
				const b3PositionConstraintManifold& pm = pc.manifolds[j];
				uint32_t* m = manOut + 116 * (size_t)mk;
				memset(m, 0, 464);
				PutV(m, vm.rA);
				PutV(m + 3, vm.rB);
				PutV(m + 6, vm.normal);
				if (vm.pointCount > 0)
				{
					PutV(m + 9, vm.tangent1);
					PutV(m + 12, vm.tangent2);
				}
				PutF(m + 15, vm.tangentSpeed1);
				PutF(m + 16, vm.tangentSpeed2);
				PutF(m + 17, vm.tangentMass.x.x);
				PutF(m + 18, vm.tangentMass.x.y);
				PutF(m + 19, vm.tangentMass.y.x);
				PutF(m + 20, vm.tangentMass.y.y);
				PutF(m + 21, vm.tangentImpulse.x);
				PutF(m + 22, vm.tangentImpulse.y);
				PutF(m + 23, vm.motorImpulse);
				PutF(m + 24, vm.motorMass);
				PutF(m + 25, vm.motorSpeed);
				m[26] = vm.pointCount;
				m[27] = i;
				for (uint32_t k = 0; k < vm.pointCount && k < 4; ++k)
				{
					const b3VelocityConstraintPoint& vp = vm.points[k];
					uint32_t* q = m + 32 + 12 * k;
					PutV(q, vp.rA);
					PutV(q + 3, vp.rB);
					PutV(q + 6, vp.normal);
					PutF(q + 9, vp.normalMass);
					PutF(q + 10, vp.normalImpulse);
					PutF(q + 11, vp.velocityBias);
					const b3PositionConstraintPoint& pp = pm.points[k];
					uint32_t* r = m + 80 + 9 * k;
					PutV(r, pp.localNormalA);
					PutV(r + 3, pp.localPointA);
					PutV(r + 6, pp.localPointB);
				}
			}
		}
	}
	for (size_t i = 0; i < nb; ++i)
	{
		w->bodies[i]->m_invMass = savedMass[i];
		w->bodies[i]->m_sweep.localCenter = savedCenter[i];
	}
	*manifoldCount = mk;
	return (uint32_t)sel.size();
}

// Mass data of every body as the reference computed it from its fixtures
// (b3Body::ResetMassData): 1 + 9 + 9 floats per body, m_invMass, m_invI and
// m_worldInvI (columns x, y, z).
REF_API void refw_mass_data(void* p, float* out)
{
	RefWorld* w = (RefWorld*)p;
	for (size_t i = 0; i < w->bodies.size(); ++i)
	{
		const b3Body* b = w->bodies[i];
		float* o = out + 19 * i;
		o[0] = (float)b->m_invMass;
		const b3Mat33* m[2] = {&b->m_invI, &b->m_worldInvI};
		for (int k = 0; k < 2; ++k)
		{
			const b3Vec3* col[3] = {&m[k]->x, &m[k]->y, &m[k]->z};
			for (int c = 0; c < 3; ++c)
			{
				o[1 + 9 * k + 3 * c] = (float)col[c]->x;
				o[2 + 9 * k + 3 * c] = (float)col[c]->y;
				o[3 + 9 * k + 3 * c] = (float)col[c]->z;
			}
		}
	}
}

// World queries through the reference's own b3World entry points.
struct QueryAll : b3QueryListener, b3QueryFilter
{
	std::vector<uint32_t> found;
	bool ReportFixture(b3Fixture* f) override
	{
		found.push_back((uint32_t)(uintptr_t)f->GetUserData());
		return true;
	}
	bool ShouldReport(b3Fixture*) override { return true; }
};

// b3World::QueryAABB with a listener that accepts every fixture; writes up
// to cap fixture indices (report order) and returns their number.
REF_API uint32_t refw_query_aabb(void* p, const float* box, uint32_t* out, uint32_t cap)
{
	RefWorld* w = (RefWorld*)p;
	QueryAll q;
	b3AABB a;
	a.lowerBound.Set(box[0], box[1], box[2]);
	a.upperBound.Set(box[3], box[4], box[5]);
	w->world->QueryAABB(&q, &q, a);
	for (uint32_t i = 0; i < q.found.size() && i < cap; ++i)
		out[i] = q.found[i];
	return (uint32_t)q.found.size();
}

struct RayAll : b3RayCastListener, b3RayCastFilter
{
	std::vector<uint32_t> fix;
	std::vector<double> hit;
	scalar ReportFixture(b3Fixture* f, const b3Vec3& point, const b3Vec3& normal, scalar fraction) override
	{
		fix.push_back((uint32_t)(uintptr_t)f->GetUserData());
		double h[7] = {(double)point.x, (double)point.y, (double)point.z, (double)normal.x, (double)normal.y,
			(double)normal.z, (double)fraction};
		hit.insert(hit.end(), h, h + 7);
		return scalar(1);
	}
	bool ShouldRayCast(b3Fixture*) override { return true; }
};

// b3World::RayCast with a listener that keeps every hit (returns 1): up to
// cap hits as fixture + (point, normal, fraction); returns the hit count.
REF_API uint32_t refw_ray_cast(void* p, const float* ray, uint32_t* fix, double* hit, uint32_t cap)
{
	RefWorld* w = (RefWorld*)p;
	RayAll r;
	w->world->RayCast(&r, &r, b3Vec3(ray[0], ray[1], ray[2]), b3Vec3(ray[3], ray[4], ray[5]));
	for (uint32_t i = 0; i < r.fix.size() && i < cap; ++i)
	{
		fix[i] = r.fix[i];
		for (int k = 0; k < 7; ++k)
			hit[7 * i + k] = r.hit[7 * i + k];
	}
	return (uint32_t)r.fix.size();
}

// b3World::RayCastSingle: 1 and the closest hit, or 0.
REF_API uint32_t refw_ray_cast_single(void* p, const float* ray, uint32_t* fix, double* hit)
{
	RefWorld* w = (RefWorld*)p;
	RayAll filter;
	b3RayCastSingleOutput o;
	if (!w->world->RayCastSingle(&o, &filter, b3Vec3(ray[0], ray[1], ray[2]), b3Vec3(ray[3], ray[4], ray[5])))
		return 0;
	*fix = (uint32_t)(uintptr_t)o.fixture->GetUserData();
	double h[7] = {(double)o.point.x, (double)o.point.y, (double)o.point.z, (double)o.normal.x, (double)o.normal.y,
		(double)o.normal.z, (double)o.fraction};
	for (int k = 0; k < 7; ++k)
		hit[k] = h[k];
	return 1;
}

// Timed batch of b3World::RayCastSingle calls (the CPU baseline of the ray
// cast bench): n rays (6 floats each); writes each ray's fixture (or
// 0xFFFFFFFF) and returns the seconds spent in the calls.
REF_API double refw_ray_cast_single_batch(void* p, const float* rays, uint32_t n, uint32_t* fix)
{
	RefWorld* w = (RefWorld*)p;
	RayAll filter;
	double t0 = Now();
	for (uint32_t i = 0; i < n; ++i)
	{
		const float* r = rays + 6 * (size_t)i;
		b3RayCastSingleOutput o;
		bool hit = w->world->RayCastSingle(&o, &filter, b3Vec3(r[0], r[1], r[2]), b3Vec3(r[3], r[4], r[5]));
		fix[i] = hit ? (uint32_t)(uintptr_t)o.fixture->GetUserData() : 0xFFFFFFFFu;
	}
	return Now() - t0;
}

// Shape casts through b3World::ShapeCast / ShapeCastSingle. A cast is 28
// words in the b3g_shape_cast_input layout: type, hull, world, pad,
// params[12], position[3], rotation[4], displacement[3], pad[2].
struct CastAll : b3ShapeCastListener, b3ShapeCastFilter
{
	std::vector<uint32_t> fix;
	std::vector<double> hit;
	scalar ReportFixture(b3Fixture* f, const b3Vec3& point, const b3Vec3& normal, scalar fraction) override
	{
		fix.push_back((uint32_t)(uintptr_t)f->GetUserData());
		double h[7] = {(double)point.x, (double)point.y, (double)point.z, (double)normal.x, (double)normal.y,
			(double)normal.z, (double)fraction};
		hit.insert(hit.end(), h, h + 7);
		return scalar(1);
	}
	bool ShouldShapeCast(b3Fixture*) override { return true; }
};

static const b3Shape* CastShape(ShapeStore& store, const RefWorld* w, const float* cast)
{
	uint32_t type, hull;
	memcpy(&type, cast, 4);
	memcpy(&hull, cast + 1, 4);
	return MakeShape(store, type, cast + 4, hull, w->pool);
}

static b3Transform CastXf(const float* cast)
{
	b3Transform xf;
	xf.translation.Set(cast[16], cast[17], cast[18]);
	xf.rotation.v.Set(cast[19], cast[20], cast[21]);
	xf.rotation.s = cast[22];
	return xf;
}

// b3World::ShapeCast with a listener that returns 1 (keeps every hit): up to
// cap hits as fixture + (point, normal, fraction); returns the hit count.
REF_API uint32_t refw_shape_cast(void* p, const float* cast, uint32_t* fix, double* hit, uint32_t cap)
{
	RefWorld* w = (RefWorld*)p;
	ShapeStore store;
	const b3Shape* shape = CastShape(store, w, cast);
	CastAll all;
	w->world->ShapeCast(&all, &all, shape, CastXf(cast), b3Vec3(cast[23], cast[24], cast[25]));
	uint32_t n = (uint32_t)all.fix.size();
	for (uint32_t i = 0; i < n && i < cap; ++i)
	{
		fix[i] = all.fix[i];
		for (int k = 0; k < 7; ++k)
			hit[7 * i + k] = all.hit[7 * i + k];
	}
	return n;
}

// b3World::ShapeCastSingle: 1 and the closest hit, or 0.
REF_API uint32_t refw_shape_cast_single(void* p, const float* cast, uint32_t* fix, double* hit)
{
	RefWorld* w = (RefWorld*)p;
	ShapeStore store;
	const b3Shape* shape = CastShape(store, w, cast);
	CastAll filter;
	b3ShapeCastSingleOutput o;
	if (!w->world->ShapeCastSingle(&o, &filter, shape, CastXf(cast), b3Vec3(cast[23], cast[24], cast[25])))
		return 0;
	*fix = (uint32_t)(uintptr_t)o.fixture->GetUserData();
	double h[7] = {(double)o.point.x, (double)o.point.y, (double)o.point.z, (double)o.normal.x, (double)o.normal.y,
		(double)o.normal.z, (double)o.fraction};
	for (int k = 0; k < 7; ++k)
		hit[k] = h[k];
	return 1;
}

// Timed batch of b3World::ShapeCastSingle calls (the CPU baseline of the
// shape cast bench): writes each cast's fixture (or 0xFFFFFFFF) and returns
// the seconds spent in the calls; frac (may be null) receives each hit's
// fraction (0 without a hit).
REF_API double refw_shape_cast_single_batch(void* p, const float* casts, uint32_t n, uint32_t* fix, float* frac)
{
	RefWorld* w = (RefWorld*)p;
	std::vector<ShapeStore> stores(n);
	std::vector<const b3Shape*> shapes(n);
	for (uint32_t i = 0; i < n; ++i)
		shapes[i] = CastShape(stores[i], w, casts + 28 * (size_t)i);
	CastAll filter;
	double t0 = Now();
	for (uint32_t i = 0; i < n; ++i)
	{
		const float* c = casts + 28 * (size_t)i;
		b3ShapeCastSingleOutput o;
		bool hit = w->world->ShapeCastSingle(&o, &filter, shapes[i], CastXf(c), b3Vec3(c[23], c[24], c[25]));
		fix[i] = hit ? (uint32_t)(uintptr_t)o.fixture->GetUserData() : 0xFFFFFFFFu;
		if (frac)
			frac[i] = hit ? (float)o.fraction : 0.0f;
	}
	return Now() - t0;
}

// Layout of b3ManifoldPoint / b3Manifold (collision.h:97-128) for checking the
// device records: sizes and field offsets.
REF_API void ref_manifold_layout(uint32_t* out)
{
	out[0] = (uint32_t)sizeof(b3ManifoldPoint);
	out[1] = (uint32_t)offsetof(b3ManifoldPoint, localNormal1);
	out[2] = (uint32_t)offsetof(b3ManifoldPoint, localPoint1);
	out[3] = (uint32_t)offsetof(b3ManifoldPoint, localPoint2);
	out[4] = (uint32_t)offsetof(b3ManifoldPoint, normalImpulse);
	out[5] = (uint32_t)offsetof(b3ManifoldPoint, id);
	out[6] = (uint32_t)(offsetof(b3ManifoldPoint, id) + offsetof(b3ContactID, key));
	out[7] = (uint32_t)offsetof(b3ManifoldPoint, persisting);
	out[8] = (uint32_t)offsetof(b3ManifoldPoint, edgeContact);
	out[9] = (uint32_t)sizeof(b3Manifold);
	out[10] = (uint32_t)offsetof(b3Manifold, pointCount);
	out[11] = (uint32_t)offsetof(b3Manifold, tangentImpulse);
	out[12] = (uint32_t)offsetof(b3Manifold, motorImpulse);
	out[13] = (uint32_t)offsetof(b3Manifold, motorSpeed);
	out[14] = (uint32_t)offsetof(b3Manifold, tangentSpeed1);
	out[15] = (uint32_t)offsetof(b3Manifold, tangentSpeed2);
}

REF_API uint32_t ref_sizeof_dump_contact() { return (uint32_t)sizeof(DumpContact); }
REF_API uint32_t ref_sizeof_scalar() { return (uint32_t)sizeof(scalar); }

// ---------------------------------------------------------------------------
// Direct calls of the b3Collide* routines (collision.h:152-202) for unit-level
// checks. xf: 7 floats (translation xyz, rotation xyzw). cache4 (hull-hull
// only) is read and written back. xf0 is the previous-step transform used by
// the hull feature cache (hull_contact.cpp:43-44).

static b3Transform MakeXf(const float* x)
{
	b3Transform xf;
	xf.translation.Set(x[0], x[1], x[2]);
	xf.rotation.v.Set(x[3], x[4], x[5]);
	xf.rotation.s = x[6];
	return xf;
}

// As ref_collide, with edge wings for triangle shapes (12 floats each, or NULL).
REF_API int ref_collide_wings(void* hullPool, uint32_t typeA, const float* pA, uint32_t hullA,
	uint32_t typeB, const float* pB, uint32_t hullB, const float* xfA, const float* xfB,
	const float* xf0A, const float* xf0B, uint32_t* cache4, void* out, const float* wingsA, const float* wingsB);

REF_API int ref_collide(void* hullPool, uint32_t typeA, const float* pA, uint32_t hullA,
	uint32_t typeB, const float* pB, uint32_t hullB, const float* xfA, const float* xfB,
	const float* xf0A, const float* xf0B, uint32_t* cache4, void* out)
{
	return ref_collide_wings(hullPool, typeA, pA, hullA, typeB, pB, hullB, xfA, xfB, xf0A, xf0B, cache4, out,
		nullptr, nullptr);
}

REF_API int ref_collide_wings(void* hullPool, uint32_t typeA, const float* pA, uint32_t hullA,
	uint32_t typeB, const float* pB, uint32_t hullB, const float* xfA, const float* xfB,
	const float* xf0A, const float* xf0B, uint32_t* cache4, void* out, const float* wingsA, const float* wingsB)
{
	const HullPool* pool = (const HullPool*)hullPool;
	ShapeStore sa, sb;
	const b3Shape* A = MakeShape(sa, typeA, pA, hullA, pool);
	const b3Shape* B = MakeShape(sb, typeB, pB, hullB, pool);
	if (typeA == 2 && wingsA)
		SetWings(sa.triangle, wingsA);
	if (typeB == 2 && wingsB)
		SetWings(sb.triangle, wingsB);
	b3Transform XA = MakeXf(xfA), XB = MakeXf(xfB);
	b3Manifold m;
	m.Initialize();
	int rc = 0;
	if (typeA == 0 && typeB == 0)
		b3CollideSpheres(m, XA, (const b3SphereShape*)A, XB, (const b3SphereShape*)B);
	else if (typeA == 1 && typeB == 0)
		b3CollideCapsuleAndSphere(m, XA, (const b3CapsuleShape*)A, XB, (const b3SphereShape*)B);
	else if (typeA == 1 && typeB == 1)
		b3CollideCapsules(m, XA, (const b3CapsuleShape*)A, XB, (const b3CapsuleShape*)B);
	else if (typeA == 2 && typeB == 0)
		b3CollideTriangleAndSphere(m, XA, (const b3TriangleShape*)A, XB, (const b3SphereShape*)B);
	else if (typeA == 2 && typeB == 1)
		b3CollideTriangleAndCapsule(m, XA, (const b3TriangleShape*)A, XB, (const b3CapsuleShape*)B);
	else if (typeA == 3 && typeB == 0)
		b3CollideHullAndSphere(m, XA, (const b3HullShape*)A, XB, (const b3SphereShape*)B);
	else if (typeA == 3 && typeB == 1)
		b3CollideHullAndCapsule(m, XA, (const b3HullShape*)A, XB, (const b3CapsuleShape*)B);
	else if (typeA == 3 && typeB == 2)
		b3CollideHullAndTriangle(m, XA, (const b3HullShape*)A, XB, (const b3TriangleShape*)B);
	else if (typeA == 3 && typeB == 3)
	{
		b3FeatureCache cache;
		cache.cacheType = (b3CacheType)cache4[0];
		cache.featureType = (b3FeatureType)cache4[1];
		cache.index1 = cache4[2];
		cache.index2 = cache4[3];
		b3CollideHulls(m, XA, (const b3HullShape*)A, XB, (const b3HullShape*)B, cache, MakeXf(xf0A), MakeXf(xf0B));
		cache4[0] = (uint32_t)cache.cacheType;
		cache4[1] = (uint32_t)cache.featureType;
		cache4[2] = cache.index1;
		cache4[3] = cache.index2;
	}
	else
		rc = -1;
	DumpM((DumpManifold*)out, m);
	return rc;
}

// b3Sweep::GetTransform(0) (sweep.h:43-63) for checking the device's xf0.
REF_API void ref_sweep_xf0(const float* c0, const float* q0, const float* q, const float* lc, float* out)
{
	b3Sweep s;
	s.worldCenter0.Set(c0[0], c0[1], c0[2]);
	s.orientation0.v.Set(q0[0], q0[1], q0[2]);
	s.orientation0.s = q0[3];
	s.worldCenter = s.worldCenter0;
	s.orientation.v.Set(q[0], q[1], q[2]);
	s.orientation.s = q[3];
	s.localCenter.Set(lc[0], lc[1], lc[2]);
	s.t0 = 0;
	b3Transform xf = s.GetTransform(scalar(0));
	out[0] = (float)xf.translation.x; out[1] = (float)xf.translation.y; out[2] = (float)xf.translation.z;
	out[3] = (float)xf.rotation.v.x; out[4] = (float)xf.rotation.v.y; out[5] = (float)xf.rotation.v.z;
	out[6] = (float)xf.rotation.s;
}

// b3ContactManager on the GPU: the member functions of
// include/bounce/dynamics/contact_manager.h implemented with the C ABI of
// libb3g.so (include/b3g.h). A Bounce build compiles this file in place of
// src/bounce/dynamics/contact_manager.cpp and links libb3g.so; nothing else
// of the engine changes. b3World::Step then runs its collision pass on the
// device and its own solver, islands, sleep and joints on the manifolds this
// file writes into the b3Contact objects.
//
// What moves to the device, per b3World::Step:
//  - the fixture sync and fat-AABB update of the "Find New Pairs" block
//    (world.cpp:424-449), FindNewContacts / AddPair (contact_manager.cpp:98-223)
//    and UpdateContacts (:225-287), as one b3g_collide in UpdateContacts:
//    FindNewContacts at the end of a step and UpdateContacts at the start of
//    the next one see the same body transforms, so one pass does both;
//  - the contact list (order included), the fixtures' edge lists, begun and
//    destroyed contacts, touching flags, manifolds with warm-started impulses,
//    and the wake-ups of UpdateContacts.
// The b3Contact objects stay on the host for the solver: created with the
// reference's factory (b3Contact::Create), linked in the device's list order,
// destroyed with b3Contact::Destroy (which makes its own wake-ups), with the
// listener called as b3Contact::Update and Destroy call it.
//
// The host broadphase keeps its proxies (b3Body::SynchronizeFixtures still
// moves them, so b3World's queries keep working); its pair search is not used.
// The scene (hulls, meshes, bodies, fixtures) is uploaded when the number of
// proxies changes, and the contacts then restart from a creation pass; the
// fixtures are found through the broadphase's public QueryAABB. The filters
// are the device's: joints with collideConnected false and the world's
// b3ContactFilter (a round trip per pass when one is set at the first pass).
// b3g_shim_release() frees the device state of a contact manager (call it
// from b3World::~b3World).

#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <unordered_map>
#include <vector>

#include <bounce/bounce.h>
#include <bounce/dynamics/contact_manager.h>
#include <bounce/dynamics/contacts/contact.h>
#include <bounce/dynamics/world_callbacks.h>
#include <bounce/common/profiler.h>

#include "b3g.h"

namespace {

struct Gpu
{
	b3g_ctx* ctx = nullptr;
	bool filterFlag = false;
	// scene as uploaded
	std::vector<b3Fixture*> fixtures; // by device index (proxy id order)
	std::vector<b3Body*> bodies;
	std::unordered_map<const b3Fixture*, uint32_t> fixtureIndex;
	std::unordered_map<const b3Body*, uint32_t> bodyIndex;
	uint32_t proxyCount = 0;
	bool havePass = false;
	bool inPass = false; // UpdateContacts is destroying contacts it tracks itself
	// contacts of the last pass in list order (null: destroyed by the world
	// since), and by fixture pair
	std::vector<b3Contact*> list;
	std::unordered_map<uint64_t, b3Contact*> byPair;
	// per-pass host buffers
	std::vector<float> state;
	std::vector<uint8_t> awake;
	std::vector<uint32_t> records, ended, edgeOffsets, edges;
	std::vector<b3Manifold> manifolds;
	std::vector<uint32_t> touchIndex;
	std::vector<b3Manifold> touchManifolds;
	std::vector<float> normal, tangent, motor, normal2, tangent2, motor2;
};

std::unordered_map<const b3ContactManager*, Gpu*>& table()
{
	static std::unordered_map<const b3ContactManager*, Gpu*> t;
	return t;
}

Gpu& gpu_of(const b3ContactManager* cm)
{
	Gpu*& g = table()[cm];
	if (!g)
		g = new Gpu;
	return *g;
}

inline uint64_t pair_key(uint32_t a, uint32_t b) { return ((uint64_t)a << 32) | b; }

// Every proxy of the broadphase: its fixture.
struct ProxyCollector
{
	const b3BroadPhase* bp;
	std::vector<std::pair<uint32_t, b3Fixture*>> out;
	bool Report(uint32_t proxyId)
	{
		out.push_back({proxyId, (b3Fixture*)bp->GetUserData(proxyId)});
		return true;
	}
};

// The engine has no error returns; a failed device call is a broken
// invariant, reported like the engine's own (B3_ASSERT) and counted.
uint32_t g_failures = 0;
void check(int rc)
{
	if (rc < 0)
		++g_failures;
	B3_ASSERT(rc >= 0);
}

// The world's scene in the C ABI's arrays: hulls (b3Hull), meshes (b3Mesh),
// bodies, fixtures with their proxy ids as keys.
void upload_scene(b3ContactManager* cm, Gpu& g)
{
	ProxyCollector pc;
	pc.bp = &cm->m_broadPhase;
	b3AABB all;
	all.lowerBound.Set(-B3_MAX_SCALAR, -B3_MAX_SCALAR, -B3_MAX_SCALAR);
	all.upperBound.Set(B3_MAX_SCALAR, B3_MAX_SCALAR, B3_MAX_SCALAR);
	cm->m_broadPhase.QueryAABB(&pc, all);
	std::sort(pc.out.begin(), pc.out.end());
	g.fixtures.clear();
	g.bodies.clear();
	g.fixtureIndex.clear();
	g.bodyIndex.clear();
	for (auto& e : pc.out)
	{
		g.fixtureIndex[e.second] = (uint32_t)g.fixtures.size();
		g.fixtures.push_back(e.second);
		b3Body* b = e.second->GetBody();
		if (g.bodyIndex.find(b) == g.bodyIndex.end())
		{
			g.bodyIndex[b] = (uint32_t)g.bodies.size();
			g.bodies.push_back(b);
		}
	}
	const uint32_t nf = (uint32_t)g.fixtures.size(), nb = (uint32_t)g.bodies.size();

	// Shared geometry, each hull and mesh once.
	std::vector<const b3Hull*> hulls;
	std::vector<const b3Mesh*> meshes;
	std::unordered_map<const void*, uint32_t> geom;
	std::vector<uint32_t> fixBody(nf), fixType(nf), fixHull(nf, 0), fixFlags(nf), keys(nf);
	std::vector<float> params(12 * (size_t)nf, 0.0f);
	std::vector<uint32_t> triFix;
	std::vector<float> wings;
	for (uint32_t i = 0; i < nf; ++i)
	{
		b3Fixture* f = g.fixtures[i];
		fixBody[i] = g.bodyIndex[f->GetBody()];
		fixType[i] = (uint32_t)f->GetType();
		fixFlags[i] = f->IsSensor() ? B3G_FIXTURE_SENSOR : 0u;
		keys[i] = pc.out[i].first;
		float* p = params.data() + 12 * (size_t)i;
		const b3Shape* s = f->GetShape();
		switch (f->GetType())
		{
		case b3Shape::e_sphere:
		{
			const b3SphereShape* sp = (const b3SphereShape*)s;
			p[0] = sp->m_center.x, p[1] = sp->m_center.y, p[2] = sp->m_center.z, p[3] = sp->m_radius;
			break;
		}
		case b3Shape::e_capsule:
		{
			const b3CapsuleShape* cp = (const b3CapsuleShape*)s;
			p[0] = cp->m_vertex1.x, p[1] = cp->m_vertex1.y, p[2] = cp->m_vertex1.z;
			p[3] = cp->m_vertex2.x, p[4] = cp->m_vertex2.y, p[5] = cp->m_vertex2.z, p[6] = cp->m_radius;
			break;
		}
		case b3Shape::e_triangle:
		{
			const b3TriangleShape* tp = (const b3TriangleShape*)s;
			const b3Vec3* v[3] = {&tp->m_vertex1, &tp->m_vertex2, &tp->m_vertex3};
			for (int k = 0; k < 3; ++k)
				p[3 * k] = v[k]->x, p[3 * k + 1] = v[k]->y, p[3 * k + 2] = v[k]->z;
			p[9] = tp->m_radius;
			const b3Vec3* w[3] = {&tp->m_e1Vertex, &tp->m_e2Vertex, &tp->m_e3Vertex};
			const bool has[3] = {tp->m_hasE1Vertex, tp->m_hasE2Vertex, tp->m_hasE3Vertex};
			triFix.push_back(i);
			for (int k = 0; k < 3; ++k)
				wings.push_back(w[k]->x), wings.push_back(w[k]->y), wings.push_back(w[k]->z);
			for (int k = 0; k < 3; ++k)
				wings.push_back(has[k] ? 1.0f : 0.0f);
			break;
		}
		case b3Shape::e_hull:
		{
			const b3HullShape* hp = (const b3HullShape*)s;
			auto it = geom.find(hp->m_hull);
			if (it == geom.end())
			{
				it = geom.emplace(hp->m_hull, (uint32_t)hulls.size()).first;
				hulls.push_back(hp->m_hull);
			}
			fixHull[i] = it->second;
			p[0] = hp->m_radius;
			break;
		}
		case b3Shape::e_mesh:
		{
			const b3MeshShape* mp = (const b3MeshShape*)s;
			auto it = geom.find(mp->m_mesh);
			if (it == geom.end())
			{
				it = geom.emplace(mp->m_mesh, (uint32_t)meshes.size()).first;
				meshes.push_back(mp->m_mesh);
			}
			fixHull[i] = it->second;
			p[0] = mp->m_scale.x, p[1] = mp->m_scale.y, p[2] = mp->m_scale.z, p[3] = mp->m_radius;
			break;
		}
		default:
			break;
		}
	}

	std::vector<uint32_t> desc, edges, faces;
	std::vector<float> verts, planes, centroids;
	for (const b3Hull* h : hulls)
	{
		desc.insert(desc.end(), {(uint32_t)verts.size() / 3, h->vertexCount, (uint32_t)edges.size() / 5, h->edgeCount,
									(uint32_t)faces.size(), h->faceCount});
		for (uint32_t k = 0; k < h->vertexCount; ++k)
			verts.insert(verts.end(), {(float)h->vertices[k].x, (float)h->vertices[k].y, (float)h->vertices[k].z});
		for (uint32_t k = 0; k < h->edgeCount; ++k)
		{
			const b3HalfEdge& e = h->edges[k];
			edges.insert(edges.end(), {(uint32_t)e.origin, (uint32_t)e.twin, (uint32_t)e.face, (uint32_t)e.prev,
										  (uint32_t)e.next});
		}
		for (uint32_t k = 0; k < h->faceCount; ++k)
		{
			faces.push_back((uint32_t)h->faces[k].edge);
			const b3Plane& pl = h->planes[k];
			planes.insert(planes.end(), {(float)pl.normal.x, (float)pl.normal.y, (float)pl.normal.z, (float)pl.offset});
		}
		centroids.insert(centroids.end(), {(float)h->centroid.x, (float)h->centroid.y, (float)h->centroid.z});
	}
	if (!g.ctx)
	{
		b3g_config cfg;
		cfg.max_proxies = nf ? nf : 1;
		cfg.max_contacts = std::max<uint32_t>(1024u, 32u * nf);
		cfg.max_hull_data = 0;
		g.filterFlag = cm->m_contactFilter != nullptr;
		cfg.flags = B3G_FLAG_WARM_STARTING | B3G_FLAG_CONVEX_CACHE | (g.filterFlag ? B3G_FLAG_CONTACT_FILTER : 0u);
		cfg.device = 0;
		check(b3g_create(&cfg, &g.ctx));
	}
	check(b3g_set_hulls(g.ctx, (uint32_t)hulls.size(), desc.data(), verts.data(), edges.data(), faces.data(),
		planes.data(), centroids.data()));
	if (!meshes.empty())
	{
		std::vector<uint32_t> md, mt;
		std::vector<float> mv;
		for (const b3Mesh* m : meshes)
		{
			md.insert(md.end(), {(uint32_t)mv.size() / 3, m->vertexCount, (uint32_t)mt.size() / 3, m->triangleCount});
			for (uint32_t k = 0; k < m->vertexCount; ++k)
				mv.insert(mv.end(), {(float)m->vertices[k].x, (float)m->vertices[k].y, (float)m->vertices[k].z});
			for (uint32_t k = 0; k < m->triangleCount; ++k)
				mt.insert(mt.end(), {m->triangles[k].v1, m->triangles[k].v2, m->triangles[k].v3});
		}
		check(b3g_set_meshes(g.ctx, (uint32_t)meshes.size(), md.data(), mv.data(), mt.data(), 0));
	}
	std::vector<uint32_t> world(nb, 0), type(nb);
	g.awake.assign(nb, 0);
	for (uint32_t b = 0; b < nb; ++b)
	{
		type[b] = (uint32_t)g.bodies[b]->GetType();
		g.awake[b] = g.bodies[b]->IsAwake() ? 1 : 0;
	}
	check(b3g_set_bodies(g.ctx, nb, world.data(), type.data(), g.awake.data()));
	check(b3g_set_fixtures(g.ctx, nf, fixBody.data(), fixType.data(), fixHull.data(), params.data(), fixFlags.data(),
		keys.data()));
	if (!triFix.empty())
		check(b3g_set_triangle_wings(g.ctx, (uint32_t)triFix.size(), triFix.data(), wings.data()));
	g.proxyCount = cm->m_broadPhase.GetProxyCount();
	g.havePass = false;
}

// Joints whose bodies must not collide (b3Body::ShouldCollide, body.cpp:248-260).
void upload_joints(Gpu& g)
{
	std::vector<uint32_t> pairs;
	for (b3Body* b : g.bodies)
		for (const b3JointEdge* je = b->GetJointList(); je; je = je->next)
		{
			auto it = g.bodyIndex.find(je->other);
			uint32_t self = g.bodyIndex[b];
			if (it != g.bodyIndex.end() && !je->joint->GetCollideConnected() && self < it->second)
			{
				pairs.push_back(self);
				pairs.push_back(it->second);
			}
		}
	check(b3g_set_joint_pairs(g.ctx, (uint32_t)(pairs.size() / 2), pairs.empty() ? nullptr : pairs.data()));
}

} // namespace

b3ContactManager::b3ContactManager()
{
	m_contactList = nullptr;
	m_contactCount = 0;
	m_contactListener = nullptr;
	m_contactFilter = nullptr;
	m_allocator = nullptr;
	m_profiler = nullptr;
}

// Pairs come from the device pass; the host broadphase never reports any.
void b3ContactManager::AddPair(void*, void*) {}

// The device pass synchronises mesh contacts' reference AABBs itself.
void b3ContactManager::SynchronizeFixtures() {}

// The pair search runs in the same device pass as UpdateContacts.
void b3ContactManager::FindNewContacts() {}

void b3ContactManager::UpdateContacts()
{
	B3_PROFILE(m_profiler, "Update Contacts");
	Gpu& g = gpu_of(this);
	if (!g.ctx || g.proxyCount != m_broadPhase.GetProxyCount())
	{
		// A changed fixture set: contacts restart from a creation pass.
		g.inPass = true;
		while (m_contactList)
			Destroy(m_contactList);
		g.inPass = false;
		g.list.clear();
		g.byPair.clear();
		upload_scene(this, g);
	}
	const uint32_t nb = (uint32_t)g.bodies.size();
	upload_joints(g);

	// The solver's impulses of the last pass's contacts warm-start this pass.
	if (g.havePass)
	{
		const size_t n = g.list.size();
		g.normal.assign(4 * n, 0.0f);
		g.tangent.assign(2 * n, 0.0f);
		g.motor.assign(n, 0.0f);
		g.normal2.assign(8 * n, 0.0f);
		g.tangent2.assign(4 * n, 0.0f);
		g.motor2.assign(2 * n, 0.0f);
		bool mesh = false;
		for (size_t i = 0; i < n; ++i)
		{
			const b3Contact* c = g.list[i];
			if (!c)
				continue;
			for (uint32_t k = 0; k < c->m_manifoldCount && k < 3; ++k)
			{
				const b3Manifold& m = c->m_manifolds[k];
				float* nn = k == 0 ? &g.normal[4 * i] : &g.normal2[8 * i + 4 * (k - 1)];
				float* tt = k == 0 ? &g.tangent[2 * i] : &g.tangent2[4 * i + 2 * (k - 1)];
				float* mm = k == 0 ? &g.motor[i] : &g.motor2[2 * i + (k - 1)];
				for (uint32_t p = 0; p < 4; ++p)
					nn[p] = (float)m.points[p].normalImpulse;
				tt[0] = (float)m.tangentImpulse.x;
				tt[1] = (float)m.tangentImpulse.y;
				mm[0] = (float)m.motorImpulse;
				mesh |= k > 0;
			}
		}
		check(b3g_load_impulses(g.ctx, g.normal.data(), g.tangent.data(), g.motor.data()));
		if (mesh)
			check(b3g_load_mesh_impulses(g.ctx, g.normal2.data(), g.tangent2.data(), g.motor2.data()));
	}

	// Body state and awake flags (the solver's sleep decisions).
	g.state.resize(17 * (size_t)nb);
	g.awake.resize(nb);
	for (uint32_t b = 0; b < nb; ++b)
	{
		const b3Body* body = g.bodies[b];
		float* s = g.state.data() + 17 * (size_t)b;
		const b3Transform& xf = body->m_xf;
		const b3Sweep& sw = body->m_sweep;
		s[0] = xf.translation.x, s[1] = xf.translation.y, s[2] = xf.translation.z;
		s[3] = xf.rotation.v.x, s[4] = xf.rotation.v.y, s[5] = xf.rotation.v.z, s[6] = xf.rotation.s;
		s[7] = sw.worldCenter0.x, s[8] = sw.worldCenter0.y, s[9] = sw.worldCenter0.z;
		s[10] = sw.orientation0.v.x, s[11] = sw.orientation0.v.y, s[12] = sw.orientation0.v.z;
		s[13] = sw.orientation0.s;
		s[14] = sw.localCenter.x, s[15] = sw.localCenter.y, s[16] = sw.localCenter.z;
		g.awake[b] = body->IsAwake() ? 1 : 0;
	}
	check(b3g_set_awake(g.ctx, g.awake.data()));

	// The world's contact filter, asked as UpdateContacts asks it (every
	// contact of the list) and as AddPair asks it (every new pair).
	if (g.filterFlag && g.havePass)
	{
		std::vector<uint8_t> veto(g.list.size(), 0);
		for (size_t i = 0; i < g.list.size(); ++i)
			veto[i] = g.list[i] && m_contactFilter &&
					  !m_contactFilter->ShouldCollide(g.list[i]->GetFixtureA(), g.list[i]->GetFixtureB());
		check(b3g_set_contact_veto(g.ctx, (uint32_t)veto.size(), veto.empty() ? nullptr : veto.data()));
	}
	check(b3g_collide(g.ctx, g.state.data(), 0, nullptr));
	if (g.filterFlag)
	{
		int n = b3g_fetch_new_pairs(g.ctx, nullptr, 0);
		check(n);
		n = std::max(n, 0);
		std::vector<uint32_t> pairs(2 * (size_t)std::max(n, 1));
		check(b3g_fetch_new_pairs(g.ctx, pairs.data(), (uint32_t)n));
		std::vector<uint8_t> keep((size_t)std::max(n, 1), 1);
		for (int i = 0; i < n; ++i)
			keep[i] = !m_contactFilter ||
					  m_contactFilter->ShouldCollide(g.fixtures[pairs[2 * i]], g.fixtures[pairs[2 * i + 1]]);
		check(b3g_finish_pass(g.ctx, keep.data(), (uint32_t)n));
	}
	b3g_counts cnt;
	memset(&cnt, 0, sizeof(cnt));
	check(b3g_get_counts(g.ctx, &cnt));

	// Destroyed contacts, in the order UpdateContacts destroys them.
	g.ended.resize(3 * (size_t)std::max(cnt.ended, 1u));
	int ne = b3g_fetch_ended(g.ctx, g.ended.data(), cnt.ended);
	check(ne);
	g.inPass = true;
	for (int i = 0; i < ne; ++i)
	{
		auto it = g.byPair.find(pair_key(g.ended[3 * i], g.ended[3 * i + 1]));
		if (it == g.byPair.end())
			continue;
		b3Contact* c = it->second;
		g.byPair.erase(it);
		Destroy(c);
	}
	g.inPass = false;

	// The contact list in the device's order, new contacts from the factory.
	const uint32_t n = cnt.contacts;
	g.records.resize(3 * (size_t)std::max(n, 1u));
	g.manifolds.resize(std::max(n, 1u));
	check(b3g_fetch_contacts(g.ctx, g.records.data(), n));
	check(b3g_fetch_manifolds(g.ctx, g.manifolds.data(), n));
	g.touchIndex.resize(std::max(cnt.manifolds, 1u));
	g.touchManifolds.resize(std::max(cnt.manifolds, 1u));
	int nt = b3g_fetch_touching(g.ctx, g.touchIndex.data(), g.touchManifolds.data(), cnt.manifolds);
	check(nt);
	g.list.resize(n);
	for (uint32_t i = 0; i < n; ++i)
	{
		uint32_t a = g.records[3 * i], b = g.records[3 * i + 1], flags = g.records[3 * i + 2];
		b3Contact*& c = g.byPair[pair_key(a, b)];
		if (!c)
		{
			// The device reports A and B after the factory's swap, so the
			// factory keeps this order (contact.cpp:306-317).
			c = b3Contact::Create(g.fixtures[a], g.fixtures[b], m_allocator);
			B3_ASSERT(c);
			++m_contactCount;
		}
		g.list[i] = c;
		const bool sensor = c->GetFixtureA()->IsSensor() || c->GetFixtureB()->IsSensor();
		const bool wasTouching = (c->m_flags & b3Contact::e_touchingFlag) != 0;
		const bool touching = (flags & 1u) != 0;
		c->m_manifoldCount = (flags >> 8) & 0xFFu;
		if (c->m_manifoldCount > 0)
			c->m_manifolds[0] = g.manifolds[i];
		for (uint32_t k = 1; k < c->m_manifoldCount; ++k)
			c->m_manifolds[k].Initialize();
		if (touching)
			c->m_flags |= b3Contact::e_touchingFlag;
		else
			c->m_flags &= ~b3Contact::e_touchingFlag;
		// b3Contact::Update's wake-up and listener calls (contact.cpp:249-282).
		if (!sensor && touching != wasTouching)
		{
			c->GetFixtureA()->GetBody()->SetAwake(true);
			c->GetFixtureB()->GetBody()->SetAwake(true);
		}
		if (m_contactListener)
		{
			if (!wasTouching && touching)
				m_contactListener->BeginContact(c);
			if (wasTouching && !touching)
				m_contactListener->EndContact(c);
			if (!sensor && touching)
				m_contactListener->PreSolve(c);
		}
	}
	// Manifolds 1 and 2 of mesh contacts (the compact output lists them after
	// manifold 0 of their contact).
	for (int k = 1; k < nt; ++k)
	{
		uint32_t i = g.touchIndex[k];
		uint32_t slot = 0;
		for (int j = k - 1; j >= 0 && g.touchIndex[j] == i; --j)
			++slot;
		if (slot > 0 && slot < g.list[i]->m_manifoldCount)
			g.list[i]->m_manifolds[slot] = g.touchManifolds[k];
	}

	// Relink the contact list and the fixtures' edge lists in the device's order.
	for (uint32_t i = 0; i < n; ++i)
	{
		b3Contact* c = g.list[i];
		c->m_prev = i ? g.list[i - 1] : nullptr;
		c->m_next = i + 1 < n ? g.list[i + 1] : nullptr;
	}
	m_contactList = n ? g.list[0] : nullptr;
	const uint32_t nf = (uint32_t)g.fixtures.size();
	g.edgeOffsets.resize(nf + 1);
	g.edges.resize(2 * (size_t)std::max(n, 1u));
	check(b3g_fetch_fixture_contacts(g.ctx, g.edgeOffsets.data(), g.edges.data(), 2 * n));
	for (uint32_t f = 0; f < nf; ++f)
	{
		b3Fixture* fx = g.fixtures[f];
		b3ContactEdge* prev = nullptr;
		fx->m_contactList = nullptr;
		for (uint32_t e = g.edgeOffsets[f]; e < g.edgeOffsets[f + 1]; ++e)
		{
			b3Contact* c = g.list[g.edges[e]];
			const bool isA = c->GetFixtureA() == fx;
			b3ContactEdge* edge = isA ? &c->m_nodeA : &c->m_nodeB;
			edge->contact = c;
			edge->other = isA ? c->GetFixtureB() : c->GetFixtureA();
			edge->prev = prev;
			edge->next = nullptr;
			if (prev)
				prev->next = edge;
			else
				fx->m_contactList = edge;
			prev = edge;
		}
	}

	// Wake-ups the pass resolved that the calls above did not make (bodies
	// woken through contacts skipped as inactive earlier in the list).
	check(b3g_fetch_awake(g.ctx, g.awake.data(), nb));
	for (uint32_t b = 0; b < nb; ++b)
		if (g.awake[b] && !g.bodies[b]->IsAwake())
			g.bodies[b]->SetAwake(true);
	g.havePass = true;
}

// Destroys a contact: the listener's EndContact, the list surgery, and
// b3Contact::Destroy, which wakes the bodies of a contact with points
// (contact_manager.cpp:229-287, contact.cpp:108-126). Called by the world
// when it destroys a fixture or a body (the contact's slot in the last pass's
// list then warm-starts nothing) and by UpdateContacts for the contacts the
// pass destroyed.
void b3ContactManager::Destroy(b3Contact* c)
{
	auto t = table().find(this);
	if (t != table().end() && !t->second->inPass)
	{
		Gpu& g = *t->second;
		auto a = g.fixtureIndex.find(c->GetFixtureA());
		auto b = g.fixtureIndex.find(c->GetFixtureB());
		if (a != g.fixtureIndex.end() && b != g.fixtureIndex.end())
			g.byPair.erase(pair_key(a->second, b->second));
		std::replace(g.list.begin(), g.list.end(), c, (b3Contact*)nullptr);
	}
	if (m_contactListener && c->IsTouching())
		m_contactListener->EndContact(c);
	if (c->m_prev)
		c->m_prev->m_next = c->m_next;
	if (c->m_next)
		c->m_next->m_prev = c->m_prev;
	if (c == m_contactList)
		m_contactList = c->m_next;
	b3Fixture* fa = c->GetFixtureA();
	b3Fixture* fb = c->GetFixtureB();
	if (c->m_nodeA.prev)
		c->m_nodeA.prev->next = c->m_nodeA.next;
	if (c->m_nodeA.next)
		c->m_nodeA.next->prev = c->m_nodeA.prev;
	if (&c->m_nodeA == fa->m_contactList)
		fa->m_contactList = c->m_nodeA.next;
	if (c->m_nodeB.prev)
		c->m_nodeB.prev->next = c->m_nodeB.next;
	if (c->m_nodeB.next)
		c->m_nodeB.next->prev = c->m_nodeB.prev;
	if (&c->m_nodeB == fb->m_contactList)
		fb->m_contactList = c->m_nodeB.next;
	b3Contact::Destroy(c, m_allocator);
	--m_contactCount;
}

// Frees the device state of a contact manager (from b3World::~b3World).
extern "C" __attribute__((visibility("default"))) void b3g_shim_release(b3ContactManager* cm)
{
	auto t = table().find(cm);
	if (t == table().end())
		return;
	if (t->second->ctx)
		b3g_destroy(t->second->ctx);
	delete t->second;
	table().erase(t);
}

// Device calls that failed since the library was loaded (0 when all went well).
extern "C" __attribute__((visibility("default"))) uint32_t b3g_shim_failures() { return g_failures; }

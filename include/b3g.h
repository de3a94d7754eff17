/*
 * b3g.h - C ABI of the B200 collision pipeline for the Bounce physics engine.
 *
 * One call of b3g_collide() is one collision pass of Bounce's b3World::Step:
 * the per-fixture fat-AABB update of the "Find New Pairs" block
 * (src/bounce/dynamics/world.cpp:424-449), the broadphase pair search and
 * contact creation of b3ContactManager::FindNewContacts / AddPair
 * (src/bounce/dynamics/contact_manager.cpp:98-223) and the narrowphase of
 * b3ContactManager::UpdateContacts (contact_manager.cpp:225-287), all on the
 * GPU. The reference's solver iterations, island search and sleep decisions
 * stay host code and consume the manifolds this library writes in the
 * reference's own b3Manifold layout (include/bounce/collision/collision.h:110-128,
 * 320 bytes). Around the pass, the world queries (AABB, ray and shape casts),
 * the fixtures' contact edge lists and the contact solver's constraints are
 * built here too.
 *
 * Conventions
 *  - Every entry point returns B3G_OK (0) or a negative status; the message of
 *    the last failure is available from b3g_last_error(). The reference has
 *    no error returns (it asserts and grows buffers); capacity overflows here
 *    are reported as B3G_E_CAPACITY and leave the previous state intact.
 *  - Host buffers are owned by the caller. Device memory is owned by the
 *    context and allocated in b3g_create (fixed capacities).
 *  - Calls on one context are serialised by the caller; a context runs on one
 *    CUDA stream. Different contexts are independent.
 *  - Indices of fixtures/bodies/hulls are the positions in the arrays given to
 *    b3g_set_*; a "world" groups bodies whose fixtures may collide.
 */
#ifndef B3G_H
#define B3G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; the entry points below are
 * the only exported symbols. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define B3G_OK 0
#define B3G_E_INVALID (-1)   /* bad argument or call order */
#define B3G_E_CAPACITY (-2)  /* a fixed device capacity was exceeded */
#define B3G_E_CUDA (-3)      /* a CUDA runtime call failed */
#define B3G_E_TIMEOUT (-4)   /* a bounded device wait gave up */
#define B3G_E_STATE (-5)     /* the context holds no scene yet */

/* b3Shape::Type (include/bounce/collision/shapes/shape.h:45-53) */
#define B3G_SHAPE_SPHERE 0
#define B3G_SHAPE_CAPSULE 1
#define B3G_SHAPE_TRIANGLE 2
#define B3G_SHAPE_HULL 3
#define B3G_SHAPE_MESH 4

/* b3BodyType (include/bounce/dynamics/body.h:39-44) */
#define B3G_BODY_STATIC 0
#define B3G_BODY_KINEMATIC 1
#define B3G_BODY_DYNAMIC 2

/* Context flags. */
#define B3G_FLAG_WARM_STARTING 1u /* b3World::SetWarmStarting (world.h:95) */
#define B3G_FLAG_CONVEX_CACHE 2u  /* b3_convexCache (collide_hulls.cpp:27, forced on by b3World()) */
/* Replay each steady-state pass from a captured CUDA graph (see b3g_collide). */
#define B3G_FLAG_GRAPH 4u
/* The caller has a contact filter (b3World::SetContactFilter, world.h:77):
 * each b3g_collide stops after the broadphase until b3g_finish_pass hands in
 * the filter's answers for the new pairs (see "Collision filters"). */
#define B3G_FLAG_CONTACT_FILTER 8u

/* Fixture flags. */
#define B3G_FIXTURE_SENSOR 1u     /* b3FixtureDef::isSensor (fixture.h:60) */

typedef struct b3g_ctx b3g_ctx;

typedef struct b3g_config
{
	uint32_t max_proxies;   /* fixtures (broadphase proxies) over all worlds */
	uint32_t max_contacts;  /* contacts (overlapping fat-AABB pairs) over all worlds */
	uint32_t max_hull_data; /* total hull vertices + half-edges + faces */
	uint32_t flags;         /* B3G_FLAG_* */
	int32_t device;         /* CUDA device ordinal */
} b3g_config;

/* Counters of the last pass. */
typedef struct b3g_counts
{
	uint32_t contacts;     /* contacts after the pass (b3ContactManager::m_contactCount) */
	uint32_t begun;        /* contacts created by this pass (AddPair) */
	uint32_t ended;        /* contacts destroyed by this pass (Destroy) */
	uint32_t touching;     /* contacts with the touching flag */
	uint32_t manifolds;    /* manifolds with at least one point */
	uint32_t points;       /* manifold points */
	uint32_t moved;        /* proxies whose fat AABB was re-inserted (BufferMove) */
	uint32_t status;       /* 0 or the B3G_E_* of a device-side failure (positive) */
} b3g_counts;

/* Lifetime -------------------------------------------------------------- */

/* Replaces: b3World::b3World / b3ContactManager::b3ContactManager
 * (world.cpp:26-75, contact_manager.cpp:26-34). */
int b3g_create(const b3g_config* config, b3g_ctx** out);
void b3g_destroy(b3g_ctx* ctx);
const char* b3g_last_error(const b3g_ctx* ctx);

/* Scene ----------------------------------------------------------------- */

/* Shared convex hull geometry, the b3Hull half-edge layout
 * (include/bounce/collision/geometry/hull.h:24-72): per hull desc[6] =
 * {vertexOffset, vertexCount, edgeOffset, edgeCount, faceOffset, faceCount};
 * verts 3 floats, edges 5 u32 (origin, twin, face, prev, next; hull-local,
 * twin of edge i is i^1 as b3QueryEdgeSeparation asserts, sat.cpp:131),
 * faces 1 u32 (first half-edge), planes 4 floats (normal, offset), centroid
 * 3 floats. Replaces the b3HullShape::m_hull pointer (hull_shape.h:42). */
int b3g_set_hulls(b3g_ctx* ctx, uint32_t hull_count, const uint32_t* desc,
	const float* verts, const uint32_t* edges, const uint32_t* faces,
	const float* planes, const float* centroids);

/* Triangle meshes (b3Mesh, mesh.h:40-60): desc 4 u32 per mesh (vertex
 * offset, vertex count, triangle offset, triangle count into the arrays),
 * vertices 3 floats, triangles 3 u32 (mesh-local vertex indices). The edge
 * wings (b3Mesh::BuildAdjacency, mesh.cpp:36-119) and the static AABB tree
 * (b3Mesh::BuildTree / b3StaticTree::Build, static_tree.cpp:22-167) are built
 * here as the reference builds them. max_triangle_pairs bounds the
 * (contact, triangle) work items of one pass (0: 4 x max_contacts); more are
 * reported as B3G_E_CAPACITY. Call before b3g_set_fixtures; a mesh fixture
 * (shape type B3G_SHAPE_MESH) names its mesh in the hull argument and has
 * params p[0..2] = scale (b3MeshShape::m_scale, non-zero), p[3] = radius
 * (B3_HULL_RADIUS = 0 in the reference); it must sit on a static body.
 * Replaces b3MeshShape::m_mesh (mesh_shape.h:50). */
int b3g_set_meshes(b3g_ctx* ctx, uint32_t mesh_count, const uint32_t* desc, const float* vertices,
	const uint32_t* triangles, uint32_t max_triangle_pairs);

/* The wing vertices of mesh m's triangles as built (3 u32 per triangle,
 * 0xFFFFFFFF for an open edge). Returns the number of triangles written. */
int b3g_mesh_wings(b3g_ctx* ctx, uint32_t mesh, uint32_t* out, uint32_t capacity);

/* Bodies: world index, b3BodyType, awake flag (b3Body::IsAwake, body.h:585).
 * Replaces: b3World::CreateBody (world.cpp:98-126). */
int b3g_set_bodies(b3g_ctx* ctx, uint32_t body_count, const uint32_t* world,
	const uint32_t* type, const uint8_t* awake);

/* Fixtures (one broadphase proxy each). params: 12 floats per fixture:
 *   sphere   p[0..2] center, p[3] radius           (sphere_shape.h)
 *   capsule  p[0..2] vertex1, p[3..5] vertex2, p[6] radius (capsule_shape.h)
 *   triangle p[0..8] vertices, p[9] radius         (triangle_shape.h; wings:
 *            b3g_set_triangle_wings)
 *   hull     p[0] radius (B3_HULL_RADIUS = 0)       (hull_shape.cpp:28)
 * proxy_key orders the two fixtures of a pair exactly as the reference's
 * proxy ids do (b3BroadPhase::Report keeps (min, max), broad_phase.cpp:341-342);
 * NULL uses the fixture index, which equals the reference's proxy order for
 * fixtures created in index order and never destroyed.
 * Replaces: b3Body::CreateFixture + b3BroadPhase::CreateProxy (body.cpp:105-136,
 * broad_phase.cpp:291-297). The next pass is a creation pass (fat AABB = AABB
 * +/- B3_AABB_EXTENSION, every proxy buffered as moved, dynamic_tree.cpp:108-128). */
int b3g_set_fixtures(b3g_ctx* ctx, uint32_t fixture_count, const uint32_t* body,
	const uint32_t* shape_type, const uint32_t* hull, const float* params,
	const uint32_t* flags, const uint32_t* proxy_key);

/* Edge wings of triangle fixtures (b3TriangleShape::m_e1Vertex..m_e3Vertex and
 * m_hasE1Vertex..m_hasE3Vertex, triangle_shape.h:45-48): for fixture
 * fixture[i], 12 floats: the wing vertices of edges 1-2, 2-3 and 3-1 (3 each,
 * shape frame) and three flags (non-zero: the edge has a wing). Fixtures
 * without a call have no wings. Needs b3g_set_fixtures first; a later
 * b3g_set_fixtures clears them. */
int b3g_set_triangle_wings(b3g_ctx* ctx, uint32_t count, const uint32_t* fixture, const float* wings);

/* Awake flags per body. Replaces: b3Body::SetAwake (body.h:588-603). A pass
 * applies its own wake-ups to these flags (see b3g_fetch_awake), so the host
 * only needs to call this when its solver puts bodies to sleep or wakes them. */
int b3g_set_awake(b3g_ctx* ctx, const uint8_t* awake);

/* Scene updates between passes --------------------------------------------
 *
 * For a host that keeps many worlds resident in one context and replaces
 * some of them between passes (admitting new worlds, retiring finished ones)
 * without disturbing the others; the reference has no counterpart (a new
 * b3World per request). Needs a scene set with proxy keys equal to the
 * fixture indices (NULL keys).
 *
 * b3g_update_scene overwrites body_count bodies (body_index[i]: world, type,
 * awake, as b3g_set_bodies) and fixture_count fixtures (fixture_index[j]:
 * body, shape type, hull, 12 params, flags, as b3g_set_fixtures; spheres,
 * capsules and hulls), and retires retire_count fixtures (retire_index[k]).
 * Retiring applies first, so an index may be retired and rewritten in one
 * call. The next pass creates the proxy of every written fixture
 * (b3DynamicTree::CreateProxy, dynamic_tree.cpp:108-128), treats each of its
 * pairs as a new contact (AddPair) and destroys the contacts the slot's
 * previous fixture had; a retired fixture has no proxy and its contacts are
 * destroyed. Other fixtures keep their proxies, contacts and manifolds.
 * World indices stay below the count set by b3g_set_bodies. Asynchronous on
 * stream (NULL: the context's stream); the host arrays may be reused when
 * the call returns.
 *
 * b3g_set_active limits the passes to bodies [0, bodies) and fixtures
 * [0, fixtures) of the uploaded scene; everything past them must be retired
 * (or unused). Captured passes are dropped when the limits change.
 *
 * b3g_world_counts writes, for worlds [0, worlds) of the last pass, 3 u32
 * each into out (device memory): contacts touching, manifolds with points,
 * manifold points. Asynchronous on stream. */
int b3g_update_scene(b3g_ctx* ctx, uint32_t body_count, const uint32_t* body_index,
	const uint32_t* world, const uint32_t* type, const uint8_t* awake,
	uint32_t fixture_count, const uint32_t* fixture_index, const uint32_t* body,
	const uint32_t* shape_type, const uint32_t* hull, const float* params, const uint32_t* flags,
	uint32_t retire_count, const uint32_t* retire_index, void* stream);
/* The same update from device memory (every array a device pointer, bodies
 * written awake): the host never sees the records, so they are checked on
 * the device; invalid ones are skipped and the next b3g_get_counts returns
 * B3G_E_INVALID. */
int b3g_update_scene_device(b3g_ctx* ctx, uint32_t body_count, const uint32_t* body_index,
	const uint32_t* world, const uint32_t* type,
	uint32_t fixture_count, const uint32_t* fixture_index, const uint32_t* body,
	const uint32_t* shape_type, const uint32_t* hull, const float* params, const uint32_t* flags,
	uint32_t retire_count, const uint32_t* retire_index, void* stream);
int b3g_set_active(b3g_ctx* ctx, uint32_t bodies, uint32_t fixtures);
int b3g_world_counts(b3g_ctx* ctx, uint32_t worlds, uint32_t* out, void* stream);

/* Kinematic motion on the device, for hosts whose body state lives in device
 * memory (the serving loop): advances bodies [0, n) by dt. state: 17 floats
 * per body (the b3g_collide layout); motion: 17 floats per body (centre 3,
 * orientation x y z s, local centre 3, linear velocity 3, angular velocity 3,
 * moving flag: 0 keeps the body where it is). The sweep start becomes the
 * current pose, c += dt v, q = normalize(q + dt/2 (w, 0) q), and the
 * transform follows (b3Body::SynchronizeTransform). Not part of the
 * reference's collision pass (its solver moves bodies). Asynchronous. */
int b3g_kinematic_step(float* state, float* motion, uint32_t n, float dt, void* stream);

/* Pass ------------------------------------------------------------------ */

/* One collision pass. body_state holds 17 floats per body:
 *   m_xf.translation (3), m_xf.rotation (x, y, z, s), m_sweep.worldCenter0 (3),
 *   m_sweep.orientation0 (x, y, z, s), m_sweep.localCenter (3)
 * (body.h; sweep.h:28-36). If state_on_device is non-zero the pointer is a
 * device pointer, otherwise host memory that is copied in on the context's
 * stream. stream is a cudaStream_t or NULL for the context's own stream.
 * Replaces, in this order: b3Body::SynchronizeFixtures + b3Fixture::Synchronize
 * + b3BroadPhase::MoveProxy (body.cpp:216-238, fixture.cpp:120-132,
 * dynamic_tree.cpp:139-207), b3ContactManager::FindNewContacts
 * (contact_manager.cpp:213-223), b3ContactManager::UpdateContacts
 * (contact_manager.cpp:225-287). The call is asynchronous.
 * With B3G_FLAG_GRAPH, a pass whose state is on the device, that follows an
 * earlier pass of the same scene, with profiling off and no body asleep, is
 * captured once into a CUDA graph per contact-buffer parity (and state
 * pointer, stream and warm-start source) and replayed afterwards: one graph
 * launch per pass, same kernels, same results. Other passes launch their
 * kernels one by one. stream must not be the legacy NULL stream for capture;
 * NULL selects the context's own stream. */
int b3g_collide(b3g_ctx* ctx, const float* body_state, int state_on_device, void* stream);

/* Waits for the last pass and returns its counters. */
int b3g_get_counts(b3g_ctx* ctx, b3g_counts* out);

/* Collision filters ------------------------------------------------------
 *
 * Beyond the shape-type rules, the reference asks two questions about every
 * pair: b3Body::ShouldCollide (body.cpp:240-263: at least one dynamic body,
 * and no joint between the two bodies with collideConnected == false) and the
 * world's b3ContactFilter::ShouldCollide (world_callbacks.h:131-138). Both are
 * asked by AddPair before a contact is created (contact_manager.cpp:78-92)
 * and again for every contact by UpdateContacts, before it skips inactive
 * contacts (contact_manager.cpp:176-199); a contact that fails is destroyed
 * at its place in the contact list. While any filter is in use, a new contact
 * also needs one of its proxies to have moved this pass, as FindPairs only
 * reports pairs of moved proxies (broad_phase.h:158-207): a pair a filter once
 * refused stays no contact until one of its proxies moves, as in the
 * reference. Passes with a filter in use run kernel by kernel (no graph).
 *
 * b3g_set_joint_pairs: the body pairs of every joint whose collideConnected
 * is false (2 u32 each, any order; repeats allowed; count 0 clears). Replaces
 * the joint-list walk of b3Body::ShouldCollide; holds for the following
 * passes until set again, and is cleared by b3g_set_bodies.
 *
 * b3g_set_contact_veto: the contact filter's answers for the contacts of the
 * last pass, in contact-list order (count = b3g_counts.contacts; veto[i] != 0
 * when ShouldCollide(fixtureA, fixtureB) of contact i is false). The next pass
 * destroys those contacts; it holds for that pass only.
 *
 * With B3G_FLAG_CONTACT_FILTER, b3g_collide runs the pass up to the
 * broadphase and returns. b3g_fetch_new_pairs then waits for it and returns
 * the number of overlapping pairs that would become new contacts, writing up
 * to capacity of them (2 u32 each: the fixture of the smaller proxy key, then
 * the other, as AddPair receives them) in the order AddPair meets them
 * (ascending proxy keys). b3g_finish_pass takes the filter's answer for each
 * (keep[i] != 0: create the contact; keep = NULL keeps them all, count
 * ignored) and runs the rest of the pass. Until b3g_finish_pass, other calls
 * on the context fail with B3G_E_INVALID. The filter is not asked about pairs
 * whose shape types have no collide routine (b3Contact::Create returns none,
 * contact.cpp:318-321): such pairs never become contacts either way. */
int b3g_set_joint_pairs(b3g_ctx* ctx, uint32_t count, const uint32_t* body_pairs);
int b3g_set_contact_veto(b3g_ctx* ctx, uint32_t count, const uint8_t* veto);
int b3g_fetch_new_pairs(b3g_ctx* ctx, uint32_t* pairs, uint32_t capacity);
int b3g_finish_pass(b3g_ctx* ctx, const uint8_t* keep, uint32_t count);

/* Inner counters of the last pass, for diagnostics and work accounting: the
 * overlapping pairs the broadphase found, previous contacts kept, hull-hull
 * contacts the feature cache did not resolve (full SAT), traversal records
 * past a leaf's scratch slots, mesh (contact, triangle) work items, wake-up
 * events and the contacts they activated or destroyed, bodies asleep after
 * the pass, and the size of each narrowphase bucket (one per b3Contact
 * subclass of contact.cpp:256-267, then sensor, inactive and apart pairs).
 * Writes min(capacity, B3G_STAT_COUNT) values; returns that number or a
 * negative status. Waits for the pass. Counterpart of the reference's
 * per-step collision statistics (b3_convexCalls, b3_gjkCalls and the like,
 * world.cpp:191-199). */
enum
{
	B3G_STAT_RAW_PAIRS = 0,
	B3G_STAT_KEPT,
	B3G_STAT_HULL_MISS,
	B3G_STAT_TRAV_OVERFLOW,
	B3G_STAT_MESH_ITEMS,
	B3G_STAT_WAKE_EVENTS,
	B3G_STAT_WAKE_ACTIVATED,
	B3G_STAT_LATE_DESTROYED,
	B3G_STAT_ASLEEP,
	B3G_STAT_BUCKET0, /* 13 bucket sizes: spheres, capsule-sphere, capsules,
	                     triangle-sphere, triangle-capsule, hull-sphere,
	                     hull-capsule, hull-triangle, hulls, mesh, sensor,
	                     inactive, apart */
	B3G_STAT_COUNT = B3G_STAT_BUCKET0 + 13
};
int b3g_get_pass_stats(b3g_ctx* ctx, uint32_t* out, uint32_t capacity);

/* Results ---------------------------------------------------------------- */

/* Contacts of the last pass, 3 u32 each: fixtureA, fixtureB (after the
 * b3Contact::Create A/B swap, contact.cpp:306-317), flags (bit0 touching,
 * bit1 begun this pass, bits 8-15 manifold count). Up to capacity records;
 * returns the number written or a negative status.
 * Every per-contact output is in the order of the reference's contact list
 * (b3ContactManager::m_contactList) after UpdateContacts: the contacts this
 * pass created, in descending (smaller proxy key, larger proxy key) order
 * (AddPair prepends the pairs FindPairs reports in ascending order,
 * broad_phase.h:181-206, contact_manager.cpp:105-111), then the older contacts
 * in their previous order. A contact whose fat AABBs no longer overlap is kept
 * (state unchanged) while neither body is active, as UpdateContacts skips it
 * (contact_manager.cpp:253-259). */
int b3g_fetch_contacts(b3g_ctx* ctx, uint32_t* out, uint32_t capacity);

/* Manifolds of the last pass in contact order, each in the reference's
 * b3Manifold layout (320 bytes, collision.h:110-128). */
int b3g_fetch_manifolds(b3g_ctx* ctx, void* out, uint32_t capacity);

/* Compact output: contact index (u32) and b3Manifold (320 bytes) of every
 * manifold with points, in contact order; a mesh contact appears once per
 * manifold (up to B3_MAX_MANIFOLDS = 3, in manifold order). Returns the count.
 * b3g_fetch_manifolds returns the first manifold of each contact. */
int b3g_fetch_touching(b3g_ctx* ctx, uint32_t* index, void* manifolds, uint32_t capacity);

/* The last pass's contact records (as b3g_fetch_contacts) and touching
 * output (as b3g_fetch_touching) copied to host buffers asynchronously, on a
 * stream of their own, so that the next b3g_collide runs while they travel.
 * Waits for the pass itself, fills *counts, starts the copies and returns;
 * the buffers hold the results once b3g_wait_results returns (pinned host
 * memory makes the copies asynchronous). The next pass waits for the copies
 * only before rewriting the contact records, at its end. */
int b3g_fetch_results_async(b3g_ctx* ctx, uint32_t* contacts, uint32_t contact_capacity, uint32_t* index,
	void* manifolds, uint32_t touch_capacity, b3g_counts* counts);

/* b3g_fetch_results_async with the touching output packed: per manifold
 * with points, the 32 bytes of b3Manifold that follow its points array
 * (pointCount, tangentImpulse, motorImpulse, motorSpeed, tangentSpeed1,
 * tangentSpeed2, padding) and then its pointCount points (72 bytes each,
 * b3ManifoldPoint), back to back; index holds the contact of each record as
 * in b3g_fetch_touching. The packed size is 32 * counts->manifolds +
 * 72 * counts->points bytes (a full b3Manifold is 320 bytes), so less data
 * crosses the host link; the host copies the records into b3Manifold. */
int b3g_fetch_results_packed_async(b3g_ctx* ctx, uint32_t* contacts, uint32_t contact_capacity, uint32_t* index,
	void* packed, uint32_t touch_capacity, uint64_t packed_capacity, b3g_counts* counts);

/* Waits for the copies of the last b3g_fetch_results_async or
 * b3g_fetch_results_packed_async. */
int b3g_wait_results(b3g_ctx* ctx);

/* The island graph's edges: for every fixture, its contacts in the order of
 * its edge list b3Fixture::m_contactList (which b3World::Solve walks to build
 * islands, world.cpp:324-370; AddPair prepends an edge, Destroy unlinks it,
 * contact_manager.cpp:115-137). offsets receives nFixtures + 1 entries
 * (fixture f's edges are contacts[offsets[f] .. offsets[f + 1])), contacts
 * the contact indices (positions in the contact list of the last pass), up
 * to capacity. Returns the number of edges, 2 per contact. */
int b3g_fetch_fixture_contacts(b3g_ctx* ctx, uint32_t* offsets, uint32_t* contacts, uint32_t capacity);

/* Contacts destroyed by the last pass: fixtureA, fixtureB, flags as above
 * (flags of the destroyed contact), in the order UpdateContacts destroys them.
 * Replaces the Destroy calls of UpdateContacts (contact_manager.cpp:270-281). */
int b3g_fetch_ended(b3g_ctx* ctx, uint32_t* out, uint32_t capacity);

/* Awake flag per body after the last pass: the flags the pass started with
 * plus the wake-ups of UpdateContacts, resolved in contact-list order (a
 * contact that starts or stops touching wakes both bodies, contact.cpp:249-254;
 * a destroyed contact with points wakes both, contact.cpp:108-126; contacts
 * later in the list see those bodies awake). Writes min(body count, capacity)
 * bytes and returns the body count. */
int b3g_fetch_awake(b3g_ctx* ctx, uint8_t* out, uint32_t capacity);

/* Hull feature caches (b3FeatureCache, sat.h:65-86) in contact order:
 * cacheType, featureType, index1, index2; 0xFFFFFFFF for non hull-hull. */
int b3g_fetch_caches(b3g_ctx* ctx, uint32_t* out, uint32_t capacity);

/* Fat AABBs of all proxies (6 floats: lower, upper), b3BroadPhase::GetFatAABB. */
int b3g_fetch_fat_aabbs(b3g_ctx* ctx, float* out, uint32_t capacity);

/* Warm-start state written by the host solver after a pass, in contact order
 * of that pass: 4 normal impulses per contact and per-manifold tangent (2) and
 * motor (1) impulses. The next pass matches points by b3ContactID exactly as
 * b3Manifold::Initialize(old) does (collision.cpp:40-61). */
int b3g_load_impulses(b3g_ctx* ctx, const float* normal_impulse, const float* tangent_impulse,
	const float* motor_impulse);

/* The same for manifolds 1 and 2 of mesh contacts (b3MeshContact keeps up to
 * B3_MAX_MANIFOLDS = 3, mesh_contact.h:61): per contact in contact order 8
 * normal impulses (4 per manifold), 4 tangent and 2 motor impulses; entries of
 * manifolds a contact does not have are ignored. Call after the pass, before
 * the next b3g_collide; manifold 0 comes from b3g_load_impulses. */
int b3g_load_mesh_impulses(b3g_ctx* ctx, const float* normal_impulse, const float* tangent_impulse,
	const float* motor_impulse);

/* Cumulative counters since creation or the last reset: out[0] passes,
 * out[1] contacts, out[2] manifolds with points, out[3] manifold points,
 * out[4] contacts created, out[5] contacts destroyed, out[6] CUDA kernels the
 * passes launched (counted on the host, graph replays included), out[7]
 * passes replayed from a captured graph (8 entries). Kept on the device and
 * summed without host synchronisation inside the passes. Replaces the
 * reference's per-step statistics (b3_convexCalls etc., world.cpp:191-199). */
int b3g_get_totals(b3g_ctx* ctx, uint64_t* out, int reset);

/* Stage timing with CUDA events on the pass's stream, the device-side
 * counterpart of b3Profiler scopes (include/bounce/common/profiler.h:96-161).
 * enable != 0 starts (and clears) accumulation. b3g_get_profile waits for the
 * recorded passes and returns per stage the summed milliseconds and the
 * number of passes, in the order of b3g_stage_name(0 .. count-1): upload,
 * sync, sort, build, traverse, diff, bucket, narrow_hulls, narrow_convex,
 * narrow_mesh, finalize. A profiled pass runs all its kernels on one stream
 * so that each stage's events enclose its own kernels (an unprofiled pass
 * runs the hull and mesh stages beside the convex one). */
int b3g_set_profiling(b3g_ctx* ctx, int enable);
int b3g_get_profile(b3g_ctx* ctx, double* ms, uint32_t* passes, uint32_t capacity);
const char* b3g_stage_name(uint32_t stage);

/* Launch shapes ------------------------------------------------------------
 *
 * No counterpart in the reference (its loops are sequential). The bucket,
 * hull and traversal kernels are grid-stride loops whose results do not
 * depend on their launch shape; the shape only changes their speed. The
 * tuning table holds B3G_TUNE_COUNT entries:
 *   [B3G_TUNE_CONVEX + k]  blocks per SM of the thread-per-pair kernel of
 *                          bucket k: spheres, capsule-sphere, capsules,
 *                          triangle-sphere, triangle-capsule, hull-sphere,
 *                          hull-capsule, sensor, inactive (128 threads per block)
 *   [B3G_TUNE_PROBE]       blocks per SM of the hull feature-cache probe
 *   [B3G_TUNE_SAT_WARPS]   warps per block of the hull-hull and hull-triangle
 *                          SAT kernels (2, 4, 8)
 *   [B3G_TUNE_SAT_BLOCKS]  blocks per SM of those kernels
 *   [B3G_TUNE_TRAVERSE]    threads per block of the LBVH traversal (64, 128, 256)
 * Defaults: 4 blocks per SM everywhere but the hull-sphere kernel (8: its
 * face scan holds few registers), 4 SAT warps per block, 2 SAT blocks per SM,
 * 128 traversal threads.
 * b3g_autotune picks each entry by timing the kernel it drives on the last
 * pass's data (the kernels re-run on the same inputs write the same outputs,
 * so the pass's results are unchanged), reps launches per candidate; it
 * needs a pass first and writes the chosen table to out (may be NULL).
 * b3g_set_tuning / b3g_get_tuning set and read the table directly;
 * set_tuning rejects values outside the candidate sets with B3G_E_INVALID. */
#define B3G_TUNE_CONVEX 0
#define B3G_TUNE_PROBE 9
#define B3G_TUNE_SAT_WARPS 10
#define B3G_TUNE_SAT_BLOCKS 11
#define B3G_TUNE_TRAVERSE 12
#define B3G_TUNE_COUNT 13
int b3g_autotune(b3g_ctx* ctx, uint32_t reps, void* stream, uint32_t* out);
int b3g_set_tuning(b3g_ctx* ctx, const uint32_t* table);

/* Bounded waits. The device work never waits without a bound: the radix
 * sort's, the scans' and the solver input's look-backs and the hull SAT
 * kernel's wait for its shared-memory copies spin at most 2^22 times, and every
 * tree walk (broadphase pair search, queries) visits at most the nodes of a
 * depth-first walk; a wait that runs out sets the pass status, and the call
 * that reads it (b3g_get_counts) returns B3G_E_TIMEOUT with the context still
 * usable; the next pass starts clean. b3g_set_walk_limit lowers the bound of
 * the broadphase walks to max_nodes node visits (0 restores the depth-first
 * bound), so that a test can make a wait run out on purpose: the walks stop
 * early, leave fewer pairs than exist, and report the timeout. The captured
 * passes are dropped so the new bound takes effect. The reference has no
 * counterpart (its walks and sorts run on the host without bounds). */
int b3g_set_walk_limit(b3g_ctx* ctx, uint32_t max_nodes);

/* LBVH reuse. A pass rebuilds the broadphase tree (Morton keys, sort, build)
 * only every `passes` passes, and whenever the set of proxies changed (a
 * fixture created, destroyed or replaced, another fixture or world count, a
 * new scene); the passes in between put the new fat AABBs in the leaves and
 * refit the internal boxes, as the reference's b3DynamicTree keeps its tree
 * across steps (dynamic_tree.cpp:108-207). The pairs found, their order and
 * every result are the same for any interval; only the walk lengths change.
 * 1 rebuilds every pass. Default B3G_TREE_REBUILD_INTERVAL. The captured
 * passes are dropped. The reference has no counterpart (its tree is
 * incremental by construction). */
#define B3G_TREE_REBUILD_INTERVAL 8u
int b3g_set_tree_rebuild_interval(b3g_ctx* ctx, uint32_t passes);
int b3g_get_tuning(b3g_ctx* ctx, uint32_t* table);

/* Device pointers of the last pass's results for zero-copy consumers:
 * contacts (3 u32 each) and manifolds (320 bytes each). */
int b3g_device_results(b3g_ctx* ctx, const void** contacts, const void** manifolds);

/* Stand-alone narrowphase ------------------------------------------------ */

/* Runs the b3Collide* routine of each pair (collision.h:152-202) on the GPU:
 * for pair i, fixtures fixA[i] / fixB[i] of the current scene, transforms
 * xfA/xfB (7 floats each) and, for hull pairs, previous transforms xf0A/xf0B
 * and the feature cache cache4 (read and written back). Writes one b3Manifold
 * (320 bytes) per pair. Hosts use it to call the narrowphase on their own
 * pair lists, e.g. for unit checks against the reference's collide functions. */
int b3g_collide_pairs(b3g_ctx* ctx, uint32_t n, const uint32_t* fixA, const uint32_t* fixB,
	const float* xfA, const float* xfB, const float* xf0A, const float* xf0B,
	uint32_t* cache4, void* manifolds);

/* World queries on the proxies, fat AABBs and body transforms of the last
 * pass (after b3g_collide; a scene update takes effect at the next pass).
 * Host buffers; at most max(max_proxies, max_contacts) queries per call;
 * worlds (one per query) may be NULL for world 0. Filters (b3QueryFilter,
 * b3RayCastFilter) are left to the caller: every live fixture of the query's
 * world is considered, sensors included.
 *
 * b3g_query_aabb replaces b3World::QueryAABB (world.cpp:854-878) with a
 * listener that accepts every fixture: boxes are 6 floats (lower, upper);
 * writes (query, fixture) pairs of every fixture whose fat AABB overlaps the
 * box (b3TestOverlap), up to capacity, and returns their number. */
int b3g_query_aabb(b3g_ctx* ctx, uint32_t n, const float* boxes, const uint32_t* worlds, uint32_t* out,
	uint32_t capacity);

/* b3World::RayCast (world.cpp:452-500) with a listener that returns 1 for
 * every fixture (keeps every hit): rays are 6 floats (p1, p2); writes
 * (ray, fixture) pairs into index and 7 floats per hit into hits (point as
 * b3World computes it, (1 - fraction) p1 + fraction p2; the shape's normal;
 * fraction), up to capacity, and returns the number of hits. The shapes' ray
 * casts are the reference's (sphere_shape.cpp:69-122, capsule_shape.cpp:180-322,
 * hull_shape.cpp:189-275, triangle_shape.cpp:95-180, mesh_shape.cpp:81-146). */
int b3g_ray_cast(b3g_ctx* ctx, uint32_t n, const float* rays, const uint32_t* worlds, uint32_t* index,
	float* hits, uint32_t capacity);

/* b3World::RayCastSingle (world.cpp:502-566): per ray the hit with the
 * smallest fraction: fixture (0xFFFFFFFF when none) and 7 floats (point,
 * normal, fraction). Of two hits at exactly the same fraction the smaller
 * fixture index is kept (the reference keeps the first its tree meets).
 * Returns the number of rays that hit. */
int b3g_ray_cast_single(b3g_ctx* ctx, uint32_t n, const float* rays, const uint32_t* worlds, uint32_t* fixture,
	float* hit);

/* b3g_ray_cast_single on device buffers (rays, worlds, fixture, hit as above,
 * all device memory; worlds may be NULL), asynchronous on stream (NULL: the
 * context's stream), for callers that keep their rays on the GPU. Nothing is
 * copied or allocated; the result is ready when the stream reaches it. */
int b3g_ray_cast_single_device(b3g_ctx* ctx, uint32_t n, const float* rays, const uint32_t* worlds,
	uint32_t* fixture, float* hit, void* stream);

/* One shape cast: a convex shape (sphere, capsule, triangle or hull; params
 * and hull as in b3g_set_fixtures) at a transform, swept along a
 * displacement, in a world. A mesh cannot be cast (the reference returns
 * without a hit, world.cpp:755-760); such casts report nothing. 112 bytes. */
typedef struct b3g_shape_cast_input
{
	uint32_t shape_type;
	uint32_t hull;
	uint32_t world;
	uint32_t pad;
	float params[12];
	float position[3]; /* b3Transform::translation */
	float rotation[4]; /* b3Transform::rotation, xyzw */
	float displacement[3];
	float pad2[2];
} b3g_shape_cast_input;

/* b3World::ShapeCast (world.cpp:752-786) with a listener that returns 1 for
 * every fixture: each fixture (each triangle of a mesh fixture) whose
 * translational time of impact (b3TimeOfImpact, time_of_impact.cpp:666-776)
 * reports touching. Writes (cast, fixture, triangle or 0) into index (3 u32
 * per hit) and 7 floats per hit (point on the fixture and normal from b3GJK
 * at the time of impact, world.cpp:719-731; fraction) up to capacity, and
 * returns the number of hits. A cast's hits come in no particular order. */
int b3g_shape_cast(b3g_ctx* ctx, uint32_t n, const b3g_shape_cast_input* casts, uint32_t* index, float* hits,
	uint32_t capacity);

/* b3World::ShapeCastSingle (world.cpp:788-851): per cast the hit with the
 * smallest fraction: fixture and triangle (2 u32; 0xFFFFFFFF when none) and 7
 * floats (point, normal, fraction). Of two hits at exactly the same fraction
 * the smaller fixture, then triangle, is kept (the reference keeps the first
 * its tree meets). Returns the number of casts that hit. */
int b3g_shape_cast_single(b3g_ctx* ctx, uint32_t n, const b3g_shape_cast_input* casts, uint32_t* fixture,
	float* hit);

/* b3g_shape_cast_single on device buffers (casts, fixture, hit as above, all
 * device memory), asynchronous on stream (NULL: the context's stream), for
 * callers that keep their casts on the GPU. The casts are not checked: every
 * hull index must be below the hull count. Nothing is copied; the scratch of
 * the cast ordering is the context's query scratch (grown on first use). */
int b3g_shape_cast_single_device(b3g_ctx* ctx, uint32_t n, const b3g_shape_cast_input* casts, uint32_t* fixture,
	float* hit, void* stream);

/* Time of impact and GJK shape cast ---------------------------------------
 *
 * Batched forms of the reference's free functions (no world needed; hull
 * shapes refer to the hulls of b3g_set_hulls). Host buffers, synchronous.
 * Shapes are convex (sphere, capsule, triangle, hull) with params as in
 * b3g_set_fixtures. Results per query: 4 u32 = b3TOIOutput state
 * (0 unknown, 1 failed, 2 overlapped, 3 touching, 4 separated), t (float
 * bits), iterations, 0. Each returns the query count. */

/* b3TOIInput (time_of_impact.h:27-34): two shapes, their b3Sweeps (18 floats
 * each in member order: localCenter, orientation0 xyzw, worldCenter0, t0,
 * orientation xyzw, worldCenter) and tMax. 272 bytes. */
typedef struct b3g_toi_input
{
	uint32_t type_a, hull_a, type_b, hull_b;
	float params_a[12], params_b[12];
	float sweep_a[18], sweep_b[18];
	float t_max;
	float pad[3];
} b3g_toi_input;

/* b3TimeOfImpact(const b3TOIInput&) (time_of_impact.cpp:465-660): the local
 * separating axis method over the two sweeps. Where the reference reaches a
 * simplex feature combination it asserts never happens, the query ends as
 * failed at the current time. */
int b3g_time_of_impact(b3g_ctx* ctx, uint32_t n, const b3g_toi_input* queries, uint32_t* out);

/* The same on device buffers, asynchronous on stream (NULL: the context's
 * stream); the queries are not checked (hull indices below the hull count,
 * convex types only). Nothing is copied or allocated. */
int b3g_time_of_impact_device(b3g_ctx* ctx, uint32_t n, const b3g_toi_input* queries, uint32_t* out,
	void* stream);

/* b3TimeOfImpact(aabb1, d1, aabb2, d2) (time_of_impact.cpp:782-902): 18
 * floats per query (aabb1 lower, upper, d1, aabb2 lower, upper, d2). */
int b3g_time_of_impact_aabb(b3g_ctx* ctx, uint32_t n, const float* queries, uint32_t* out);

/* b3ShapeCast (gjk.cpp:938-1102): proxy B moved by translation_b from its
 * transform against proxy A. 192 bytes. */
typedef struct b3g_gjk_cast_input
{
	uint32_t type_a, hull_a, type_b, hull_b;
	float params_a[12], params_b[12];
	float xf_a[7], xf_b[7]; /* translation, rotation xyzw */
	float translation_b[3];
	float pad[3];
} b3g_gjk_cast_input;

/* Writes 9 words per query: hit (u32 0 or 1), t, point (on A, radius
 * included), normal, iterations (u32); zeros where there is no hit. */
int b3g_gjk_shape_cast(b3g_ctx* ctx, uint32_t n, const b3g_gjk_cast_input* queries, float* out);

/* Solver input -------------------------------------------------------------
 *
 * b3ContactSolver's constructor and InitializeVelocityConstraints
 * (src/bounce/dynamics/contacts/contact_solver.cpp:28-149, :177-305) on the
 * manifolds of the last pass, bit for bit. The reference fills them island
 * by island from b3Position / b3Velocity arrays indexed by the bodies'
 * island indices (island.cpp:130-152); here the caller gives one
 * b3g_solver_body per body (body index of b3g_set_bodies) and, optionally,
 * the contacts to solve in its own order (an island's m_contacts). Body-level
 * fields of b3ContactPositionConstraint (invMass, localInvI, localCenter) stay
 * in the caller's body arrays; the records name the bodies by index. */

/* Friction and restitution per fixture (b3Fixture::m_friction, m_restitution;
 * b3FixtureDef's defaults 0.3 and 0 until this call, fixture.h:46-47). Host
 * arrays of the fixture count. */
int b3g_set_materials(b3g_ctx* ctx, const float* friction, const float* restitution);

/* One body: its b3Position and b3Velocity entries (island.cpp:130-134) and
 * the fields the constraints read from b3Body. 112 bytes, 16-byte aligned. */
typedef struct b3g_solver_body
{
	float x[3];           /* b3Position::x, centre of mass (b3Sweep::worldCenter) */
	float q[4];           /* b3Position::q, xyzw */
	float v[3];           /* b3Velocity::v */
	float w[3];           /* b3Velocity::w */
	float inv_mass;       /* b3Body::m_invMass */
	float local_center[3]; /* b3Body::m_sweep.localCenter */
	float inv_i[9];       /* b3Position::I, world inverse inertia, columns x, y, z */
	float pad[2];
} b3g_solver_body;

/* b3ContactVelocityConstraint (contact_solver.h:93-105) with the radii of
 * b3ContactPositionConstraint; its manifolds are records manifold_start ..
 * manifold_start + manifold_count - 1. 128 bytes. */
typedef struct b3g_contact_constraint
{
	uint32_t index_a, index_b;    /* bodies (0xFFFFFFFF: listed index past the contact list) */
	uint32_t manifold_start, manifold_count;
	float inv_mass_a, inv_mass_b;
	float friction;               /* b3MixFriction: sqrt(fA * fB) */
	float restitution;            /* b3MixRestitution: max(eA, eB) */
	float inv_i_a[9], inv_i_b[9]; /* b3Position::I of the bodies */
	float radius_a, radius_b;     /* b3Shape::m_radius */
	uint32_t contact;             /* position in the contact list */
	uint32_t pad[3];
} b3g_contact_constraint;

/* b3VelocityConstraintPoint (contact_solver.h:60-69). */
typedef struct b3g_velocity_point
{
	float r_a[3], r_b[3], normal[3];
	float normal_mass, normal_impulse, velocity_bias;
} b3g_velocity_point;

/* b3PositionConstraintPoint (contact_solver.h:31-36). */
typedef struct b3g_position_point
{
	float local_normal_a[3], local_point_a[3], local_point_b[3];
} b3g_position_point;

/* b3VelocityConstraintManifold (contact_solver.h:71-91) and the points of
 * the matching b3PositionConstraintManifold; points past point_count are
 * zero. Fields the reference leaves unset when a manifold has no points
 * (tangents) are zero. 464 bytes. */
typedef struct b3g_manifold_constraint
{
	float r_a[3], r_b[3];
	float normal[3], tangent1[3], tangent2[3];
	float tangent_speed1, tangent_speed2;
	float tangent_mass[4];        /* b3Mat22 columns x, y */
	float tangent_impulse[2];
	float motor_impulse, motor_mass, motor_speed;
	uint32_t point_count;
	uint32_t constraint;          /* its b3g_contact_constraint */
	uint32_t pad[4];
	b3g_velocity_point points[4];
	b3g_position_point position_points[4];
} b3g_manifold_constraint;

/* Builds the constraints on device buffers, asynchronously on stream (NULL:
 * the context's stream), without host synchronisation; the first call
 * allocates a small scratch array (tile sums), later calls allocate nothing.
 * contacts: count contact indices (device memory) in the order to solve
 * them; NULL selects every touching contact whose fixtures are not sensors,
 * in contact-list order (the contacts b3World::Solve puts on islands,
 * world.cpp:336-348), and count is ignored (count <= max_contacts).
 * bodies: one b3g_solver_body per body. dt_ratio, warm_starting: the
 * b3TimeStep fields (impulses are dt_ratio times the manifolds' warm-start
 * impulses, or zero). Writes up to constraint_capacity and
 * manifold_capacity records and, into counts (device memory, 2 u32), the
 * numbers of constraints and manifolds (which may exceed the capacities).
 * All device pointers 16-byte aligned. */
int b3g_contact_constraints_device(b3g_ctx* ctx, uint32_t count, const uint32_t* contacts,
	const b3g_solver_body* bodies, float dt_ratio, int warm_starting, b3g_contact_constraint* constraints,
	uint32_t constraint_capacity, b3g_manifold_constraint* manifolds, uint32_t manifold_capacity,
	uint32_t* counts, void* stream);

/* The same on host buffers (copied in and out on the context's stream;
 * synchronous). counts (host, 2 u32) receives the totals; returns the number
 * of constraints, or B3G_E_INVALID for a listed index past the contact list. */
int b3g_contact_constraints(b3g_ctx* ctx, uint32_t count, const uint32_t* contacts,
	const b3g_solver_body* bodies, float dt_ratio, int warm_starting, b3g_contact_constraint* constraints,
	uint32_t constraint_capacity, b3g_manifold_constraint* manifolds, uint32_t manifold_capacity,
	uint32_t* counts);

/* Pair search without device allocation ------------------------------------
 *
 * No counterpart in the reference. For callers that cannot allocate device
 * memory: an engine that owns all GPU memory through its own arena, code that
 * runs while a CUDA graph is being captured (cudaMalloc cannot be captured),
 * or a thread that must not wait on the allocator. It allocates nothing (no
 * cudaMalloc, cudaFree or allocating library call); its scratch is one
 * file-scope device array sized for B3G_STATIC_MAX_PROXIES proxies (about
 * 200 KB on every GPU that loads the library, held until exit).
 *
 * aabbs: n fat AABBs in device memory, 6 floats each (lower, upper), as
 * b3g_fetch_fat_aabbs returns them. Writes every overlapping pair (closed
 * test, b3TestOverlap) as (min index, max index) into pairs (device memory,
 * 2 u32 each, up to capacity pairs, unspecified order) and the number of
 * overlapping pairs into *count (device memory; may exceed capacity).
 * Asynchronous on stream (a cudaStream_t, NULL for the legacy stream), on
 * the current device. Returns B3G_E_CAPACITY when n > B3G_STATIC_MAX_PROXIES,
 * and B3G_E_CUDA without running anything when a CUDA error of earlier work
 * is pending on the calling thread (cudaPeekAtLastError; that error is left
 * in place for its owner).
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls on a device share the array: the counters that must start at
 * zero are cleared by each call, and calls that overlap on the GPU (e.g. on
 * two unordered streams) race. */
#define B3G_STATIC_MAX_PROXIES 16384u
int b3g_find_pairs_static(const float* aabbs, uint32_t n, uint32_t* pairs, uint32_t capacity,
	uint32_t* count, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* B3G_H */

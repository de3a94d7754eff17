// Internal state of a b3g context and the launchers shared by the .cu files.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/b3g.h"
#include "b3g_math.cuh"

// Device-side status bits (b3g_counts::status).
#define B3G_ST_PAIR_OVERFLOW 1u
#define B3G_ST_HASH_OVERFLOW 2u
#define B3G_ST_POLY_OVERFLOW 4u
#define B3G_ST_WAIT_TIMEOUT 8u

// Narrowphase buckets: one per b3Contact subclass (contact.cpp:256-267).
enum Bucket : uint32_t
{
	BK_SPHERES = 0,      // b3SphereContact
	BK_CAPSULE_SPHERE,   // b3CapsuleAndSphereContact
	BK_CAPSULES,         // b3CapsuleContact
	BK_TRIANGLE_SPHERE,  // b3TriangleAndSphereContact
	BK_TRIANGLE_CAPSULE, // b3TriangleAndCapsuleContact
	BK_HULL_SPHERE,      // b3HullAndSphereContact
	BK_HULL_CAPSULE,     // b3HullAndCapsuleContact
	BK_HULL_TRIANGLE,    // b3HullAndTriangleContact
	BK_HULLS,            // b3HullContact
	BK_MESH,             // b3MeshContact subclasses (mesh-sphere, mesh-capsule, hull-mesh), sensors included
	BK_SENSOR,           // any other pair with a sensor: b3Contact::TestOverlap path
	BK_INACTIVE,         // both bodies asleep or static: state carried over
	BK_APART,            // convex pairs whose bounding spheres are apart: empty manifold
	BK_COUNT
};

// b3Manifold / b3ManifoldPoint, byte-identical to the reference layout
// (collision.h:66-128; 72 and 320 bytes).
struct alignas(8) DevPoint
{
	float n[3];
	float p1[3];
	float p2[3];
	float normalImpulse;
	uint32_t triangleKey;
	uint32_t pad0;
	uint32_t key[4];
	uint8_t persisting;
	uint8_t edgeContact;
	uint8_t pad1[6];
};
static_assert(sizeof(DevPoint) == 72, "b3ManifoldPoint layout");

struct alignas(8) DevManifold
{
	DevPoint points[4];
	uint32_t pointCount;
	float tangentImpulse[2];
	float motorImpulse;
	float motorSpeed;
	float tangentSpeed1;
	float tangentSpeed2;
	uint32_t pad;
};
static_assert(sizeof(DevManifold) == 320, "b3Manifold layout");

struct HullDesc
{
	uint32_t vOff, vCnt, eOff, eCnt, fOff, fCnt;
	float cx, cy, cz;
	uint32_t pad[3];
};
static_assert(sizeof(HullDesc) == 48, "HullDesc");

// A triangle mesh (b3Mesh, mesh.h:40-60): vertices, triangles with their
// edge wings (b3Mesh::BuildAdjacency) and the static AABB tree
// (b3StaticTree, built on the host exactly as b3Mesh::BuildTree does).
struct MeshDesc
{
	uint32_t vOff, vCnt;   // vertices (float4)
	uint32_t tOff, tCnt;   // triangles (uint4 vertex indices) and wings (uint4)
	uint32_t nOff, nCnt;   // tree nodes (2 float4 each)
	uint32_t root, pad;
};
static_assert(sizeof(MeshDesc) == 32, "MeshDesc");
#define B3G_NULL_NODE 0xFFFFFFFFu

// Scene and per-pass device buffers.
struct DevScene
{
	// hulls
	const HullDesc* hulls;
	const float4* hverts;  // xyz
	const uint4* hedges;   // origin, face, prev, next (twin = i ^ 1)
	const uint32_t* hfaces;
	const float4* hplanes; // normal, offset
	uint32_t hullMaxV, hullMaxE, hullMaxF; // the largest hull's counts (shared-memory staging)

	// bodies
	const uint32_t* bodyWorld;
	const uint32_t* bodyType;
	const uint8_t* bodyAwake;
	const float* bodyState; // 17 floats per body
	float4* bodyXf;         // per pass: m_xf, 2 float4 per body
	float4* bodyXf0;        // per pass: b3Sweep::GetTransform(0), 2 float4 per body

	// fixtures
	const uint32_t* fixBody;
	const uint32_t* fixType;
	const uint32_t* fixHull;
	const float4* fixParams; // 3 float4 per fixture
	const float4* fixBound;  // bounding sphere per fixture: body-frame centre, radius
	const uint32_t* fixFlags;
	const uint32_t* fixKey;
	const uint32_t* fixRank; // rank of the fixture's proxy key among all keys
	uint8_t* fixLife;        // FIX_LIVE / FIX_FRESH / FIX_DEAD (scene updates between passes)
	// triangle fixtures: b3TriangleHull per fixture (vertices 0-2, planes 3-4,
	// centroid 5; 6 float4) and the edge wings (3 float4: wing vertex, w = 1
	// when the edge has one)
	const float4* fixTri;
	const float4* fixWing;

	// triangle meshes: fixtures of type mesh keep the mesh index in fixHull
	// and p[0..2] = scale, p[3] = radius
	const MeshDesc* meshes;
	const float4* meshVerts;  // xyz
	const uint4* meshTris;    // mesh-local vertex indices
	const uint4* meshWings;   // wing vertex per edge, B3G_NULL for an open edge
	const float4* meshNodes;  // (lower, child1 bits), (upper, child2 or triangle bits)
};

// Fixture life states. A fresh fixture was written by a scene update since the
// last pass: the pass creates its proxy (CreateProxy fattening) and none of
// its pairs continues a contact of the fixture that held the slot before. A
// dead fixture has no proxy: it sorts after every live one, never pairs, and
// the contacts it had are destroyed.
enum : uint8_t
{
	FIX_LIVE = 0,
	FIX_FRESH = 1,
	FIX_DEAD = 2
};

struct Buffers
{
	// broadphase, per proxy
	float4* fatLo;
	float4* fatHi;
	uint8_t* moved;
	unsigned long long* keysA;
	unsigned long long* keysB;
	uint32_t* valsA;
	uint32_t* valsB;
	uint32_t* sortHist;
	float* sceneBounds; // 6 floats (ordered-int encoded during reduction)
	// LBVH: internal nodes [0, n-1), leaves [n-1, 2n-1)
	float4* nodeLo;
	float4* nodeHi;
	uint32_t* nodeLeft;   // internal: left child node; leaf: proxy index
	uint32_t* nodeRight;  // internal: right child node
	uint32_t* nodeRope;
	uint32_t* nodeFirst;  // first sorted leaf of the node's range
	uint32_t* nodeParent;
	uint32_t* nodeEnd;    // internal: last sorted leaf of the range
	uint32_t* splitRight; // right child of the internal node whose split is i
	uint32_t* refitFlag;
	uint32_t* worldEnd;   // per sorted leaf: last sorted leaf of its world
	uint32_t* proxyInfo;  // per proxy: body (bits 0-27), dynamic body (bit 28), shape type (bits 29-31)
	uint2* leafData;      // per sorted leaf: its proxy's proxyInfo word and fixture key
	uint32_t* leafOf;     // per proxy: its sorted leaf (set when the LBVH is built)
	uint32_t* leafCount;  // pair count per sorted leaf (then exclusive offsets)
	uint32_t* pairScratch; // first contact records (A, B) found per leaf, slot-major (B3G_TRAV_SLOTS x n uint2)
	uint32_t* scanAux;
	uint32_t* rawA;       // overlapping pairs in traversal order (this pass)
	uint32_t* rawB;
	uint4* travOverflow;  // records past a leaf's scratch slots: A, B, leaf, index in the leaf

	// contact-list order: new contacts, then the kept previous ones
	uint32_t* newList;    // raw indices of pairs without a previous contact
	uint32_t* newOff;     // per smaller-key rank (reversed): offsets, nFixtures + 1
	uint32_t* newFill;
	uint32_t* newTmp;     // raw index per new-contact slot, grouped by smaller key
	uint32_t* newTmpMax;  // larger key rank per slot
	uint32_t* keptScan;   // per previous contact: kept flag, then exclusive offsets
	uint32_t* posKey;     // per contact: position in the list UpdateContacts walks

	// contacts, double-buffered [cur], [prev]
	uint32_t* pairA[2];
	uint32_t* pairB[2];
	uint32_t* cstate[2]; // bit0 touching, bits 8-15 manifold count, bit 16 begun
	uint4* cache[2];
	DevManifold* man[2];
	int32_t* prevIndex; // per current contact
	uint32_t* prevFound; // per previous contact: its pair overlaps again this pass
	unsigned long long* hashKeys[2];
	uint32_t* hashVals[2];
	uint32_t hashCap;     // slots allocated per table (for the contact capacity)
	uint32_t* hashMask;   // per table: slots in use - 1 (a power of two - 1), sized to its pass's contacts

	// narrowphase work lists
	uint32_t* bucketList; // BK_COUNT lists of max_contacts entries
	uint32_t* missList;   // hull-hull contacts for the SAT kernel
	float4* hcPost;       // hull-capsule contacts past their GJK: 2 float4 each
	uint32_t* hsPost;     // hull-sphere contacts past their face scan
	uint32_t* counters;   // device counters (see CTR_*)
	unsigned long long* totals; // cumulative: passes, contacts, manifolds, points, begun, ended
	uint32_t* endedList;  // 3 u32 per ended contact
	uint32_t* touchIndex;
	DevManifold* touchMan;
	uint32_t* contactOut; // 3 u32 per contact: A, B, flags

	// mesh contacts (allocated when the scene has meshes)
	float4* meshAABB[2];      // per contact: the other shape's fat AABB in mesh space (2 float4)
	DevManifold* extraMan[2]; // per contact: manifolds 1 and 2 of a mesh contact
	uint32_t* meshCount;      // per contact: overlapping triangles, then exclusive offsets
	uint32_t* meshPairC;      // per (contact, triangle) work item: contact
	uint32_t* meshPairT;      // ... triangle
	DevManifold* meshPairMan; // ... its b3Manifold (triangleKey set)
	float4* meshObs;          // 3 per point slot of a work item: cluster observations
	float4* meshPoly;         // 1 per point slot: a cluster's polygon vertices
	float* meshImpulses;      // 14 per contact: host impulses of manifolds 1 and 2
	uint32_t meshPairCap;

	// wake-ups of UpdateContacts (only when some body is asleep)
	uint32_t* tWake;        // per body: earliest list position that woke it
	uint32_t* wakeList;     // contacts activated this round
	uint32_t* inactiveSave; // contacts skipped as inactive in the first round
	uint32_t* activated;    // per inactiveSave entry
	uint32_t* lateDestroyed; // per contact

	// warm start from the host solver
	float* impulseNormal;
	float* impulseTangent;
	float* impulseMotor;
};

// Collision filters beyond the shape-type rules, decided pass by pass: joints
// that keep their bodies from colliding (b3Body::ShouldCollide, body.cpp:240-263)
// and the caller's contact filter (b3ContactFilter::ShouldCollide, called by
// AddPair, contact_manager.cpp:86-92, and for every contact by UpdateContacts,
// :189-199). mode 0: none (the default pass); 1: joints and the per-contact
// veto applied inside k_diff / k_kept; 2: as 1, plus new pairs the caller's
// filter rejected, precomputed per overlapping pair in rawDrop.
// With a filter in use a new contact also needs a proxy that moved this pass
// (was re-inserted or created): FindPairs reports only pairs of moved proxies
// (broad_phase.h:158-207), so a pair that a filter once refused stays no
// contact until one of its proxies moves. Without filters every such pair is
// already a contact, and the rule changes nothing.
struct FilterArgs
{
	int mode;
	const unsigned long long* jointKeys; // sorted (smaller body << 32 | larger body)
	uint32_t nJoints;
	const uint8_t* bodyJoint;            // per body: in some joint pair
	const uint8_t* vetoPrev;             // per contact of the previous pass: destroy it
	uint32_t nVeto;
	uint8_t* rawDrop;                    // per overlapping pair of the pass: no contact (mode 2)
};

__device__ __forceinline__ bool joint_excluded(const FilterArgs& F, uint32_t ba, uint32_t bb)
{
	if (F.nJoints == 0 || !F.bodyJoint[ba] || !F.bodyJoint[bb])
		return false;
	unsigned long long k = ba < bb ? ((unsigned long long)ba << 32) | bb : ((unsigned long long)bb << 32) | ba;
	uint32_t lo = 0, hi = F.nJoints;
	while (lo < hi)
	{
		uint32_t mid = (lo + hi) >> 1;
		if (F.jointKeys[mid] < k)
			lo = mid + 1;
		else
			hi = mid;
	}
	return lo < F.nJoints && F.jointKeys[lo] == k;
}

// Contact records a leaf's walk keeps in its scratch slots; leaves with more
// partners walk again for the rest.
#define B3G_TRAV_SLOTS 32u

// Counter slots in Buffers::counters.
enum
{
	CTR_PAIRS = 0,      // contacts this pass
	CTR_PREV_PAIRS,     // contacts of the previous pass
	CTR_BEGUN,
	CTR_ENDED,
	CTR_TOUCHING,
	CTR_MANIFOLDS,
	CTR_POINTS,
	CTR_MOVED,
	CTR_STATUS,
	CTR_TOUCH_OUT,
	CTR_HULL_MISS,      // hull-hull contacts the feature cache did not resolve
	CTR_RAW,            // overlapping pairs found by the traversal
	CTR_KEPT,           // previous contacts kept
	CTR_WAKE_EVENTS,
	CTR_WAKE_ACTIVATED,
	CTR_LATE_DESTROYED,
	CTR_BUCKET0 = 16,   // BK_COUNT bucket sizes
	CTR_ASLEEP = 29,    // non-static bodies still asleep after the wake-ups
	CTR_SCRATCH = 30,
	CTR_MESH_PAIRS = 31, // (contact, triangle) work items of the pass
	CTR_TRAV_OVERFLOW = 32, // traversal records past the scratch slots
	CTR_CANDIDATES = 33,    // new pairs handed to the caller's contact filter
	CTR_HC_POST = 34,       // hull-capsule contacts past their GJK (k_hull_capsule_post): at a distance
	CTR_HC_DEEP = 35,       // ... and overlapping
	CTR_HS_POST = 36,       // hull-sphere contacts past their face scan (k_hull_sphere_gjk)
	CTR_COUNT = 37
};
static_assert(CTR_BUCKET0 + BK_COUNT <= CTR_ASLEEP, "bucket counters overlap");

// Launch shapes of the tunable kernels (include/b3g.h, B3G_TUNE_*).
#define B3G_CONVEX_KERNELS 9
struct Tune
{
	uint32_t v[B3G_TUNE_COUNT];
};

// A captured steady-state pass (one per contact-buffer parity and warm-start
// source), valid for the stream it was captured on; the state copy node is
// re-pointed when a pass brings its state from another address.
struct PassGraph
{
	cudaGraph_t graph;
	cudaGraphExec_t exec;
	cudaGraphNode_t copyNode;
	const float* state;
	cudaStream_t stream;
	cudaMemcpyKind kind; // of the state copy node
};

// One staging block of b3g_update_scene.
#define B3G_STAGE_RING 4
struct StageSlot
{
	void* host;
	void* dev;
	size_t bytes;
	cudaEvent_t done; // the block's last copy to the device finished
};

struct b3g_ctx
{
	b3g_config cfg;
	int device;
	cudaStream_t stream;
	std::string err;
	uint32_t treeLeaves;  // leaves of the LBVH built by the last pass
	uint32_t treeWorlds;  // worlds of the scene the LBVH was last asked to rebuild for
	uint32_t treeInterval; // passes between LBVH rebuilds (refit in between), b3g_set_tree_rebuild_interval
	uint32_t treeSince;   // passes since the LBVH was last rebuilt
	bool treeForce;       // the next pass rebuilds the LBVH (the proxy set may have changed)
	bool treeRebuild;     // the pass being issued rebuilds the LBVH
	cudaStream_t copyStream;  // device-to-host copies of b3g_fetch_results_async
	cudaEvent_t copyReady;    // results of the pass ready to copy
	cudaEvent_t copyDone;     // those copies finished
	bool copyPending;
	uint32_t* touchBytes;     // per contact: packed bytes of its manifolds
	void* edgeBuf;            // b3g_fetch_fixture_contacts scratch (allocated on first use)
	size_t edgeBytes;
	cudaStream_t sideStream;  // hull-hull / hull-triangle narrowphase, beside the convex buckets
	cudaStream_t meshStream;  // mesh midphase (tree queries, work items), beside both
	cudaEvent_t forkEvent, joinEvent, meshFork, meshJoin;
	void* qScratch;       // device scratch of the world queries
	size_t qScratchBytes;
	float2* dFixMaterial;         // per fixture: friction, restitution (b3g_set_materials)
	unsigned long long* ciTiles;  // b3g_contact_constraints_device: tile counter and states (allocated on first use)
	uint32_t ciTileCap;
	void* ciHost;                 // b3g_contact_constraints: device copies of its host buffers
	size_t ciHostBytes;
	void* toiScratch;             // time-of-impact batches: device copies of their host buffers
	size_t toiScratchBytes;

	uint32_t nHulls, nBodies, nFixtures, nWorlds;
	uint32_t hullVerts, hullEdges, hullFaces;
	uint32_t maxUniqueEdges; // unique edges (half-edge pairs) of the largest hull
	uint32_t cur; // index of the current contact buffer
	bool creationPass;
	bool havePass;
	bool impulsesLoaded;

	DevScene scene;
	Buffers buf;

	// owned scene allocations
	HullDesc* dHulls;
	float4* dHverts;
	uint4* dHedges;
	uint32_t* dHfaces;
	float4* dHplanes;
	uint32_t *dBodyWorld, *dBodyType;
	uint8_t* dBodyAwake;
	float* dBodyState;
	uint32_t *dFixBody, *dFixType, *dFixHull, *dFixFlags, *dFixKey, *dFixRank;
	uint8_t* dFixLife;
	float4* dFixTri;
	float4* dFixWing;
	uint32_t triSlots; // fixtures with triangle storage (all, or 1 when there are no triangles)

	// triangle meshes
	uint32_t nMeshes;
	MeshDesc* dMeshes;
	float4* dMeshVerts;
	uint4* dMeshTris;
	uint4* dMeshWings;
	float4* dMeshNodes;
	std::vector<MeshDesc> hMeshes;
	uint32_t* dMeshFix;       // mesh fixtures of the scene
	uint32_t nMeshFix;
	uint32_t capBodies, capFixtures; // uploaded counts; nBodies / nFixtures are the processed prefixes
	bool keysAreIndex;               // proxy keys = fixture indices (scene updates need it)
	// staging of b3g_update_scene: a ring of pinned host / device blocks
	StageSlot stage[B3G_STAGE_RING];
	uint32_t stageNext;
	uint32_t* dWorldCounts;
	uint32_t* dUpdateBad;        // a device-side scene update skipped invalid records
	bool fixTypeStale;           // hFixType lags device-side scene updates
	std::vector<uint8_t> hAwake; // host copy of the awake flags (sleep count)
	float4* dFixParams;
	float4* dFixBound;

	// host copies of the hull arrays (bounding spheres at fixture upload)
	std::vector<uint32_t> hHullDesc;
	std::vector<float> hHullVerts;

	// pinned host staging
	uint32_t* hCounters;

	// host copies of fixture types (for the stand-alone narrowphase)
	std::vector<uint32_t> hFixType;

	// host copy of body types; non-static bodies asleep at the start of the
	// next pass
	std::vector<uint32_t> hBodyType;
	uint32_t asleep;
	bool anyTriangle;     // some fixture may be a triangle (the triangle buckets can be non-empty)
	bool anySensor;       // some fixture may be a sensor

	// kernels launched by passes (host count)
	uint64_t launches;

	// launch shapes and captured passes
	Tune tune;
	PassGraph graphs[2][2][2]; // [contact buffer][warm start from host impulses][LBVH rebuilt]
	uint64_t graphLaunches;
	bool lastPassImpulses;  // the last pass warm-started from host impulses

	// collision filters (b3g_set_joint_pairs, b3g_set_contact_veto,
	// B3G_FLAG_CONTACT_FILTER); device arrays allocated on first use
	unsigned long long* dJointKeys;
	uint32_t nJoints, jointCap;
	uint8_t* dBodyJoint;
	uint32_t bodyJointCap;
	uint8_t* dVetoPrev;  // max_contacts bytes
	uint32_t nVeto;      // contacts of the last pass the veto covers (0: none)
	uint8_t* dRawDrop;   // max_contacts bytes
	uint32_t* dCand;     // candidates: raw index of each (max_contacts)
	uint4* dCandPairs;   // per candidate: fixtures as AddPair gets them and their keys; then
	                     // the raw indices the caller's filter rejected (max_contacts uint4)
	std::vector<uint32_t> hCandOrder; // raw indices of the candidates in AddPair order
	uint32_t nCand;
	bool candFetched;
	bool passOpen;       // b3g_collide stopped before the contact list for the filter
	cudaStream_t passStream; // the stream of the open pass
	int filterMode;      // FilterArgs::mode of the pass under way
	uint32_t walkLimit;  // node visits per broadphase walk (0: the depth-first bound), b3g_set_walk_limit

	// stage profiling: a ring of per-pass event sets
	bool profiling;
	uint64_t profPass;     // passes recorded since enabling
	uint64_t profHarvest;  // passes already accumulated
	cudaEvent_t* profEvents; // PROF_RING * PROF_MARKS
	double profMs[16];
	uint32_t profCount[16];
};

// Stage boundaries of one pass (see b3g_stage_name).
enum
{
	PM_BEGIN = 0,
	PM_UPLOADED,
	PM_SYNCED,
	PM_SORTED,
	PM_BUILT,
	PM_TRAVERSED,
	PM_DIFFED,
	PM_BUCKETED,
	PM_HULLS,
	PM_CONVEX,
	PM_MESH,
	PM_FINAL,
	PROF_MARKS
};
constexpr int PROF_STAGES = PROF_MARKS - 1;
constexpr int PROF_RING = 64;

// Records boundary `mark` of the current pass when profiling is on.
void prof_mark(b3g_ctx* c, int mark, cudaStream_t s);
uint32_t broadphase_launches(const b3g_ctx* c);

// Launchers (defined in the .cu files).
void launch_sync(b3g_ctx* c, cudaStream_t s);
void launch_broadphase(b3g_ctx* c, cudaStream_t s);
void launch_traverse(b3g_ctx* c, cudaStream_t s);
void launch_pairs_diff(b3g_ctx* c, cudaStream_t s);
void launch_candidates(b3g_ctx* c, cudaStream_t s);
void launch_candidate_pairs(b3g_ctx* c, uint32_t n, cudaStream_t s);
void launch_apply_veto(b3g_ctx* c, const uint32_t* rejected, uint32_t n, cudaStream_t s);
void launch_narrowphase(b3g_ctx* c, cudaStream_t s);
void launch_finalize(b3g_ctx* c, cudaStream_t s);
uint32_t pairs_diff_launches(const b3g_ctx* c);
void launch_mesh_fat(b3g_ctx* c, cudaStream_t s);
void launch_mesh_prepare(b3g_ctx* c, cudaStream_t s);
void launch_mesh_collide(b3g_ctx* c, const uint32_t* list, const uint32_t* count, cudaStream_t s);
uint32_t mesh_launches(const b3g_ctx* c);
void free_mesh(b3g_ctx* c);
void free_queries(b3g_ctx* c);
int resolve_wakeups(b3g_ctx* c, cudaStream_t s);
void launch_collide_pairs(b3g_ctx* c, cudaStream_t s, uint32_t n, const uint32_t* fixA,
	const uint32_t* fixB, const float* xfA, const float* xfB, const float* xf0A,
	const float* xf0B, uint4* cache, DevManifold* out);

// One b3g_contact_constraints_device call (solver_input.cu).
struct ConstraintCall
{
	const uint32_t* list; // contacts to solve, or null for every touching non-sensor contact
	uint32_t listCount;
	const float2* material;
	const b3g_solver_body* bodies;
	float dtRatio;
	int warm;
	unsigned long long* tiles;
	uint32_t* counts;
	b3g_contact_constraint* constraints;
	uint32_t constraintCap;
	b3g_manifold_constraint* manifolds;
	uint32_t manifoldCap;
};
uint32_t contact_constraint_tiles(uint32_t items);
void launch_contact_constraints(b3g_ctx* c, const ConstraintCall& q, cudaStream_t s);

// Grid size for grid-stride loops over device-side counts.
inline int persistent_blocks(int perSM = 8) { return 148 * perSM; }

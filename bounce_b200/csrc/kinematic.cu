// Kinematic body motion between passes for hosts that keep body state on the
// device (the serving loop): one thread per body advances the sweep the way
// b3Body's integration and SynchronizeTransform leave it (sweep start = the
// current pose, c += dt v, q = normalize(q + dt/2 (w, 0) q), xf.p = c - R(q) lc).
// Not part of the reference's collision pass (its solver moves the bodies).

#include "b3g_math.cuh"
#include "../../include/b3g.h"

namespace {

// motion: 17 floats per body: centre (3), orientation (x, y, z, s), local
// centre (3), linear velocity (3), angular velocity (3), moving flag (1 = moves).
__global__ void k_kinematic(float* state, float* motion, uint32_t n, float dt)
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	float* m = motion + 17 * (size_t)i;
	if (m[16] == 0.0f)
		return;
	float* st = state + 17 * (size_t)i;
	V3 c = V3{m[0], m[1], m[2]};
	Q4 q = Q4{V3{m[3], m[4], m[5]}, m[6]};
	V3 lc = V3{m[7], m[8], m[9]};
	V3 v = V3{m[10], m[11], m[12]};
	V3 w = V3{m[13], m[14], m[15]};
	// sweep start
	st[7] = c.x, st[8] = c.y, st[9] = c.z;
	st[10] = q.v.x, st[11] = q.v.y, st[12] = q.v.z, st[13] = q.s;
	// qdot = 0.5 (w, 0) q = 0.5 (w x qv + qs w, -w . qv)
	V3 dv = cross(w, q.v) + q.s * w;
	float ds = -dot(w, q.v);
	Q4 q1;
	q1.v = q.v + dt * (0.5f * dv);
	q1.s = q.s + dt * (0.5f * ds);
	qnormalize_inplace(q1);
	V3 c1 = c + dt * v;
	m[0] = c1.x, m[1] = c1.y, m[2] = c1.z;
	m[3] = q1.v.x, m[4] = q1.v.y, m[5] = q1.v.z, m[6] = q1.s;
	V3 p = c1 - rot(q1, lc);
	st[0] = p.x, st[1] = p.y, st[2] = p.z;
	st[3] = q1.v.x, st[4] = q1.v.y, st[5] = q1.v.z, st[6] = q1.s;
	st[14] = lc.x, st[15] = lc.y, st[16] = lc.z;
}

} // namespace

extern "C" int b3g_kinematic_step(float* state, float* motion, uint32_t n, float dt, void* stream)
{
	if ((!state || !motion) && n)
		return B3G_E_INVALID;
	if (n == 0)
		return B3G_OK;
	k_kinematic<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(state, motion, n, dt);
	return cudaGetLastError() == cudaSuccess ? B3G_OK : B3G_E_CUDA;
}

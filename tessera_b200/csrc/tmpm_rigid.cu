// tmpm_rigid.cu -- device side of the MPM-owned two-way rigid coupling.
//
// Rigid bodies drive obstacles and take back the impulses the grid and the
// particles exert on them, without a round trip to the host between
// substeps (GpuRigidMpmCoupler::submit_mpm_owned_step,
// crates/tessera-mpm/src/gpu_rigid_sync.rs:187-214).  Per coupled substep:
//   k_rigid_sync   obstacle pose and velocity from its body
//                  (gpu_rigid_sync.wgsl:46-61)
//   (one MPM substep with reaction accumulation)
//   k_rigid_apply  the obstacle impulses summed per body change its linear and
//                  angular velocity; gravity, a speed limit and the pose
//                  integration follow (gpu_rigid_reaction.wgsl:71-150)
// Both kernels use f32 like the reference shaders; the impulses are summed
// from the f64 per-obstacle accumulators.

#include "tmpm_internal.h"

namespace tmpm {

namespace {

struct Q4 {
    float x, y, z, w;
};
struct R3 {
    float x, y, z;
};

__device__ __forceinline__ R3 r3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ R3 add3(R3 a, R3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ R3 sub3(R3 a, R3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ R3 mul3(R3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ R3 had3(R3 a, R3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ float dot3(R3 a, R3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ R3 cross3(R3 a, R3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// v rotated by the unit quaternion q: v + w t + q_v x t with t = 2 q_v x v.
__device__ __forceinline__ R3 rotate(Q4 q, R3 v) {
    const R3 u = r3(q.x, q.y, q.z);
    const R3 t = mul3(cross3(u, v), 2.0f);
    return add3(add3(v, mul3(t, q.w)), cross3(u, t));
}

// Hamilton product a b.
__device__ __forceinline__ Q4 qmul(Q4 a, Q4 b) {
    const R3 av = r3(a.x, a.y, a.z), bv = r3(b.x, b.y, b.z);
    const R3 v = add3(add3(mul3(bv, a.w), mul3(av, b.w)), cross3(av, bv));
    return {v.x, v.y, v.z, a.w * b.w - dot3(av, bv)};
}

__device__ __forceinline__ Q4 qnormalize(Q4 q) {
    const float s = rsqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    return {q.x * s, q.y * s, q.z * s, q.w * s};
}

// Rotation by the vector r (axis r / |r|, angle |r|); first order below 1e-5 rad.
__device__ __forceinline__ Q4 quat_from_rotation(R3 r) {
    const float angle = sqrtf(dot3(r, r));
    if (angle < 1e-5f) return qnormalize({0.5f * r.x, 0.5f * r.y, 0.5f * r.z, 1.0f});
    const float s = sinf(0.5f * angle) / angle;
    return {r.x * s, r.y * s, r.z * s, cosf(0.5f * angle)};
}

__global__ void k_rigid_sync(const DevRigid *__restrict__ bodies, const DevRigidMap *__restrict__ maps, int count,
                             DevObstacle *obstacles) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const DevRigidMap m = maps[i];
    if (m.body < 0) return;
    const DevRigid b = bodies[m.body];
    const Q4 q = {b.q.x, b.q.y, b.q.z, b.q.w};
    const R3 offset = rotate(q, r3(m.local_center.x, m.local_center.y, m.local_center.z));
    DevObstacle &o = obstacles[i];
    o.center[0] = b.pos_inv_mass.x + offset.x;
    o.center[1] = b.pos_inv_mass.y + offset.y;
    o.center[2] = b.pos_inv_mass.z + offset.z;
    const Q4 oq = qmul(q, {m.local_q.x, m.local_q.y, m.local_q.z, m.local_q.w});
    o.q[0] = oq.x;
    o.q[1] = oq.y;
    o.q[2] = oq.z;
    o.q[3] = oq.w;
    const R3 w = r3(b.ang.x, b.ang.y, b.ang.z);
    const R3 v = add3(r3(b.lin.x, b.lin.y, b.lin.z), cross3(w, offset));
    o.lin[0] = v.x;
    o.lin[1] = v.y;
    o.lin[2] = v.z;
    o.ang[0] = w.x;
    o.ang[1] = w.y;
    o.ang[2] = w.z;
}

__global__ void k_rigid_apply(DevRigid *bodies, int body_count, const DevRigidMap *__restrict__ maps, int obstacle_count,
                              const DevObstacle *__restrict__ obstacles, const double *__restrict__ reactions,
                              RigidParams p) {
    const int bi = blockIdx.x * blockDim.x + threadIdx.x;
    if (bi >= body_count) return;
    DevRigid b = bodies[bi];
    const float inv_mass = b.pos_inv_mass.w;
    if (inv_mass <= 0.0f) return;
    const R3 pos = r3(b.pos_inv_mass.x, b.pos_inv_mass.y, b.pos_inv_mass.z);
    R3 lin = r3(0.f, 0.f, 0.f), ang = r3(0.f, 0.f, 0.f);
    bool mapped = false;
    for (int oi = 0; oi < obstacle_count; ++oi) {
        if (maps[oi].body != bi) continue;
        mapped = true;
        const double *r = reactions + 6 * oi;
        const R3 imp = r3(static_cast<float>(r[0]), static_cast<float>(r[1]), static_cast<float>(r[2]));
        lin = add3(lin, imp);
        const R3 c = r3(obstacles[oi].center[0], obstacles[oi].center[1], obstacles[oi].center[2]);
        ang = add3(add3(ang, r3(static_cast<float>(r[3]), static_cast<float>(r[4]), static_cast<float>(r[5]))),
                   cross3(sub3(c, pos), imp));
    }
    const bool finite = fabsf(lin.x) < 1e30f && fabsf(lin.y) < 1e30f && fabsf(lin.z) < 1e30f &&
                        fabsf(ang.x) < 1e30f && fabsf(ang.y) < 1e30f && fabsf(ang.z) < 1e30f;
    if (!finite || !mapped) return;
    if (dot3(lin, lin) == 0.0f && dot3(ang, ang) == 0.0f && !p.integrate_pose) return;
    const Q4 q = {b.q.x, b.q.y, b.q.z, b.q.w};
    const Q4 conj = {-q.x, -q.y, -q.z, q.w};
    const R3 torque_body = rotate(conj, ang);
    const R3 dw = rotate(q, had3(torque_body, r3(b.inv_inertia.x, b.inv_inertia.y, b.inv_inertia.z)));
    R3 v = add3(r3(b.lin.x, b.lin.y, b.lin.z), mul3(lin, inv_mass));
    const R3 w = add3(r3(b.ang.x, b.ang.y, b.ang.z), dw);
    b.inv_inertia.w = 0.0f;  // awake
    if (p.integrate_pose) v = add3(v, mul3(r3(p.gravity[0], p.gravity[1], p.gravity[2]), p.dt));
    if (p.max_speed > 0.0f) {
        const float speed = sqrtf(dot3(v, v));
        if (speed > p.max_speed) v = mul3(v, p.max_speed / speed);
    }
    b.lin.x = v.x;
    b.lin.y = v.y;
    b.lin.z = v.z;
    b.ang.x = w.x;
    b.ang.y = w.y;
    b.ang.z = w.z;
    if (p.integrate_pose) {
        b.pos_inv_mass.x = pos.x + v.x * p.dt;
        b.pos_inv_mass.y = pos.y + v.y * p.dt;
        b.pos_inv_mass.z = pos.z + v.z * p.dt;
        const Q4 nq = qnormalize(qmul(quat_from_rotation(mul3(w, p.dt)), q));
        b.q = make_float4(nq.x, nq.y, nq.z, nq.w);
    }
    bodies[bi] = b;
}

}  // namespace

void launch_rigid_sync(const DevRigid *bodies, const DevRigidMap *maps, int obstacle_count, DevObstacle *obstacles,
                       cudaStream_t stream) {
    if (obstacle_count <= 0) return;
    k_rigid_sync<<<(obstacle_count + 63) / 64, 64, 0, stream>>>(bodies, maps, obstacle_count, obstacles);
}

void launch_rigid_apply(DevRigid *bodies, int body_count, const DevRigidMap *maps, int obstacle_count,
                        const DevObstacle *obstacles, const double *reactions, const RigidParams &p,
                        cudaStream_t stream) {
    if (body_count <= 0) return;
    k_rigid_apply<<<(body_count + 63) / 64, 64, 0, stream>>>(bodies, body_count, maps, obstacle_count, obstacles,
                                                             reactions, p);
}

}  // namespace tmpm

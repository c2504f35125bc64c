// SPDX-License-Identifier: Apache-2.0
//
// The body passes of the soft step, one body per lane (engine/physics/src/solver.c):
// prepare_body (131-168), integrate_velocity with the implicit gyroscopic step (176-259),
// integrate_position (261-270), and the GPU part of finalize_body (304-324): the pose, the
// velocities, cleared force and torque, the sleep timer. Continuous collision and the
// broadphase boxes stay with the host.
//
// Integration reads per body six rows itg[6i + r]:
//   0 linear_accel.xyz, linear_damping      1 angular_accel.xyz, angular_damping
//   2 q0 (the rotation at the step's start)  3 inertia_local c0, max_angular_speed_sq
//   4 inertia_local c1, max_linear_speed_sq 5 inertia_local c2, flags | locks << 8
// and prm[3i + 1].w is 1 for a dynamic body (the constraints' prepare reads it there).
#pragma once

#include "layout.cuh"

namespace nph {

constexpr uint32_t kParamDynamic = 1u;    // PHYS_PARAM_DYNAMIC
constexpr uint32_t kParamGyroscopic = 2u; // PHYS_PARAM_GYROSCOPIC

struct BodyArrays {
    float4 *vel;
    float4 *pos;
    float4 *prm;
    float4 *itg;
};

// solver.c:103-117.
NPH_D M3 lock_inertia(M3 m, uint32_t locks)
{
    if ((locks & NPH_GPU_LOCK_ANGULAR_X) != 0u) {
        m.c0 = v3(0.f, 0.f, 0.f);
        m.c0.x = 0.f;
        m.c1.x = 0.f;
        m.c2.x = 0.f;
    }
    if ((locks & NPH_GPU_LOCK_ANGULAR_Y) != 0u) {
        m.c1 = v3(0.f, 0.f, 0.f);
        m.c0.y = 0.f;
        m.c1.y = 0.f;
        m.c2.y = 0.f;
    }
    if ((locks & NPH_GPU_LOCK_ANGULAR_Z) != 0u) {
        m.c2 = v3(0.f, 0.f, 0.f);
        m.c0.z = 0.f;
        m.c1.z = 0.f;
        m.c2.z = 0.f;
    }
    return m;
}

// solver.c:123-129.
NPH_D bool inertia_is_isotropic(const float *m)
{
    const float tol = 1e-6f * (fabsf(m[0]) + fabsf(m[4]) + fabsf(m[8]));
    return fabsf(m[4] - m[0]) <= tol && fabsf(m[8] - m[0]) <= tol && fabsf(m[1]) <= tol &&
           fabsf(m[2]) <= tol && fabsf(m[5]) <= tol;
}

NPH_D M3 load_m3(const float *p)
{
    return M3{v3(p[0], p[1], p[2]), v3(p[3], p[4], p[5]), v3(p[6], p[7], p[8])};
}

// solver.c:131-168: solver body i (an awake body's record) and its parameters.
NPH_D void prepare_body(const BodyArrays &B, uint32_t i, const NphGpuBody &b, const StepConsts &K)
{
    B.vel[2u * i] = make_float4(b.linear_velocity[0], b.linear_velocity[1], b.linear_velocity[2], 0.f);
    B.vel[2u * i + 1u] = make_float4(b.angular_velocity[0], b.angular_velocity[1], b.angular_velocity[2], 0.f);
    B.pos[2u * i] = make_float4(0.f, 0.f, 0.f, 0.f);
    B.pos[2u * i + 1u] = make_float4(0.f, 0.f, 0.f, 1.f);
    const Q4 q = Q4{b.rotation[0], b.rotation[1], b.rotation[2], b.rotation[3]};
    uint32_t flags = 0u;
    V3 la = v3(0.f, 0.f, 0.f);
    V3 aa = v3(0.f, 0.f, 0.f);
    float ld = 0.f;
    float ad = 0.f;
    M3 ii = m_zero();
    M3 il = m_zero();
    float inv_mass = 0.f;
    if (b.type == NPH_GPU_BODY_DYNAMIC) {
        flags = kParamDynamic;
        if ((b.flags & NPH_GPU_BODY_GYROSCOPIC) != 0u && !inertia_is_isotropic(b.inertia)) {
            flags |= kParamGyroscopic;
        }
        const V3 g = v3(K.gravity[0], K.gravity[1], K.gravity[2]);
        la = add(scale(g, b.gravity_scale), scale(v3(b.force[0], b.force[1], b.force[2]), b.inv_mass));
        const M3 r = M3{axis_x(q), axis_y(q), axis_z(q)};
        ii = lock_inertia(m_mul(m_mul(r, load_m3(b.inv_inertia)), m_transpose(r)), b.locks);
        aa = m_mul_v(ii, v3(b.torque[0], b.torque[1], b.torque[2]));
        il = load_m3(b.inertia);
        ld = 1.0f / (1.0f + K.h * b.linear_damping);
        ad = 1.0f / (1.0f + K.h * b.angular_damping);
        inv_mass = b.inv_mass;
    }
    B.prm[3u * i + 0u] = f4(ii.c0, inv_mass);
    B.prm[3u * i + 1u] = f4(ii.c1, (flags & kParamDynamic) != 0u ? 1.f : 0.f);
    B.prm[3u * i + 2u] = f4(ii.c2, 0.f);
    B.itg[6u * i + 0u] = f4(la, ld);
    B.itg[6u * i + 1u] = f4(aa, ad);
    B.itg[6u * i + 2u] = f4(q);
    B.itg[6u * i + 3u] = f4(il.c0, K.max_angular_speed_sq);
    B.itg[6u * i + 4u] = f4(il.c1, K.max_linear_speed_sq);
    B.itg[6u * i + 5u] = f4(il.c2, __uint_as_float(flags | (b.locks << 8)));
}

// The dummy: at rest, identity rotation, no mass (solver.c:971-973).
NPH_D void prepare_dummy(const BodyArrays &B, uint32_t n)
{
    B.vel[2u * n] = make_float4(0.f, 0.f, 0.f, 0.f);
    B.vel[2u * n + 1u] = make_float4(0.f, 0.f, 0.f, 0.f);
    B.pos[2u * n] = make_float4(0.f, 0.f, 0.f, 0.f);
    B.pos[2u * n + 1u] = make_float4(0.f, 0.f, 0.f, 1.f);
    B.prm[3u * n + 0u] = make_float4(0.f, 0.f, 0.f, 0.f);
    B.prm[3u * n + 1u] = make_float4(0.f, 0.f, 0.f, 0.f);
    B.prm[3u * n + 2u] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// solver.c:176-202.
NPH_D V3 gyroscopic(V3 w_world, Q4 q, const M3 &inertia, float h)
{
    const V3 w = rotate(q_conj(q), w_world);
    const V3 iw = m_mul_v(inertia, w);
    const V3 f = scale(cross(w, iw), h);
    const V3 j0 = mul_add(inertia.c0, sub(cross(w, inertia.c0), cross(iw, v3(1.f, 0.f, 0.f))), h);
    const V3 j1 = mul_add(inertia.c1, sub(cross(w, inertia.c1), cross(iw, v3(0.f, 1.f, 0.f))), h);
    const V3 j2 = mul_add(inertia.c2, sub(cross(w, inertia.c2), cross(iw, v3(0.f, 0.f, 1.f))), h);
    const V3 c12 = cross(j1, j2);
    const float det = dot(j0, c12);
    if (!(det > 0.0f)) {
        return w_world;
    }
    const float inv_det = 1.0f / det;
    const V3 x = v3(dot(f, c12) * inv_det, dot(j0, cross(f, j2)) * inv_det,
                    dot(j0, cross(j1, f)) * inv_det);
    return rotate(q, sub(w, x));
}

NPH_D V3 lock_linear(V3 v, uint32_t locks)
{
    if ((locks & NPH_GPU_LOCK_LINEAR_X) != 0u) v.x = 0.f;
    if ((locks & NPH_GPU_LOCK_LINEAR_Y) != 0u) v.y = 0.f;
    if ((locks & NPH_GPU_LOCK_LINEAR_Z) != 0u) v.z = 0.f;
    return v;
}

NPH_D V3 lock_angular(V3 w, uint32_t locks)
{
    if ((locks & NPH_GPU_LOCK_ANGULAR_X) != 0u) w.x = 0.f;
    if ((locks & NPH_GPU_LOCK_ANGULAR_Y) != 0u) w.y = 0.f;
    if ((locks & NPH_GPU_LOCK_ANGULAR_Z) != 0u) w.z = 0.f;
    return w;
}

// solver.c:232-259.
NPH_D void integrate_velocity(const BodyArrays &B, uint32_t i, float h)
{
    const float4 r5 = B.itg[6u * i + 5u];
    const uint32_t bits = __float_as_uint(r5.w);
    if ((bits & kParamDynamic) == 0u) {
        return; // kinematic: moves by its velocity only
    }
    const uint32_t locks = bits >> 8;
    const float4 r0 = B.itg[6u * i + 0u];
    const float4 r1 = B.itg[6u * i + 1u];
    const float4 r3 = B.itg[6u * i + 3u];
    const float4 r4 = B.itg[6u * i + 4u];
    const BodyState s = load_state(B.vel, i);
    V3 v = scale(mul_add(s.v, v3(r0), h), r0.w);
    V3 av = scale(mul_add(s.w, v3(r1), h), r1.w);
    if ((bits & kParamGyroscopic) != 0u) {
        const Q4 q0 = q4(B.itg[6u * i + 2u]);
        const Q4 dq = q4(B.pos[2u * i + 1u]);
        av = gyroscopic(av, q_mul(dq, q0), M3{v3(r3), v3(r4), v3(r5)}, h);
    }
    const float v_sq = dot(v, v);
    if (v_sq > r4.w) {
        v = scale(v, sqrtf(r4.w / v_sq));
    }
    const float w_sq = dot(av, av);
    if (w_sq > r3.w) {
        av = scale(av, sqrtf(r3.w / w_sq));
    }
    store_state(B.vel, i, BodyState{lock_linear(v, locks), lock_angular(av, locks)});
}

// solver.c:261-270.
NPH_D void integrate_position(const BodyArrays &B, uint32_t i, float h)
{
    const uint32_t locks = __float_as_uint(B.itg[6u * i + 5u].w) >> 8;
    BodyState s = load_state(B.vel, i);
    s.v = lock_linear(s.v, locks);
    s.w = lock_angular(s.w, locks);
    if (locks != 0u) {
        store_state(B.vel, i, s);
    }
    const BodyPose p = load_pose(B.pos, i);
    const V3 dp = mul_add(p.dp, s.v, h);
    const Q4 dq = q_integrate(p.dq, s.w, h);
    B.pos[2u * i] = f4(dp, 0.f);
    B.pos[2u * i + 1u] = f4(dq);
}

// finalize_body, solver.c:304-324 (continuous collision and boxes excluded).
NPH_D void finalize_body(const BodyArrays &B, uint32_t i, NphGpuBody &b, float dt)
{
    const BodyState s = load_state(B.vel, i);
    const BodyPose p = load_pose(B.pos, i);
    const Q4 q0 = q4(B.itg[6u * i + 2u]);
    b.linear_velocity[0] = s.v.x;
    b.linear_velocity[1] = s.v.y;
    b.linear_velocity[2] = s.v.z;
    b.angular_velocity[0] = s.w.x;
    b.angular_velocity[1] = s.w.y;
    b.angular_velocity[2] = s.w.z;
    const Q4 q = q_normalize(q_mul(p.dq, q0));
    b.rotation[0] = q.x;
    b.rotation[1] = q.y;
    b.rotation[2] = q.z;
    b.rotation[3] = q.w;
    const double cx = b.center[0] + (double)p.dp.x;
    const double cy = b.center[1] + (double)p.dp.y;
    const double cz = b.center[2] + (double)p.dp.z;
    b.center[0] = cx;
    b.center[1] = cy;
    b.center[2] = cz;
    const V3 rc = rotate(q, v3(b.local_center[0], b.local_center[1], b.local_center[2]));
    b.origin[0] = cx + (double)(-rc.x);
    b.origin[1] = cy + (double)(-rc.y);
    b.origin[2] = cz + (double)(-rc.z);
    b.force[0] = 0.f;
    b.force[1] = 0.f;
    b.force[2] = 0.f;
    b.torque[0] = 0.f;
    b.torque[1] = 0.f;
    b.torque[2] = 0.f;
    const float speed = fmax_ref(length(s.v), b.max_extent * length(s.w));
    if ((b.flags & NPH_GPU_BODY_ENABLE_SLEEP) == 0u || speed > b.sleep_threshold) {
        b.sleep_time = 0.0f;
    } else {
        b.sleep_time = b.sleep_time + dt;
    }
}

} // namespace nph

// SPDX-License-Identifier: Apache-2.0
//
// Ball and hinge joints, one joint per lane (engine/physics/src/joint_solver.c): prepare
// (726-771), warm start (826-868), and the soft or rigid solve (870-897) with the ball's
// friction, cone and twist limits (341-394) and the hinge's spring, motor, limits and axis
// lock (264-336), each ending in the point block (207-230). The reference keeps joints
// scalar, so every formula here is its scalar formula in its order. Joints of a colour share
// no dynamic body with each other or with the colour's contacts, so a colour's joints run
// in parallel. The angle of a hinge limit or spring and of a ball cone or twist limit is the
// correctly rounded FP32 arctangent (the double-precision atan2 rounded once to FP32): the
// reference's is the host C library's atan2f, which is not correctly rounded, so those rows
// match the reference within floating-point tolerance, the others bit for bit.
#pragma once

#include "layout.cuh"

namespace nph {

struct JointBodies {
    uint32_t sa, sb;
    bool wa, wb;
    float ma, mb;
    M3 ia, ib;
    BodyState a, b;
    BodyPose pa, pb;
};

// joint_solver.c:114-133: the anchors and frames now.
struct JointNow {
    V3 ra, rb;
    Q4 qa, qb;
};

NPH_D float4 jrow(const DevSolver &S, uint32_t r, uint32_t j) { return S.jw[r * S.jcap + j]; }
NPH_D void jset(const DevSolver &S, uint32_t r, uint32_t j, float4 v) { S.jw[r * S.jcap + j] = v; }

// joint_solver.c:32-42.
NPH_D V3 solve3(V3 k0, V3 k1, V3 k2, V3 b)
{
    const V3 c12 = cross(k1, k2);
    const float det = dot(k0, c12);
    if (!(det > 0.0f)) {
        return v3(0.0f, 0.0f, 0.0f);
    }
    const float inv = 1.0f / det;
    return v3(dot(b, c12) * inv, dot(k0, cross(b, k2)) * inv, dot(k0, cross(k1, b)) * inv);
}

// joint_solver.c:68-73.
NPH_D float axial_mass(const JointBodies &jb, V3 axis)
{
    const float k = dot(axis, m_mul_v(jb.ia, axis)) + dot(axis, m_mul_v(jb.ib, axis));
    return k > 0.0f ? 1.0f / k : 0.0f;
}

// atan2(y, x) rounded once to FP32 from the double-precision value.
NPH_D float atan2_rn(float y, float x) { return (float)atan2((double)y, (double)x); }

// joint_solver.c:77-84.
NPH_D float twist_angle(Q4 qa, Q4 qb)
{
    Q4 r = q_mul(q_conj(qa), qb);
    if (r.w < 0.0f) {
        r = Q4{-r.x, -r.y, -r.z, -r.w};
    }
    return 2.0f * atan2_rn(r.x, r.w);
}

// joint_solver.c:86-96.
NPH_D float unwind(float a)
{
    const float pi = 3.14159265f;
    if (a > pi) {
        return a - 2.0f * pi;
    }
    if (a < -pi) {
        return a + 2.0f * pi;
    }
    return a;
}

// joint_solver.c:136-148.
NPH_D void apply_linear(JointBodies &jb, const JointNow &s, V3 p)
{
    if (jb.wa) {
        jb.a.v = mul_add(jb.a.v, p, -jb.ma);
        jb.a.w = sub(jb.a.w, m_mul_v(jb.ia, cross(s.ra, p)));
    }
    if (jb.wb) {
        jb.b.v = mul_add(jb.b.v, p, jb.mb);
        jb.b.w = add(jb.b.w, m_mul_v(jb.ib, cross(s.rb, p)));
    }
}

// joint_solver.c:151-159.
NPH_D void apply_angular(JointBodies &jb, V3 l)
{
    if (jb.wa) {
        jb.a.w = sub(jb.a.w, m_mul_v(jb.ia, l));
    }
    if (jb.wb) {
        jb.b.w = add(jb.b.w, m_mul_v(jb.ib, l));
    }
}

NPH_D V3 relative_angular(const JointBodies &jb) { return sub(jb.b.w, jb.a.w); }

NPH_D JointBodies load_joint_bodies(const DevSolver &S, uint32_t sa, uint32_t sb, uint32_t flags)
{
    JointBodies jb;
    jb.sa = sa;
    jb.sb = sb;
    jb.wa = (flags & kJWriteA) != 0u;
    jb.wb = (flags & kJWriteB) != 0u;
    // prm is zero for bodies that are not dynamic: the reference's dyn ? .. : 0
    // (joint_solver.c:736-739).
    jb.ia = load_inv_inertia(S.prm, sa, &jb.ma);
    jb.ib = load_inv_inertia(S.prm, sb, &jb.mb);
    jb.a = load_state(S.vel, sa);
    jb.b = load_state(S.vel, sb);
    jb.pa = load_pose(S.pos, sa);
    jb.pb = load_pose(S.pos, sb);
    return jb;
}

NPH_D void store_joint_bodies(const DevSolver &S, const JointBodies &jb)
{
    if (jb.wa) {
        store_state(S.vel, jb.sa, jb.a);
    }
    if (jb.wb) {
        store_state(S.vel, jb.sb, jb.b);
    }
}

NPH_D JointNow joint_now(const DevSolver &S, uint32_t j, const JointBodies &jb)
{
    JointNow s;
    s.ra = rotate(jb.pa.dq, v3(jrow(S, kJrAnchorA, j)));
    s.rb = rotate(jb.pb.dq, v3(jrow(S, kJrAnchorB, j)));
    s.qa = q_mul(jb.pa.dq, q4(jrow(S, kJrFrameA, j)));
    s.qb = q_mul(jb.pb.dq, q4(jrow(S, kJrFrameB, j)));
    return s;
}

// joint_solver.c:726-771 (ball and hinge). `a`/`b` are the bodies' records; `sa`/`sb` their
// solver slots. Returns the joint's flags.
NPH_D void prepare_joint(const DevSolver &S, uint32_t j, const NphGpuJoint &jr,
                         const NphGpuBody &a, const NphGpuBody &b, uint32_t sa, uint32_t sb,
                         float h)
{
    const bool dyn_a = a.type == NPH_GPU_BODY_DYNAMIC;
    const bool dyn_b = b.type == NPH_GPU_BODY_DYNAMIC;
    uint32_t flags = (dyn_a ? kJWriteA : 0u) | (dyn_b ? kJWriteB : 0u);
    const Q4 qa = Q4{a.rotation[0], a.rotation[1], a.rotation[2], a.rotation[3]};
    const Q4 qb = Q4{b.rotation[0], b.rotation[1], b.rotation[2], b.rotation[3]};
    const V3 fa = v3(jr.frame_a_position[0], jr.frame_a_position[1], jr.frame_a_position[2]);
    const V3 fb = v3(jr.frame_b_position[0], jr.frame_b_position[1], jr.frame_b_position[2]);
    const V3 lca = v3(a.local_center[0], a.local_center[1], a.local_center[2]);
    const V3 lcb = v3(b.local_center[0], b.local_center[1], b.local_center[2]);
    const V3 anchor_a = rotate(qa, sub(fa, lca));
    const V3 anchor_b = rotate(qb, sub(fb, lcb));
    // nph_dvec3_relative (vec.h:991-994): the 64-bit difference rounded to 32 bits.
    const V3 delta = v3((float)(b.center[0] - a.center[0]), (float)(b.center[1] - a.center[1]),
                        (float)(b.center[2] - a.center[2]));
    const Q4 fqa = q_mul(qa, Q4{jr.frame_a_rotation[0], jr.frame_a_rotation[1],
                                jr.frame_a_rotation[2], jr.frame_a_rotation[3]});
    const Q4 fqb = q_mul(qb, Q4{jr.frame_b_rotation[0], jr.frame_b_rotation[1],
                                jr.frame_b_rotation[2], jr.frame_b_rotation[3]});
    float4 lin = make_float4(jr.linear_impulse[0], jr.linear_impulse[1], jr.linear_impulse[2],
                             jr.lower_impulse);
    float4 ang = make_float4(jr.angular_impulse[0], jr.angular_impulse[1], jr.angular_impulse[2],
                             jr.upper_impulse);
    float4 fric = make_float4(jr.friction_impulse[0], jr.friction_impulse[1],
                              jr.friction_impulse[2], jr.swing_impulse);
    float4 mot = make_float4(jr.motor_impulse, jr.spring_impulse, 0.0f, 0.0f);
    Soft spring = Soft{0.0f, 1.0f, 0.0f};
    float4 set_a = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 set_b = make_float4(0.f, 0.f, 0.f, 0.f);
    if (jr.type == NPH_GPU_JOINT_HINGE) {
        const NphGpuHingeJoint &hj = jr.u.hinge;
        flags |= kJHinge;
        flags |= hj.enable_limit != 0u ? kJLimit : 0u;
        flags |= hj.enable_motor != 0u ? kJMotor : 0u;
        flags |= hj.enable_spring != 0u ? kJSpring : 0u;
        if (hj.enable_motor != 0u && hj.motor_speed != 0.0f && hj.max_motor_torque > 0.0f) {
            flags |= kJDriven; // phys_joint_is_driven, joint_solver.c:1410-1415
        }
        if (hj.enable_limit == 0u) {
            lin.w = 0.0f;
            ang.w = 0.0f;
        }
        if (hj.enable_motor == 0u) {
            mot.x = 0.0f;
        }
        if (hj.enable_spring == 0u) {
            mot.y = 0.0f;
        }
        spring = make_soft(hj.enable_spring != 0u ? hj.spring_hertz : 0.0f,
                           hj.spring_damping_ratio, h);
        set_a = make_float4(hj.lower, hj.upper, hj.motor_speed, hj.max_motor_torque);
        set_b = make_float4(hj.spring_target, 0.0f, 0.0f, 0.0f);
    } else {
        const NphGpuBallJoint &bj = jr.u.ball;
        flags |= bj.enable_swing_limit != 0u ? kJSwing : 0u;
        flags |= bj.enable_twist_limit != 0u ? kJTwist : 0u;
        flags |= bj.friction_torque > 0.0f ? kJFriction : 0u;
        if (bj.enable_swing_limit == 0u) {
            fric.w = 0.0f;
        }
        if (bj.enable_twist_limit == 0u) {
            lin.w = 0.0f;
            ang.w = 0.0f;
        }
        if (!(bj.friction_torque > 0.0f)) {
            fric.x = 0.0f;
            fric.y = 0.0f;
            fric.z = 0.0f;
        }
        set_a = make_float4(bj.swing_y, bj.swing_z, bj.twist_lower, bj.twist_upper);
        set_b = make_float4(bj.friction_torque, 0.0f, 0.0f, 0.0f);
    }
    jset(S, kJrHead, j, make_float4(__uint_as_float(sa), __uint_as_float(sb), __uint_as_float(flags), 0.0f));
    jset(S, kJrAnchorA, j, f4(anchor_a, 0.0f));
    jset(S, kJrAnchorB, j, f4(anchor_b, 0.0f));
    jset(S, kJrDelta, j, f4(delta, 0.0f));
    jset(S, kJrFrameA, j, f4(fqa));
    jset(S, kJrFrameB, j, f4(fqb));
    jset(S, kJrSpring, j, make_float4(spring.bias_rate, spring.mass_scale, spring.impulse_scale, 0.0f));
    jset(S, kJrSetA, j, set_a);
    jset(S, kJrSetB, j, set_b);
    jset(S, kJrLinear, j, lin);
    jset(S, kJrAngular, j, ang);
    jset(S, kJrFric, j, fric);
    jset(S, kJrMotor, j, mot);
}

NPH_D void joint_head(const DevSolver &S, uint32_t j, uint32_t &sa, uint32_t &sb, uint32_t &flags)
{
    const float4 h = jrow(S, kJrHead, j);
    sa = __float_as_uint(h.x);
    sb = __float_as_uint(h.y);
    flags = __float_as_uint(h.z);
}

// joint_solver.c:826-868.
NPH_D void warm_joint(const DevSolver &S, uint32_t j)
{
    uint32_t sa, sb, flags;
    joint_head(S, j, sa, sb, flags);
    JointBodies jb = load_joint_bodies(S, sa, sb, flags);
    const JointNow s = joint_now(S, j, jb);
    const float4 lin = jrow(S, kJrLinear, j);
    const float4 angr = jrow(S, kJrAngular, j);
    const float4 fric = jrow(S, kJrFric, j);
    V3 angular;
    if ((flags & kJHinge) != 0u) {
        const float4 mot = jrow(S, kJrMotor, j);
        angular = add(scale(axis_y(s.qa), angr.x), scale(axis_z(s.qa), angr.y));
        const float axial = lin.w - angr.w + mot.x + mot.y;
        angular = mul_add(angular, axis_x(s.qa), axial);
    } else {
        angular = v3(fric);
        const V3 xa = axis_x(s.qa);
        const V3 xb = axis_x(s.qb);
        const V3 n = cross(xa, xb);
        const float sin_phi = length(n);
        if (fric.w != 0.0f && sin_phi > 1e-6f) {
            angular = mul_add(angular, n, -fric.w / sin_phi);
        }
        const V3 sum = add(xa, xb);
        const float len = length(sum);
        if (len > 1e-3f) {
            angular = mul_add(angular, sum, (lin.w - angr.w) / len);
        }
    }
    apply_angular(jb, angular);
    apply_linear(jb, s, v3(lin));
    store_joint_bodies(S, jb);
}

// joint_solver.c:178-204.
NPH_D void solve_angular_limit(JointBodies &jb, V3 axis, float c, float &accumulated,
                               const StepConsts &K, bool use_bias)
{
    float bias = 0.0f;
    float mass_scale = 1.0f;
    float impulse_scale = 0.0f;
    if (c > 0.0f) {
        bias = c * K.inv_h;
    } else if (use_bias) {
        bias = K.joint_soft.bias_rate * c;
        mass_scale = K.joint_soft.mass_scale;
        impulse_scale = K.joint_soft.impulse_scale;
    }
    const float cdot = -dot(relative_angular(jb), axis);
    const float impulse = -axial_mass(jb, axis) * mass_scale * (cdot + bias) - impulse_scale * accumulated;
    const float total = fmax_ref(accumulated + impulse, 0.0f);
    const float delta = total - accumulated;
    accumulated = total;
    apply_angular(jb, scale(axis, -delta));
}

// joint_solver.c:207-230.
NPH_D void solve_point(JointBodies &jb, const JointNow &s, V3 delta_center, V3 &linear_impulse,
                       const StepConsts &K, bool use_bias)
{
    const V3 va = add(jb.a.v, cross(jb.a.w, s.ra));
    const V3 vb = add(jb.b.v, cross(jb.b.w, s.rb));
    const V3 cdot = sub(vb, va);
    V3 bias = v3(0.0f, 0.0f, 0.0f);
    float mass_scale = 1.0f;
    float impulse_scale = 0.0f;
    if (use_bias) {
        const V3 c = add(add(sub(jb.pb.dp, jb.pa.dp), sub(s.rb, s.ra)), delta_center);
        bias = scale(c, K.joint_soft.bias_rate);
        mass_scale = K.joint_soft.mass_scale;
        impulse_scale = K.joint_soft.impulse_scale;
    }
    // point_mass, joint_solver.c:46-57.
    const float m = jb.ma + jb.mb;
    const V3 e0 = v3(1.0f, 0.0f, 0.0f);
    const V3 e1 = v3(0.0f, 1.0f, 0.0f);
    const V3 e2 = v3(0.0f, 0.0f, 1.0f);
    const V3 k0 = sub(sub(scale(e0, m), cross(s.ra, m_mul_v(jb.ia, cross(s.ra, e0)))),
                      cross(s.rb, m_mul_v(jb.ib, cross(s.rb, e0))));
    const V3 k1 = sub(sub(scale(e1, m), cross(s.ra, m_mul_v(jb.ia, cross(s.ra, e1)))),
                      cross(s.rb, m_mul_v(jb.ib, cross(s.rb, e1))));
    const V3 k2 = sub(sub(scale(e2, m), cross(s.ra, m_mul_v(jb.ia, cross(s.ra, e2)))),
                      cross(s.rb, m_mul_v(jb.ib, cross(s.rb, e2))));
    const V3 x = solve3(k0, k1, k2, add(cdot, bias));
    const V3 impulse = sub(scale(x, -mass_scale), scale(linear_impulse, impulse_scale));
    linear_impulse = add(linear_impulse, impulse);
    apply_linear(jb, s, impulse);
}

// joint_solver.c:264-301.
NPH_D void solve_axis_lock(JointBodies &jb, const JointNow &s, float4 &angr, const StepConsts &K,
                           bool use_bias)
{
    const V3 p1 = axis_y(s.qa);
    const V3 p2 = axis_z(s.qa);
    const V3 dw = relative_angular(jb);
    float c1 = 0.0f;
    float c2 = 0.0f;
    float mass_scale = 1.0f;
    float impulse_scale = 0.0f;
    if (use_bias) {
        const V3 e = cross(axis_x(s.qa), axis_x(s.qb));
        c1 = K.joint_soft.bias_rate * dot(e, p1);
        c2 = K.joint_soft.bias_rate * dot(e, p2);
        mass_scale = K.joint_soft.mass_scale;
        impulse_scale = K.joint_soft.impulse_scale;
    }
    const V3 ip1 = add(m_mul_v(jb.ia, p1), m_mul_v(jb.ib, p1));
    const V3 ip2 = add(m_mul_v(jb.ia, p2), m_mul_v(jb.ib, p2));
    const float k11 = dot(p1, ip1);
    const float k12 = dot(p1, ip2);
    const float k22 = dot(p2, ip2);
    const float det = k11 * k22 - k12 * k12;
    if (!(det > 0.0f)) {
        return;
    }
    const float inv = 1.0f / det;
    const float b1 = dot(dw, p1) + c1;
    const float b2 = dot(dw, p2) + c2;
    const float x1 = (k22 * b1 - k12 * b2) * inv;
    const float x2 = (k11 * b2 - k12 * b1) * inv;
    const float i1 = -mass_scale * x1 - impulse_scale * angr.x;
    const float i2 = -mass_scale * x2 - impulse_scale * angr.y;
    angr.x += i1;
    angr.y += i2;
    apply_angular(jb, add(scale(p1, i1), scale(p2, i2)));
}

// joint_solver.c:870-897, ball (360-394) and hinge (303-336).
template <bool kUseBias>
NPH_D void solve_joint(const DevSolver &S, uint32_t j, const StepConsts &K)
{
    uint32_t sa, sb, flags;
    joint_head(S, j, sa, sb, flags);
    JointBodies jb = load_joint_bodies(S, sa, sb, flags);
    const JointNow s = joint_now(S, j, jb);
    float4 lin = jrow(S, kJrLinear, j);
    float4 angr = jrow(S, kJrAngular, j);
    float4 fric = jrow(S, kJrFric, j);
    float4 mot = jrow(S, kJrMotor, j);
    const float4 set_a = jrow(S, kJrSetA, j);
    if ((flags & kJHinge) != 0u) {
        const V3 axis = axis_x(s.qa);
        const bool need_angle = ((flags & kJSpring) != 0u && kUseBias) || (flags & kJLimit) != 0u;
        const float angle = need_angle ? twist_angle(s.qa, s.qb) : 0.0f;
        const float mass = axial_mass(jb, axis);
        if ((flags & kJSpring) != 0u && kUseBias) {
            const float4 sp = jrow(S, kJrSpring, j);
            const float target = jrow(S, kJrSetB, j).x;
            const float c = unwind(angle - target);
            const float cdot = dot(relative_angular(jb), axis);
            const float impulse = -sp.y * mass * (cdot + sp.x * c) - sp.z * mot.y;
            mot.y += impulse;
            apply_angular(jb, scale(axis, impulse));
        }
        if ((flags & kJMotor) != 0u) {
            const float cdot = dot(relative_angular(jb), axis) - set_a.z;
            const float max_impulse = K.h * set_a.w;
            const float old = mot.x;
            const float v = old - mass * cdot;
            mot.x = v < -max_impulse ? -max_impulse : (v > max_impulse ? max_impulse : v);
            apply_angular(jb, scale(axis, mot.x - old));
        }
        if ((flags & kJLimit) != 0u) {
            solve_angular_limit(jb, neg(axis), angle - set_a.x, lin.w, K, kUseBias);
            solve_angular_limit(jb, axis, set_a.y - angle, angr.w, K, kUseBias);
        }
        solve_axis_lock(jb, s, angr, K, kUseBias);
    } else {
        if ((flags & kJFriction) != 0u) {
            const float friction_torque = jrow(S, kJrSetB, j).x;
            const V3 k0 = add(jb.ia.c0, jb.ib.c0);
            const V3 k1 = add(jb.ia.c1, jb.ib.c1);
            const V3 k2 = add(jb.ia.c2, jb.ib.c2);
            const V3 x = solve3(k0, k1, k2, relative_angular(jb));
            const V3 old = v3(fric);
            V3 total = sub(old, x);
            const float max_impulse = K.h * friction_torque;
            const float len_sq = dot(total, total);
            if (len_sq > max_impulse * max_impulse) {
                total = scale(total, max_impulse / sqrtf(len_sq));
            }
            fric.x = total.x;
            fric.y = total.y;
            fric.z = total.z;
            apply_angular(jb, sub(total, old));
        }
        if ((flags & kJSwing) != 0u) {
            // joint_solver.c:341-358.
            const V3 xa = axis_x(s.qa);
            const V3 xb = axis_x(s.qb);
            const V3 n = cross(xa, xb);
            const float sin_phi = length(n);
            if (sin_phi > 1e-6f) {
                const V3 axis = scale(n, 1.0f / sin_phi);
                const V3 local = rotate(q_conj(s.qa), axis);
                const float ey = local.y / set_a.x;
                const float ez = local.z / set_a.y;
                const float limit = 1.0f / sqrtf(ey * ey + ez * ez);
                const float phi = atan2_rn(sin_phi, dot(xa, xb));
                solve_angular_limit(jb, axis, limit - phi, fric.w, K, kUseBias);
            }
        }
        if ((flags & kJTwist) != 0u) {
            const V3 sum = add(axis_x(s.qa), axis_x(s.qb));
            const float len = length(sum);
            if (len > 1e-3f) {
                const V3 axis = scale(sum, 1.0f / len);
                const float twist = twist_angle(s.qa, s.qb);
                solve_angular_limit(jb, neg(axis), twist - set_a.z, lin.w, K, kUseBias);
                solve_angular_limit(jb, axis, set_a.w - twist, angr.w, K, kUseBias);
            }
        }
    }
    V3 li = v3(lin);
    solve_point(jb, s, v3(jrow(S, kJrDelta, j)), li, K, kUseBias);
    lin.x = li.x;
    lin.y = li.y;
    lin.z = li.z;
    jset(S, kJrLinear, j, lin);
    jset(S, kJrAngular, j, angr);
    jset(S, kJrFric, j, fric);
    jset(S, kJrMotor, j, mot);
    store_joint_bodies(S, jb);
}

// The accumulated impulses back into the joint's record.
NPH_D void store_joint(const DevSolver &S, uint32_t j, NphGpuJoint &jr)
{
    const float4 lin = jrow(S, kJrLinear, j);
    const float4 angr = jrow(S, kJrAngular, j);
    const float4 fric = jrow(S, kJrFric, j);
    const float4 mot = jrow(S, kJrMotor, j);
    jr.linear_impulse[0] = lin.x;
    jr.linear_impulse[1] = lin.y;
    jr.linear_impulse[2] = lin.z;
    jr.angular_impulse[0] = angr.x;
    jr.angular_impulse[1] = angr.y;
    jr.angular_impulse[2] = angr.z;
    jr.friction_impulse[0] = fric.x;
    jr.friction_impulse[1] = fric.y;
    jr.friction_impulse[2] = fric.z;
    jr.lower_impulse = lin.w;
    jr.upper_impulse = angr.w;
    jr.swing_impulse = fric.w;
    jr.motor_impulse = mot.x;
    jr.spring_impulse = mot.y;
}

} // namespace nph

// SPDX-License-Identifier: Apache-2.0
//
// Joints, one joint per lane (engine/physics/src/joint_solver.c): prepare (726-824), warm
// start (826-868), and the soft or rigid solve (870-897) of all six types: the ball's
// friction, cone and twist limits (341-394); the hinge's spring, motor, limits and axis lock
// (264-336); the fixed joint's rotation lock (232-262); the slider's and 6-DOF joint's rows per
// axis with their blocks (395-682); the distance joint's line (683-720); the point block
// (207-230) last where the type has one. The reference keeps joints scalar, so every formula
// here is its scalar formula in its order. Joints of a colour share no dynamic body with each
// other or with the colour's contacts, so a colour's joints run in parallel. Every angle (a
// hinge limit or spring, a ball cone or twist limit, a 6-DOF twist or swing) goes through
// nph_atan2f (atan2f.h), the reference's C library arctangent restated in FP32 operations, so
// the angle rows round to the reference's bits like every other row.
#pragma once

#include "atan2f.h"
#include "joint_config.h"
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

// joint_solver.c:77-84.
NPH_D float twist_angle(Q4 qa, Q4 qb)
{
    Q4 r = q_mul(q_conj(qa), qb);
    if (r.w < 0.0f) {
        r = Q4{-r.x, -r.y, -r.z, -r.w};
    }
    return 2.0f * nph_atan2f(r.x, r.w);
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

// joint_solver.c:726-824, every type. `a`/`b` are the bodies' records; `sa`/`sb` their
// solver slots. Returns the joint's flags.
NPH_D void prepare_joint(const DevSolver &S, uint32_t j, const NphGpuJoint &jr,
                         const NphGpuBody &a, const NphGpuBody &b, uint32_t sa, uint32_t sb,
                         float h)
{
    const bool dyn_a = a.type == NPH_GPU_BODY_DYNAMIC;
    const bool dyn_b = b.type == NPH_GPU_BODY_DYNAMIC;
    uint32_t flags = (dyn_a ? kJWriteA : 0u) | (dyn_b ? kJWriteB : 0u) | (jr.type << kJTypeShift);
    flags |= nph_joint_is_driven(&jr) ? kJDriven : 0u;
    uint32_t axes = 0u;
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
    } else if (jr.type == NPH_GPU_JOINT_DISTANCE) {
        // joint_solver.c:772-786: what is switched off starts from nothing when switched on.
        const NphGpuDistanceJoint &dj = jr.u.distance;
        float4 imp = make_float4(jr.axis_impulse[0][0], jr.axis_impulse[0][1], jr.axis_impulse[0][2],
                                 jr.axis_impulse[0][3]);
        if (dj.enable_limit == 0u) {
            imp.y = 0.0f;
            if (dj.enable_spring != 0u) {
                imp.x = 0.0f;
            }
        }
        if (dj.enable_motor == 0u) {
            imp.z = 0.0f;
        }
        if (dj.enable_spring == 0u) {
            imp.w = 0.0f;
        }
        const uint32_t motion = dj.enable_limit != 0u    ? NPH_GPU_AXIS_LIMITED
                                : dj.enable_spring != 0u ? NPH_GPU_AXIS_FREE
                                                         : NPH_GPU_AXIS_LOCKED;
        axes = motion | (dj.enable_motor != 0u ? kJAxisMotor : 0u) |
               (dj.enable_spring != 0u ? kJAxisSpring : 0u);
        const Soft sp = dj.enable_spring != 0u ? make_soft(dj.spring_hertz, dj.spring_damping_ratio, h)
                                               : Soft{0.0f, 1.0f, 0.0f};
        jset(S, kJrAxisSet, j, make_float4(dj.min_length, dj.max_length, dj.motor_speed, h * dj.max_motor_force));
        jset(S, kJrAxisSet + 1u, j, make_float4(dj.length, sp.bias_rate, sp.mass_scale, sp.impulse_scale));
        jset(S, kJrAxisImpulse, j, imp);
    } else if (nph_joint_has_axes(jr.type)) {
        // joint_solver.c:787-822.
        NphGpuD6Axis ax[NPH_GPU_D6_AXES];
        nph_joint_axes(&jr, ax);
#pragma unroll
        for (uint32_t i = 0; i < NPH_GPU_D6_AXES; ++i) {
            const NphGpuD6Axis &x = ax[i];
            float4 imp = make_float4(jr.axis_impulse[i][0], jr.axis_impulse[i][1], jr.axis_impulse[i][2],
                                     jr.axis_impulse[i][3]);
            if (x.motion != NPH_GPU_AXIS_LIMITED) {
                imp.y = 0.0f;
            }
            if (x.motion == NPH_GPU_AXIS_FREE) {
                imp.x = 0.0f;
            }
            if (x.motion == NPH_GPU_AXIS_LOCKED || x.enable_motor == 0u) {
                imp.z = 0.0f;
            }
            if (x.motion == NPH_GPU_AXIS_LOCKED || x.enable_spring == 0u) {
                imp.w = 0.0f;
            }
            axes |= (x.motion | (x.enable_motor != 0u ? kJAxisMotor : 0u) |
                     (x.enable_spring != 0u ? kJAxisSpring : 0u))
                    << (kJAxisBits * i);
            const Soft sp = x.enable_spring != 0u ? make_soft(x.spring_hertz, x.spring_damping_ratio, h)
                                                  : Soft{0.0f, 1.0f, 0.0f};
            jset(S, kJrAxisSet + 2u * i, j, make_float4(x.lower, x.upper, x.motor_speed, h * x.max_motor_force));
            jset(S, kJrAxisSet + 2u * i + 1u, j,
                 make_float4(x.spring_target, sp.bias_rate, sp.mass_scale, sp.impulse_scale));
            jset(S, kJrAxisImpulse + i, j, imp);
        }
        // The blocks' impulses mean what their block makes them: a change of block starts
        // them from nothing.
        const uint32_t blocks = nph_joint_blocks(ax);
        const uint32_t angular_blocks = kJBlockRotation | kJBlockSwing;
        if ((jr.flags & angular_blocks) != (blocks & angular_blocks)) {
            ang.x = 0.0f;
            ang.y = 0.0f;
            ang.z = 0.0f;
        }
        if ((jr.flags & kJBlockPoint) != (blocks & kJBlockPoint)) {
            lin.x = 0.0f;
            lin.y = 0.0f;
            lin.z = 0.0f;
        }
        flags |= blocks;
    } else if (jr.type == NPH_GPU_JOINT_BALL) {
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
    jset(S, kJrHead, j,
         make_float4(__uint_as_float(sa), __uint_as_float(sb), __uint_as_float(flags), __uint_as_float(axes)));
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

NPH_D uint32_t joint_type(uint32_t flags) { return (flags >> kJTypeShift) & kJTypeMask; }
NPH_D bool joint_has_rows(uint32_t type)
{
    return type == NPH_GPU_JOINT_SLIDER || type == NPH_GPU_JOINT_D6 || type == NPH_GPU_JOINT_DISTANCE;
}

static __device__ __noinline__ void warm_row_joint(const DevSolver &S, uint32_t j);

// Which joints a pass takes: all of them in their order (the overflow's one thread, a batch's
// worlds), or, within a colour, whose joints share no dynamic body, the ball, hinge and fixed
// joints in one launch and the slider, 6-DOF and distance joints in another, so that the
// common launch keeps the registers of its own rows.
enum JointSet : int { kJointsAll = 0, kJointsPlain = 1, kJointsRows = 2 };

// joint_solver.c:826-868.
template <int kSet = kJointsAll>
NPH_D void warm_joint(const DevSolver &S, uint32_t j)
{
    uint32_t sa, sb, flags;
    joint_head(S, j, sa, sb, flags);
    const bool rows = joint_has_rows(joint_type(flags));
    if ((kSet == kJointsPlain && rows) || (kSet == kJointsRows && !rows)) {
        return;
    }
    if (kSet != kJointsPlain && rows) {
        warm_row_joint(S, j);
        return;
    }
    JointBodies jb = load_joint_bodies(S, sa, sb, flags);
    const JointNow s = joint_now(S, j, jb);
    const float4 lin = jrow(S, kJrLinear, j);
    const float4 angr = jrow(S, kJrAngular, j);
    const float4 fric = jrow(S, kJrFric, j);
    // phys_joint_angular_impulse (joint_solver.c:826-853): the fixed joint keeps a world
    // vector, the hinge and the ball scalars about axes rebuilt from the frames.
    V3 angular = v3(angr);
    if ((flags & kJHinge) != 0u) {
        const float4 mot = jrow(S, kJrMotor, j);
        angular = add(scale(axis_y(s.qa), angr.x), scale(axis_z(s.qa), angr.y));
        const float axial = lin.w - angr.w + mot.x + mot.y;
        angular = mul_add(angular, axis_x(s.qa), axial);
    } else if (joint_type(flags) == NPH_GPU_JOINT_BALL) {
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

// ---------------------------------------------------------------------------------------
// Fixed, slider, 6-DOF and distance joints (joint_solver.c:232-262, 395-720)
// ---------------------------------------------------------------------------------------

// joint_solver.c:232-262: the frames align, three angular rows; the error is the rotation
// vector from A's frame to B's, the shorter way round. `angr.xyz` is the world vector.
NPH_D void solve_rotation_lock(JointBodies &jb, const JointNow &s, float4 &angr, const StepConsts &K,
                               bool use_bias)
{
    const V3 cdot = relative_angular(jb);
    V3 bias = v3(0.0f, 0.0f, 0.0f);
    float mass_scale = 1.0f;
    float impulse_scale = 0.0f;
    if (use_bias) {
        Q4 e = q_mul(s.qb, q_conj(s.qa));
        if (e.w < 0.0f) {
            e = Q4{-e.x, -e.y, -e.z, -e.w};
        }
        bias = scale(v3(e.x, e.y, e.z), 2.0f * K.joint_soft.bias_rate);
        mass_scale = K.joint_soft.mass_scale;
        impulse_scale = K.joint_soft.impulse_scale;
    }
    const V3 x = solve3(add(jb.ia.c0, jb.ib.c0), add(jb.ia.c1, jb.ib.c1), add(jb.ia.c2, jb.ib.c2),
                        add(cdot, bias));
    const V3 impulse = sub(scale(x, -mass_scale), scale(v3(angr), impulse_scale));
    angr.x = angr.x + impulse.x;
    angr.y = angr.y + impulse.y;
    angr.z = angr.z + impulse.z;
    apply_angular(jb, impulse);
}

// joint_solver.c:480-509: one row, a translation along `u` of B's anchor against the point
// of A under it, or a rotation (u zero, both arms the axis), with its effective mass.
struct JRow {
    V3 u, ca, cb;
    float mass;
};

NPH_D JRow row_make(const JointBodies &jb, V3 u, V3 ca, V3 cb)
{
    const float k = (jb.ma + jb.mb) * dot(u, u) + dot(ca, m_mul_v(jb.ia, ca)) + dot(cb, m_mul_v(jb.ib, cb));
    return JRow{u, ca, cb, k > 0.0f ? 1.0f / k : 0.0f};
}

NPH_D JRow linear_row(const JointBodies &jb, const JointNow &s, V3 d, V3 u)
{
    return row_make(jb, u, cross(add(s.ra, d), u), cross(s.rb, u));
}

NPH_D JRow angular_row(const JointBodies &jb, V3 axis) { return row_make(jb, v3(0.0f, 0.0f, 0.0f), axis, axis); }

// joint_solver.c:511-515.
NPH_D float row_speed(const JointBodies &jb, const JRow &r)
{
    return dot(sub(jb.b.v, jb.a.v), r.u) + dot(jb.b.w, r.cb) - dot(jb.a.w, r.ca);
}

// joint_solver.c:517-530.
NPH_D void row_apply(JointBodies &jb, const JRow &r, float lambda)
{
    if (jb.wa) {
        jb.a.v = mul_add(jb.a.v, r.u, -jb.ma * lambda);
        jb.a.w = sub(jb.a.w, m_mul_v(jb.ia, scale(r.ca, lambda)));
    }
    if (jb.wb) {
        jb.b.v = mul_add(jb.b.v, r.u, jb.mb * lambda);
        jb.b.w = add(jb.b.w, m_mul_v(jb.ib, scale(r.cb, lambda)));
    }
}

// joint_solver.c:531-549: an equality row, soft while solving, rigid while relaxing.
NPH_D void row_lock(JointBodies &jb, const JRow &r, float c, float &accumulated, const StepConsts &K,
                    bool use_bias)
{
    float bias = 0.0f;
    float mass_scale = 1.0f;
    float impulse_scale = 0.0f;
    if (use_bias) {
        bias = K.joint_soft.bias_rate * c;
        mass_scale = K.joint_soft.mass_scale;
        impulse_scale = K.joint_soft.impulse_scale;
    }
    const float impulse = -r.mass * mass_scale * (row_speed(jb, r) + bias) - impulse_scale * accumulated;
    accumulated += impulse;
    row_apply(jb, r, impulse);
}

// joint_solver.c:550-562: a one-sided row (limit_soft, 178-190): open, it closes at most the
// gap this substep.
NPH_D void row_limit(JointBodies &jb, const JRow &r, float c, float sign, float &accumulated,
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
    const float impulse =
        -r.mass * mass_scale * (sign * row_speed(jb, r) + bias) - impulse_scale * accumulated;
    const float total = fmax_ref(accumulated + impulse, 0.0f);
    const float delta = total - accumulated;
    accumulated = total;
    row_apply(jb, r, sign * delta);
}

// joint_solver.c:564-571.
NPH_D void row_motor(JointBodies &jb, const JRow &r, float speed, float max_impulse, float &accumulated)
{
    const float old = accumulated;
    const float v = old - r.mass * (row_speed(jb, r) - speed);
    accumulated = v < -max_impulse ? -max_impulse : (v > max_impulse ? max_impulse : v);
    row_apply(jb, r, accumulated - old);
}

// joint_solver.c:573-585: a spring of its own frequency and damping, the solve pass only.
NPH_D void row_spring(JointBodies &jb, const JRow &r, float c, float4 soft, float &accumulated)
{
    const float impulse = -soft.z * r.mass * (row_speed(jb, r) + soft.y * c) - soft.w * accumulated;
    accumulated += impulse;
    row_apply(jb, r, impulse);
}

// vec.h:337-350.
NPH_D V3 normalize_or(V3 v, V3 fallback)
{
    const float len_sq = dot(v, v);
    if (len_sq > 0.0f && len_sq <= 3.40282347e38f) {
        return scale(v, 1.0f / sqrtf(len_sq));
    }
    if (!(len_sq > 3.40282347e38f) || !isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) {
        return fallback;
    }
    const float ax = fabsf(v.x), ay = fabsf(v.y), az = fabsf(v.z);
    const float m = ax > (ay > az ? ay : az) ? ax : (ay > az ? ay : az);
    const V3 u = scale(v, 1.0f / m);
    return scale(u, 1.0f / sqrtf(dot(u, u)));
}

// joint_solver.c:432-470: the axes now, B's anchor's offset from A's along A's frame axes,
// and the twist and swing angles of B's frame in A's (swing-twist, twist about X).
struct AxesNow {
    V3 d;
    V3 axis[NPH_GPU_D6_AXES];
    float value[NPH_GPU_D6_AXES];
};

NPH_D AxesNow axes_of(Q4 qa, Q4 qb, V3 d)
{
    AxesNow n;
    n.d = d;
    n.axis[0] = axis_x(qa);
    n.axis[1] = axis_y(qa);
    n.axis[2] = axis_z(qa);
#pragma unroll
    for (uint32_t i = 0; i < 3u; ++i) {
        n.value[i] = dot(d, n.axis[i]);
    }
    Q4 r = q_mul(q_conj(qa), qb);
    if (r.w < 0.0f) {
        r = Q4{-r.x, -r.y, -r.z, -r.w};
    }
    n.value[3] = 2.0f * nph_atan2f(r.x, r.w);
    const float tl = sqrtf(r.x * r.x + r.w * r.w);
    const Q4 twist = tl > 1e-9f ? Q4{r.x / tl, 0.0f, 0.0f, r.w / tl} : q_identity();
    const Q4 swing = q_mul(r, q_conj(twist));
    n.value[4] = 2.0f * nph_atan2f(swing.y, swing.w);
    n.value[5] = 2.0f * nph_atan2f(swing.z, swing.w);
    n.axis[3] = normalize_or(add(n.axis[0], axis_x(qb)), n.axis[0]);
    n.axis[4] = n.axis[1];
    n.axis[5] = n.axis[2];
    return n;
}

// joint_solver.c:471-476: B's anchor less A's, now.
NPH_D V3 anchor_offset(const JointBodies &jb, const JointNow &s, V3 delta_center)
{
    return add(add(sub(jb.pb.dp, jb.pa.dp), sub(s.rb, s.ra)), delta_center);
}

NPH_D JRow axis_row(const JointBodies &jb, const JointNow &s, const AxesNow &n, uint32_t i)
{
    return i < 3u ? linear_row(jb, s, n.d, n.axis[i]) : angular_row(jb, n.axis[i]);
}

NPH_D uint32_t axis_motion(uint32_t axes, uint32_t i) { return (axes >> (kJAxisBits * i)) & 3u; }
NPH_D bool axis_has(uint32_t axes, uint32_t i, uint32_t bit) { return ((axes >> (kJAxisBits * i)) & bit) != 0u; }

// joint_solver.c:597-652: every free or limited axis's spring, motor and limits, then the
// rotation locks (one block, the swing pair, or axis by axis), then the translation locks last.
template <bool kUseBias>
NPH_D void solve_axes(const DevSolver &S, uint32_t j, JointBodies &jb, const JointNow &s, uint32_t flags,
                      uint32_t axes, const StepConsts &K)
{
    float4 lin = jrow(S, kJrLinear, j);
    float4 angr = jrow(S, kJrAngular, j);
    float4 imp[NPH_GPU_D6_AXES];
#pragma unroll
    for (uint32_t i = 0; i < NPH_GPU_D6_AXES; ++i) {
        imp[i] = jrow(S, kJrAxisImpulse + i, j);
    }
    const AxesNow n = axes_of(s.qa, s.qb, anchor_offset(jb, s, v3(jrow(S, kJrDelta, j))));
#pragma unroll
    for (uint32_t i = 0; i < NPH_GPU_D6_AXES; ++i) {
        const uint32_t motion = axis_motion(axes, i);
        if (motion == NPH_GPU_AXIS_LOCKED) {
            continue;
        }
        const float4 set0 = jrow(S, kJrAxisSet + 2u * i, j);
        const JRow r = axis_row(jb, s, n, i);
        if (axis_has(axes, i, kJAxisSpring) && kUseBias) {
            const float4 set1 = jrow(S, kJrAxisSet + 2u * i + 1u, j);
            const float v = n.value[i] - set1.x;
            row_spring(jb, r, i >= 3u ? unwind(v) : v, set1, imp[i].w);
        }
        if (axis_has(axes, i, kJAxisMotor)) {
            row_motor(jb, r, set0.z, set0.w, imp[i].z);
        }
        if (motion == NPH_GPU_AXIS_LIMITED) {
            row_limit(jb, r, n.value[i] - set0.x, 1.0f, imp[i].x, K, kUseBias);
            row_limit(jb, r, set0.y - n.value[i], -1.0f, imp[i].y, K, kUseBias);
        }
    }
    if ((flags & kJBlockRotation) != 0u) {
        solve_rotation_lock(jb, s, angr, K, kUseBias);
    } else {
        const bool swings = (flags & kJBlockSwing) != 0u;
        if (swings) {
            solve_axis_lock(jb, s, angr, K, kUseBias);
        }
#pragma unroll
        for (uint32_t i = 3u; i < NPH_GPU_D6_AXES; ++i) {
            if (axis_motion(axes, i) == NPH_GPU_AXIS_LOCKED && (i == 3u || !swings)) {
                row_lock(jb, angular_row(jb, n.axis[i]), n.value[i], imp[i].x, K, kUseBias);
            }
        }
    }
    if ((flags & kJBlockPoint) != 0u) {
        V3 li = v3(lin);
        solve_point(jb, s, v3(jrow(S, kJrDelta, j)), li, K, kUseBias);
        lin.x = li.x;
        lin.y = li.y;
        lin.z = li.z;
    } else {
#pragma unroll
        for (uint32_t i = 0; i < 3u; ++i) {
            if (axis_motion(axes, i) == NPH_GPU_AXIS_LOCKED) {
                row_lock(jb, linear_row(jb, s, n.d, n.axis[i]), n.value[i], imp[i].x, K, kUseBias);
            }
        }
    }
    jset(S, kJrLinear, j, lin);
    jset(S, kJrAngular, j, angr);
#pragma unroll
    for (uint32_t i = 0; i < NPH_GPU_D6_AXES; ++i) {
        jset(S, kJrAxisImpulse + i, j, imp[i]);
    }
}

// joint_solver.c:683-707: one row along the line between the anchors.
template <bool kUseBias>
NPH_D void solve_distance(const DevSolver &S, uint32_t j, JointBodies &jb, const JointNow &s, uint32_t axes,
                          const StepConsts &K)
{
    const V3 d = anchor_offset(jb, s, v3(jrow(S, kJrDelta, j)));
    const float len = length(d);
    if (!(len > 1e-6f)) {
        return; // the anchors meet: the line has no direction
    }
    const JRow r = linear_row(jb, s, d, scale(d, 1.0f / len));
    float4 imp = jrow(S, kJrAxisImpulse, j);
    const float4 set0 = jrow(S, kJrAxisSet, j);
    const float4 set1 = jrow(S, kJrAxisSet + 1u, j);
    const uint32_t motion = axis_motion(axes, 0u);
    if (axis_has(axes, 0u, kJAxisSpring) && kUseBias) {
        row_spring(jb, r, len - set1.x, set1, imp.w);
    }
    if (axis_has(axes, 0u, kJAxisMotor)) {
        row_motor(jb, r, set0.z, set0.w, imp.z);
    }
    if (motion == NPH_GPU_AXIS_LIMITED) {
        row_limit(jb, r, len - set0.x, 1.0f, imp.x, K, kUseBias);
        row_limit(jb, r, set0.y - len, -1.0f, imp.y, K, kUseBias);
    } else if (motion == NPH_GPU_AXIS_LOCKED) {
        row_lock(jb, r, len - set1.x, imp.x, K, kUseBias);
    }
    jset(S, kJrAxisImpulse, j, imp);
}

// Slider, 6-DOF and distance joints: the solve (joint_solver.c:870-897), kept out of line so
// the ball and hinge path keeps its registers.
template <bool kUseBias>
__device__ __noinline__ void solve_row_joint(const DevSolver &S, uint32_t j, const StepConsts &K)
{
    const float4 head = jrow(S, kJrHead, j);
    const uint32_t flags = __float_as_uint(head.z);
    JointBodies jb = load_joint_bodies(S, __float_as_uint(head.x), __float_as_uint(head.y), flags);
    const JointNow s = joint_now(S, j, jb);
    if (joint_type(flags) == NPH_GPU_JOINT_DISTANCE) {
        solve_distance<kUseBias>(S, j, jb, s, __float_as_uint(head.w), K);
    } else {
        solve_axes<kUseBias>(S, j, jb, s, flags, __float_as_uint(head.w), K);
    }
    store_joint_bodies(S, jb);
}

// joint_solver.c:654-682 and 709-720: the rows' impulses applied again about the current
// axes (the blocks' as the blocks keep them), or along the current line.
static __device__ __noinline__ void warm_row_joint(const DevSolver &S, uint32_t j)
{
    const float4 head = jrow(S, kJrHead, j);
    const uint32_t flags = __float_as_uint(head.z);
    JointBodies jb = load_joint_bodies(S, __float_as_uint(head.x), __float_as_uint(head.y), flags);
    const JointNow s = joint_now(S, j, jb);
    const V3 d = anchor_offset(jb, s, v3(jrow(S, kJrDelta, j)));
    if (joint_type(flags) == NPH_GPU_JOINT_DISTANCE) {
        const float len = length(d);
        const float4 imp = jrow(S, kJrAxisImpulse, j);
        const float total = imp.x - imp.y + imp.z + imp.w;
        if (len > 1e-6f && total != 0.0f) {
            row_apply(jb, linear_row(jb, s, d, scale(d, 1.0f / len)), total);
        }
    } else {
        const AxesNow n = axes_of(s.qa, s.qb, d);
#pragma unroll
        for (uint32_t i = 0; i < NPH_GPU_D6_AXES; ++i) {
            const float4 imp = jrow(S, kJrAxisImpulse + i, j);
            const float total = imp.x - imp.y + imp.z + imp.w;
            if (total != 0.0f) {
                row_apply(jb, axis_row(jb, s, n, i), total);
            }
        }
        const float4 angr = jrow(S, kJrAngular, j);
        if ((flags & kJBlockRotation) != 0u) {
            apply_angular(jb, v3(angr));
        } else if ((flags & kJBlockSwing) != 0u) {
            apply_angular(jb, add(scale(axis_y(s.qa), angr.x), scale(axis_z(s.qa), angr.y)));
        }
        if ((flags & kJBlockPoint) != 0u) {
            apply_linear(jb, s, v3(jrow(S, kJrLinear, j)));
        }
    }
    store_joint_bodies(S, jb);
}

// joint_solver.c:870-897, ball (360-394) and hinge (303-336).
template <bool kUseBias, int kSet = kJointsAll>
NPH_D void solve_joint(const DevSolver &S, uint32_t j, const StepConsts &K)
{
    uint32_t sa, sb, flags;
    joint_head(S, j, sa, sb, flags);
    const bool rows = joint_has_rows(joint_type(flags));
    if ((kSet == kJointsPlain && rows) || (kSet == kJointsRows && !rows)) {
        return;
    }
    if (kSet != kJointsPlain && rows) {
        solve_row_joint<kUseBias>(S, j, K);
        return;
    }
    JointBodies jb = load_joint_bodies(S, sa, sb, flags);
    const JointNow s = joint_now(S, j, jb);
    float4 lin = jrow(S, kJrLinear, j);
    float4 angr = jrow(S, kJrAngular, j);
    float4 fric = jrow(S, kJrFric, j);
    float4 mot = jrow(S, kJrMotor, j);
    const float4 set_a = jrow(S, kJrSetA, j);
    if (joint_type(flags) == NPH_GPU_JOINT_FIXED) {
        solve_rotation_lock(jb, s, angr, K, kUseBias);
    } else if ((flags & kJHinge) != 0u) {
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
                const float phi = nph_atan2f(sin_phi, dot(xa, xb));
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

// The accumulated impulses back into the joint's record (and a slider's or 6-DOF joint's
// blocks into its flags).
NPH_D void store_joint(const DevSolver &S, uint32_t j, NphGpuJoint &jr)
{
    const float4 head = jrow(S, kJrHead, j);
    const uint32_t flags = __float_as_uint(head.z);
    const uint32_t type = joint_type(flags);
    if (joint_has_rows(type)) {
        const uint32_t rows = type == NPH_GPU_JOINT_DISTANCE ? 1u : NPH_GPU_D6_AXES;
        for (uint32_t i = 0; i < rows; ++i) {
            const float4 imp = jrow(S, kJrAxisImpulse + i, j);
            jr.axis_impulse[i][0] = imp.x;
            jr.axis_impulse[i][1] = imp.y;
            jr.axis_impulse[i][2] = imp.z;
            jr.axis_impulse[i][3] = imp.w;
        }
        if (type != NPH_GPU_JOINT_DISTANCE) {
            jr.flags = (jr.flags & ~kJBlocks) | (flags & kJBlocks);
        }
    }
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

// SPDX-License-Identifier: Apache-2.0
//
// The solver stage's device-resident data: structure-of-arrays rows of float4, so a warp's
// 32 lanes read 512 contiguous bytes per row, and a body's state is two 16-byte rows (one
// 32-byte sector) per kind.
//
//   bodies (solver slots 0..n-1, then the dummy at n: at rest, never written; solver.c:967-973)
//     vel[2i]   v (w unused)          vel[2i+1] w             (PhysSolverBody rows 0-1)
//     pos[2i]   dp                    pos[2i+1] dq            (PhysSolverBody rows 2-3)
//     prm[3i+c] column c of the world inverse inertia; .w of column 0 the inverse mass;
//               all zero unless dynamic (PhysSolverParams, prepare_group's dyn ? .. : 0)
//     itg[6i..] what integration reads (PhysSolverParams, world_internal.h:403-417)
//   manifolds (colour order; capacity `mcap`), one lane each:
//     hdr       solver indices of A and B, the manifold's bits (kHdr*), its ranks (kRank*)
//     nrm       normal.xyz, friction              rest  restitution
//     per point k, row k*mcap + g:
//       pa      anchor_a.xyz, adjusted separation
//       pb      anchor_b.xyz, normal mass
//       pt      the tangent effective-mass inverse (00, 01, 11), normal approach speed
//       pi      normal impulse, max normal impulse, tangent impulses 1 and 2 (read-write)
//   joints (colour order; capacity `jcap`): kJointRows float4 rows, row r at r*jcap + j.
//
// The tangents t1 = perpendicular(n), t2 = n x t1 and the angular terms I^-1 (r x axis) are
// recomputed where they are used instead of stored: the same operations on the same values
// round to the same bits as the reference's stored ones (solver_impl.h:276-385), and it
// saves 24 + 72 x 4 bytes per manifold and pass.
#pragma once

#include <cstdint>

#include "devmath.cuh"

namespace nph {

// A constraint's rank on a body it writes, in hdr.w for a manifold (A in bits 0-7, B in bits
// 8-15): how many constraints of earlier colours write that body (at most the colours); bits
// 16 and 17: a constraint of a later colour writes A, B (only then is its finishing counted).
constexpr uint32_t kRankBits = 8u;
constexpr uint32_t kRankMask = 0xFFu;
constexpr uint32_t kRankLaterA = 1u << 16;
constexpr uint32_t kRankLaterB = 1u << 17;

// Manifold header bits (hdr.z).
constexpr uint32_t kHdrPointsMask = 7u;        // the manifold's own point count, 0..4
constexpr uint32_t kHdrGroupShift = 3u;        // its eight-lane group's largest point count
constexpr uint32_t kHdrWriteA = 1u << 6;       // A is dynamic: takes the results
constexpr uint32_t kHdrWriteB = 1u << 7;
constexpr uint32_t kHdrStaticSoft = 1u << 8;   // a static or kinematic side: stiffer springs
constexpr uint32_t kHdrImpact = 1u << 9;       // a point approaches faster than 1 m/s
constexpr uint32_t kHdrImpacted = 1u << 10;    // HIT at the step's start (warm_start scaling)

// Joint flag bits (row 0 .z).
constexpr uint32_t kJHinge = 1u << 0;
constexpr uint32_t kJWriteA = 1u << 1;
constexpr uint32_t kJWriteB = 1u << 2;
constexpr uint32_t kJLimit = 1u << 3;      // hinge limit
constexpr uint32_t kJMotor = 1u << 4;      // hinge motor
constexpr uint32_t kJSpring = 1u << 5;     // hinge spring
constexpr uint32_t kJSwing = 1u << 6;      // ball cone
constexpr uint32_t kJTwist = 1u << 7;      // ball twist limits
constexpr uint32_t kJFriction = 1u << 8;   // ball friction (torque > 0)
constexpr uint32_t kJDriven = 1u << 9;     // a motor driving to a non-zero speed (any type)
// The blocks of a slider or 6-DOF joint: the bits of NPH_GPU_JOINT_BLOCK_*.
constexpr uint32_t kJBlockRotation = 1u << 11;
constexpr uint32_t kJBlockSwing = 1u << 12;
constexpr uint32_t kJBlockPoint = 1u << 13;
constexpr uint32_t kJBlocks = kJBlockRotation | kJBlockSwing | kJBlockPoint;
constexpr uint32_t kJTypeShift = 16u;      // NPH_GPU_JOINT_* in bits 16..18
constexpr uint32_t kJTypeMask = 7u;
// Per axis of a slider, 6-DOF or distance joint, four bits of row 0 .w: the motion (2 bits,
// NPH_GPU_AXIS_*), the motor, the spring. A distance joint's axis 0 is its line: limited when
// its limits are on, else locked unless its spring is on.
constexpr uint32_t kJAxisBits = 4u;
constexpr uint32_t kJAxisMotor = 1u << 2;
constexpr uint32_t kJAxisSpring = 1u << 3;

// Joint rows.
enum : uint32_t {
    kJrHead = 0,     // sa, sb, flags (as uint bits)
    kJrAnchorA = 1,  // anchor_a.xyz
    kJrAnchorB = 2,  // anchor_b.xyz
    kJrDelta = 3,    // delta_center.xyz
    kJrFrameA = 4,   // frame_q_a
    kJrFrameB = 5,   // frame_q_b
    kJrSpring = 6,   // spring softness: bias_rate, mass_scale, impulse_scale
    kJrSetA = 7,     // hinge: lower, upper, motor_speed, max_motor_torque
                     // ball: swing_y, swing_z, twist_lower, twist_upper
    kJrSetB = 8,     // hinge: spring_target; ball: friction_torque
    kJrLinear = 9,   // linear_impulse.xyz, lower_impulse
    kJrAngular = 10, // angular_impulse.xyz, upper_impulse
    kJrFric = 11,    // friction_impulse.xyz, swing_impulse
    kJrMotor = 12,   // motor_impulse, spring_impulse
    // Slider, 6-DOF and distance joints only, per axis i (distance: axis 0):
    kJrAxisSet = 13,     // row 13 + 2i: lower, upper, motor_speed, h x max motor force
                         // row 14 + 2i: spring target, the spring's softness
                         // (distance: min and max length; length)
    kJrAxisImpulse = 25, // row 25 + i: the lock or lower, upper, motor and spring impulses
    kJointRows = 31,
};

// Device error bits.
constexpr uint32_t kErrBadIndex = 1u << 0;
constexpr uint32_t kErrBadPoints = 1u << 1;
constexpr uint32_t kErrBadJoint = 1u << 2;
constexpr uint32_t kErrBadBody = 1u << 3; // a value the stage reads is not finite
constexpr uint32_t kErrWait = 1u << 4;    // a dependency-driven pass gave up a wait

// The step's constants (StepContext, solver.c:67-85), computed on the host in FP32 with the
// reference's operations.
struct StepConsts {
    float dt, h, inv_h, push_max, restitution_threshold;
    Soft contact_soft, static_soft, joint_soft;
    float max_angular_speed_sq, max_linear_speed_sq;
    float gravity[3];
    float slop;          // TGS: the overlap its Baumgarte bias leaves alone (0: the soft step)
    uint32_t scale_hits; // TGS: a hit scales the next warm start (solver.c:411-416)
    uint32_t solver;     // NPH_GPU_SOLVER_*: the stage list (solver.c:1036-1060)
};

// The body side of a constraint: what the passes read and write of one body.
struct BodyState {
    V3 v, w;
};

struct BodyPose {
    V3 dp;
    Q4 dq;
};

// Pointers to one world's device arrays (a batched world's are offset views).
struct DevSolver {
    float4 *vel;
    float4 *pos;
    float4 *prm;
    uint4 *hdr;
    float4 *nrm;
    float *rest;
    float4 *pa, *pb, *pt, *pi; // point rows, stride mcap
    uint32_t mcap;
    float4 *jw;                // joint rows, stride jcap
    uint32_t jcap;
    // The dependency-driven passes (solver.cu k_pass_flow): per body slot, the colours whose
    // constraints write it (bit c) and how many of them have finished the current pass; per
    // joint, its rank on each body it writes (the manifolds' ranks are in hdr.w).
    const uint32_t *cmask;
    uint32_t *done;
    uint32_t *jrank;
};

NPH_D M3 load_inv_inertia(const float4 *prm, uint32_t i, float *inv_mass)
{
    const float4 c0 = prm[3u * i + 0u];
    const float4 c1 = prm[3u * i + 1u];
    const float4 c2 = prm[3u * i + 2u];
    *inv_mass = c0.w;
    return M3{v3(c0), v3(c1), v3(c2)};
}

NPH_D BodyState load_state(const float4 *vel, uint32_t i)
{
    const float4 v = vel[2u * i];
    const float4 w = vel[2u * i + 1u];
    return BodyState{v3(v), v3(w)};
}

NPH_D void store_state(float4 *vel, uint32_t i, const BodyState &s)
{
    vel[2u * i] = f4(s.v, 0.0f);
    vel[2u * i + 1u] = f4(s.w, 0.0f);
}

NPH_D BodyPose load_pose(const float4 *pos, uint32_t i)
{
    const float4 p = pos[2u * i];
    const float4 q = pos[2u * i + 1u];
    return BodyPose{v3(p), q4(q)};
}

} // namespace nph

/* SPDX-License-Identifier: Apache-2.0
 *
 * A joint record's configuration as the reference's joint solver reads it: the six axes of a
 * slider or 6-DOF joint (d6_config, joint_solver.c:399-421: a slider is a 6-DOF joint whose
 * translation along A's X is free or limited, with its drives, and whose other axes are
 * locked), the blocks its locked axes are solved as (joint_solver.c:809-822), whether a motor
 * drives it (phys_joint_is_driven, joint_solver.c:1410-1434), and the checks of a record. Plain
 * C: the device solver, the host's validation and the CPU restatement include it alike.
 */
#ifndef NPH_JOINT_CONFIG_H
#define NPH_JOINT_CONFIG_H

#include "nepheline_b200.h"

#if defined(__CUDACC__)
#define NPH_JC __host__ __device__ static inline
#else
#define NPH_JC static inline
#endif

NPH_JC int nph_joint_has_axes(uint32_t type)
{
    return type == NPH_GPU_JOINT_SLIDER || type == NPH_GPU_JOINT_D6;
}

/* d6_config: the 6-DOF joint's own axes, or the slider's (translation X from its settings,
 * every other axis locked). */
NPH_JC void nph_joint_axes(const NphGpuJoint *j, NphGpuD6Axis out[NPH_GPU_D6_AXES])
{
    if (j->type == NPH_GPU_JOINT_D6) {
        for (uint32_t i = 0U; i < NPH_GPU_D6_AXES; ++i) {
            out[i] = j->u.d6[i];
        }
        return;
    }
    for (uint32_t i = 0U; i < NPH_GPU_D6_AXES; ++i) {
        NphGpuD6Axis z;
        z.motion = NPH_GPU_AXIS_LOCKED;
        z.lower = 0.0F;
        z.upper = 0.0F;
        z.enable_motor = 0U;
        z.motor_speed = 0.0F;
        z.max_motor_force = 0.0F;
        z.enable_spring = 0U;
        z.spring_hertz = 0.0F;
        z.spring_damping_ratio = 0.0F;
        z.spring_target = 0.0F;
        out[i] = z;
    }
    const NphGpuSliderJoint *s = &j->u.slider;
    NphGpuD6Axis *x = &out[0];
    x->motion = s->enable_limit != 0U ? NPH_GPU_AXIS_LIMITED : NPH_GPU_AXIS_FREE;
    x->lower = s->lower;
    x->upper = s->upper;
    x->enable_motor = s->enable_motor;
    x->motor_speed = s->motor_speed;
    x->max_motor_force = s->max_motor_force;
    x->enable_spring = s->enable_spring;
    x->spring_hertz = s->spring_hertz;
    x->spring_damping_ratio = s->spring_damping_ratio;
    x->spring_target = s->spring_target;
}

/* all_locked (joint_solver.c:423-431). */
NPH_JC int nph_joint_all_locked(const NphGpuD6Axis *ax, uint32_t first, uint32_t count)
{
    for (uint32_t i = first; i < first + count; ++i) {
        if (ax[i].motion != NPH_GPU_AXIS_LOCKED) {
            return 0;
        }
    }
    return 1;
}

/* The blocks of a slider or 6-DOF joint: the rotation as one block when all three angular
 * axes are locked, else the swing pair when both swings are; the anchors when all three
 * translations are. */
NPH_JC uint32_t nph_joint_blocks(const NphGpuD6Axis ax[NPH_GPU_D6_AXES])
{
    const int rotation = nph_joint_all_locked(ax, 3U, 3U);
    const int swing = !rotation && nph_joint_all_locked(ax, 4U, 2U);
    const int point = nph_joint_all_locked(ax, 0U, 3U);
    return (rotation ? NPH_GPU_JOINT_BLOCK_ROTATION : 0U) | (swing ? NPH_GPU_JOINT_BLOCK_SWING : 0U) |
           (point ? NPH_GPU_JOINT_BLOCK_POINT : 0U);
}

/* phys_joint_is_driven: a motor set to a non-zero speed with a positive limit keeps the joint's
 * bodies awake. */
NPH_JC int nph_joint_is_driven(const NphGpuJoint *j)
{
    if (j->type == NPH_GPU_JOINT_HINGE) {
        const NphGpuHingeJoint *h = &j->u.hinge;
        return h->enable_motor != 0U && h->motor_speed != 0.0F && h->max_motor_torque > 0.0F;
    }
    if (j->type == NPH_GPU_JOINT_DISTANCE) {
        const NphGpuDistanceJoint *d = &j->u.distance;
        return d->enable_motor != 0U && d->motor_speed != 0.0F && d->max_motor_force > 0.0F;
    }
    if (nph_joint_has_axes(j->type)) {
        NphGpuD6Axis ax[NPH_GPU_D6_AXES];
        nph_joint_axes(j, ax);
        for (uint32_t i = 0U; i < NPH_GPU_D6_AXES; ++i) {
            if (ax[i].motion != NPH_GPU_AXIS_LOCKED && ax[i].enable_motor != 0U &&
                ax[i].motor_speed != 0.0F && ax[i].max_motor_force > 0.0F) {
                return 1;
            }
        }
    }
    return 0;
}

/* NPH_GPU_OK for a record the solver runs; NPH_GPU_UNSUPPORTED for an unknown type,
 * NPH_GPU_INVALID_ARGUMENT for a 6-DOF axis whose motion is none of NPH_GPU_AXIS_*. */
NPH_JC int nph_joint_check(const NphGpuJoint *j)
{
    if (j->type > NPH_GPU_JOINT_D6) {
        return NPH_GPU_UNSUPPORTED;
    }
    if (j->type == NPH_GPU_JOINT_D6) {
        for (uint32_t i = 0U; i < NPH_GPU_D6_AXES; ++i) {
            if (j->u.d6[i].motion > NPH_GPU_AXIS_FREE) {
                return NPH_GPU_INVALID_ARGUMENT;
            }
        }
    }
    return NPH_GPU_OK;
}

#endif /* NPH_JOINT_CONFIG_H */

// SPDX-License-Identifier: Apache-2.0
//
// The reference engine's side of the drop-in: converting an NphPhysicsWorld (the engine's
// world_internal.h records) to the solver-stage view of include/nepheline_b200.h and back.
// Compiled inside the reference's physics library, beside its own sources (it reads the
// world's internal records), by the binding (phys_solve_dispatch.c) and by the oracle's
// harness, which both need the same conversion.
//
//   export  the stage's inputs as records, in the reference's solver order: the awake list
//           (solver.c:967-973), then the bodies a constraint names without a solver slot;
//           contacts and joints colour by colour, 0..23 then the overflow (build_groups,
//           solver.c:810-843; build_step_joints, solver.c:793-806);
//   import  what phys_solve's stages write back (finalize_body, solver.c:304-349;
//           store_group, solver.c:475-499; the joints' impulses and block bits), with the
//           finalize pass's box refresh (phys_body_refresh_boxes, solver.c:351-369).
#pragma once

#include "world_internal.h"

#include "nepheline_b200.h"

#include <stdlib.h>
#include <string.h>

#define NPH_VIEW_JOINT_BLOCKS \
    (NPH_GPU_JOINT_BLOCK_ROTATION | NPH_GPU_JOINT_BLOCK_SWING | NPH_GPU_JOINT_BLOCK_POINT)
_Static_assert(NPH_GPU_CONTACT_HIT == PHYS_CONTACT_HIT && NPH_GPU_CONTACT_HIT_EVENTS == PHYS_CONTACT_HIT_EVENTS,
               "the contact record's flag bits are the world's");
_Static_assert(sizeof(((PhysJoint *)0)->axis_impulse) == sizeof(((NphGpuJoint *)0)->axis_impulse),
               "the rows per axis of PhysJoint and of the record");

// Which body slots a view holds as fixed bodies (after the awake ones), and in what order.
typedef struct NphViewMap {
    u32 *fixed_of_slot; // per body slot: its fixed-body index in the view, or PHYS_NULL
    u32 *fixed_slots;   // per fixed-body index: its body slot
    u32 cap;
} NphViewMap;

static inline void nph_view_map_release(NphViewMap *m)
{
    free(m->fixed_of_slot);
    free(m->fixed_slots);
    memset(m, 0, sizeof *m);
}

static inline const NphArrayU32 *nph_view_contact_list(const NphPhysicsWorld *w, u32 c)
{
    return c == PHYS_GRAPH_OVERFLOW ? &w->overflow : &w->colors[c].contacts;
}

static inline const NphArrayU32 *nph_view_joint_list(const NphPhysicsWorld *w, u32 c)
{
    return c == PHYS_GRAPH_OVERFLOW ? &w->overflow_joints : &w->colors[c].joints;
}

static inline void nph_view_body_record(const PhysBody *b, NphGpuBody *o)
{
    memset(o, 0, sizeof *o);
    o->center[0] = b->center.x;
    o->center[1] = b->center.y;
    o->center[2] = b->center.z;
    o->origin[0] = b->origin.x;
    o->origin[1] = b->origin.y;
    o->origin[2] = b->origin.z;
    memcpy(o->rotation, &b->rotation, sizeof o->rotation);
    memcpy(o->local_center, &b->local_center, sizeof o->local_center);
    memcpy(o->linear_velocity, &b->linear_velocity, sizeof o->linear_velocity);
    memcpy(o->angular_velocity, &b->angular_velocity, sizeof o->angular_velocity);
    memcpy(o->force, &b->force, sizeof o->force);
    memcpy(o->torque, &b->torque, sizeof o->torque);
    memcpy(o->inertia, &b->inertia, sizeof o->inertia);
    memcpy(o->inv_inertia, &b->inv_inertia, sizeof o->inv_inertia);
    o->inv_mass = b->inv_mass;
    o->linear_damping = b->linear_damping;
    o->angular_damping = b->angular_damping;
    o->gravity_scale = b->gravity_scale;
    o->sleep_threshold = b->sleep_threshold;
    o->sleep_time = b->sleep_time;
    o->max_extent = b->max_extent;
    o->type = b->type;
    o->flags = b->flags;
    o->locks = b->locks;
}

// The view index of body slot `slot`: its awake slot, or a fixed body's index after them.
static inline u32 nph_view_index(const NphPhysicsWorld *w, NphViewMap *m, u32 slot, u32 *fixed_count)
{
    const PhysBody *b = &w->bodies.data[slot];
    if (b->awake_slot != PHYS_NULL) {
        return b->awake_slot;
    }
    if (m->fixed_of_slot[slot] == PHYS_NULL) {
        m->fixed_slots[*fixed_count] = slot;
        m->fixed_of_slot[slot] = (*fixed_count)++;
    }
    return w->awake_bodies.len + m->fixed_of_slot[slot];
}

// Maps the constraints' bodies without solver slots to fixed-body indices, in the order the
// colour lists name them. Returns NPH_RESULT_OUT_OF_MEMORY when the map cannot grow.
static inline NphResult nph_view_map_fixed(const NphPhysicsWorld *w, NphViewMap *m, u32 *fixed_count)
{
    if (w->bodies.len + 1U > m->cap) {
        const u32 cap = w->bodies.len + 1U + (w->bodies.len + 1U) / 2U;
        u32 *a = (u32 *)realloc(m->fixed_of_slot, (size_t)cap * sizeof(u32));
        if (a == NULL) {
            return NPH_RESULT_OUT_OF_MEMORY;
        }
        m->fixed_of_slot = a;
        u32 *b = (u32 *)realloc(m->fixed_slots, (size_t)cap * sizeof(u32));
        if (b == NULL) {
            return NPH_RESULT_OUT_OF_MEMORY;
        }
        m->fixed_slots = b;
        m->cap = cap;
    }
    for (u32 i = 0U; i < w->bodies.len; ++i) {
        m->fixed_of_slot[i] = PHYS_NULL;
    }
    *fixed_count = 0U;
    for (u32 c = 0U; c <= PHYS_GRAPH_COLORS; ++c) {
        const NphArrayU32 *list = nph_view_contact_list(w, c);
        for (u32 i = 0U; i < list->len; ++i) {
            const PhysContact *ct = &w->contacts.data[list->data[i]];
            (void)nph_view_index(w, m, ct->body_a, fixed_count);
            (void)nph_view_index(w, m, ct->body_b, fixed_count);
        }
        const NphArrayU32 *jl = nph_view_joint_list(w, c);
        for (u32 i = 0U; i < jl->len; ++i) {
            const PhysJoint *j = &w->joints.data[jl->data[i]];
            (void)nph_view_index(w, m, j->body_a, fixed_count);
            (void)nph_view_index(w, m, j->body_b, fixed_count);
        }
    }
    return NPH_RESULT_OK;
}

// The record counts a view of the world needs (and the fixed-body map it will use).
static inline NphResult nph_view_sizes(const NphPhysicsWorld *w, NphViewMap *m, u32 *bodies, u32 *fixed,
                                       u32 *contacts, u32 *joints)
{
    NPH_TRY(nph_view_map_fixed(w, m, fixed));
    *bodies = w->awake_bodies.len;
    u32 nc = 0U;
    u32 nj = 0U;
    for (u32 c = 0U; c <= PHYS_GRAPH_COLORS; ++c) {
        nc += nph_view_contact_list(w, c)->len;
        nj += nph_view_joint_list(w, c)->len;
    }
    *contacts = nc;
    *joints = nj;
    return NPH_RESULT_OK;
}

static inline void nph_view_contact_record(const NphPhysicsWorld *w, NphViewMap *m, const PhysContact *c,
                                           NphGpuContact *o, u32 *fixed_count)
{
    memset(o, 0, sizeof *o);
    o->body_a = nph_view_index(w, m, c->body_a, fixed_count);
    o->body_b = nph_view_index(w, m, c->body_b, fixed_count);
    o->flags = c->flags & (PHYS_CONTACT_HIT | PHYS_CONTACT_HIT_EVENTS);
    o->point_count = c->point_count;
    memcpy(o->normal, &c->normal, sizeof o->normal);
    o->friction = c->friction;
    o->restitution = c->restitution;
    for (u32 k = 0U; k < c->point_count; ++k) {
        const PhysContactPoint *p = &c->points[k];
        NphGpuContactPoint *q = &o->points[k];
        memcpy(q->anchor_a, &p->anchor_a, sizeof q->anchor_a);
        memcpy(q->anchor_b, &p->anchor_b, sizeof q->anchor_b);
        q->separation = p->separation;
        q->normal_impulse = p->normal_impulse;
        q->max_normal_impulse = p->max_normal_impulse;
        memcpy(q->tangent_impulse, &p->tangent_impulse, sizeof q->tangent_impulse);
        q->relative_velocity = p->relative_velocity;
        q->id = p->id;
    }
}

static inline void nph_view_joint_record(const NphPhysicsWorld *w, NphViewMap *m, const PhysJoint *j,
                                         NphGpuJoint *o, u32 *fixed_count)
{
    memset(o, 0, sizeof *o);
    o->type = j->type;
    o->body_a = nph_view_index(w, m, j->body_a, fixed_count);
    o->body_b = nph_view_index(w, m, j->body_b, fixed_count);
    memcpy(o->frame_a_position, &j->frame_a.position, sizeof o->frame_a_position);
    memcpy(o->frame_a_rotation, &j->frame_a.rotation, sizeof o->frame_a_rotation);
    memcpy(o->frame_b_position, &j->frame_b.position, sizeof o->frame_b_position);
    memcpy(o->frame_b_rotation, &j->frame_b.rotation, sizeof o->frame_b_rotation);
    if (j->type == NPH_PHYSICS_JOINT_BALL) {
        o->u.ball.enable_swing_limit = (u32)j->ball.enable_swing_limit;
        o->u.ball.swing_y = j->ball.swing_y;
        o->u.ball.swing_z = j->ball.swing_z;
        o->u.ball.enable_twist_limit = (u32)j->ball.enable_twist_limit;
        o->u.ball.twist_lower = j->ball.twist_lower;
        o->u.ball.twist_upper = j->ball.twist_upper;
        o->u.ball.friction_torque = j->ball.friction_torque;
    } else if (j->type == NPH_PHYSICS_JOINT_HINGE) {
        o->u.hinge.enable_limit = (u32)j->hinge.enable_limit;
        o->u.hinge.lower = j->hinge.lower;
        o->u.hinge.upper = j->hinge.upper;
        o->u.hinge.enable_motor = (u32)j->hinge.enable_motor;
        o->u.hinge.motor_speed = j->hinge.motor_speed;
        o->u.hinge.max_motor_torque = j->hinge.max_motor_torque;
        o->u.hinge.enable_spring = (u32)j->hinge.enable_spring;
        o->u.hinge.spring_hertz = j->hinge.spring_hertz;
        o->u.hinge.spring_damping_ratio = j->hinge.spring_damping_ratio;
        o->u.hinge.spring_target = j->hinge.spring_target;
    } else if (j->type == NPH_PHYSICS_JOINT_SLIDER) {
        o->u.slider.enable_limit = (u32)j->slider.enable_limit;
        o->u.slider.lower = j->slider.lower;
        o->u.slider.upper = j->slider.upper;
        o->u.slider.enable_motor = (u32)j->slider.enable_motor;
        o->u.slider.motor_speed = j->slider.motor_speed;
        o->u.slider.max_motor_force = j->slider.max_motor_force;
        o->u.slider.enable_spring = (u32)j->slider.enable_spring;
        o->u.slider.spring_hertz = j->slider.spring_hertz;
        o->u.slider.spring_damping_ratio = j->slider.spring_damping_ratio;
        o->u.slider.spring_target = j->slider.spring_target;
    } else if (j->type == NPH_PHYSICS_JOINT_DISTANCE) {
        o->u.distance.length = j->distance.length;
        o->u.distance.enable_limit = (u32)j->distance.enable_limit;
        o->u.distance.min_length = j->distance.min_length;
        o->u.distance.max_length = j->distance.max_length;
        o->u.distance.enable_spring = (u32)j->distance.enable_spring;
        o->u.distance.spring_hertz = j->distance.spring_hertz;
        o->u.distance.spring_damping_ratio = j->distance.spring_damping_ratio;
        o->u.distance.enable_motor = (u32)j->distance.enable_motor;
        o->u.distance.motor_speed = j->distance.motor_speed;
        o->u.distance.max_motor_force = j->distance.max_motor_force;
    } else if (j->type == NPH_PHYSICS_JOINT_D6) {
        for (u32 i = 0U; i < NPH_PHYSICS_D6_AXES; ++i) {
            const NphPhysicsD6Axis *x = &j->d6.axes[i];
            NphGpuD6Axis *y = &o->u.d6[i];
            y->motion = (u32)x->motion;
            y->lower = x->lower;
            y->upper = x->upper;
            y->enable_motor = (u32)x->enable_motor;
            y->motor_speed = x->motor_speed;
            y->max_motor_force = x->max_motor_force;
            y->enable_spring = (u32)x->enable_spring;
            y->spring_hertz = x->spring_hertz;
            y->spring_damping_ratio = x->spring_damping_ratio;
            y->spring_target = x->spring_target;
        }
    }
    // The block bits of joint_solver.c:103-112 carry across steps; the others are the step's.
    o->flags = j->flags & NPH_VIEW_JOINT_BLOCKS;
    memcpy(o->axis_impulse, j->axis_impulse, sizeof o->axis_impulse);
    memcpy(o->linear_impulse, &j->linear_impulse, sizeof o->linear_impulse);
    memcpy(o->angular_impulse, &j->angular_impulse, sizeof o->angular_impulse);
    memcpy(o->friction_impulse, &j->friction_impulse, sizeof o->friction_impulse);
    o->lower_impulse = j->lower_impulse;
    o->upper_impulse = j->upper_impulse;
    o->swing_impulse = j->swing_impulse;
    o->motor_impulse = j->motor_impulse;
    o->spring_impulse = j->spring_impulse;
}

// Fills a view whose arrays hold the counts nph_view_sizes gave (with the same map). Returns 0,
// or 1 when the world changed since the sizes were taken.
static inline int nph_view_export(const NphPhysicsWorld *w, NphViewMap *m, NphGpuWorldView *v)
{
    u32 fixed = 0U;
    if (nph_view_map_fixed(w, m, &fixed) != NPH_RESULT_OK) {
        return 1;
    }
    v->body_count = w->awake_bodies.len;
    for (u32 i = 0U; i < w->awake_bodies.len; ++i) {
        nph_view_body_record(&w->bodies.data[w->awake_bodies.data[i]], &v->bodies[i]);
    }
    v->fixed_count = fixed;
    for (u32 i = 0U; i < fixed; ++i) {
        nph_view_body_record(&w->bodies.data[m->fixed_slots[i]], (NphGpuBody *)&v->fixed_bodies[i]);
    }
    u32 nc = 0U;
    u32 nj = 0U;
    u32 again = fixed;
    for (u32 c = 0U; c <= PHYS_GRAPH_COLORS; ++c) {
        const NphArrayU32 *list = nph_view_contact_list(w, c);
        v->contact_color_counts[c] = list->len;
        for (u32 i = 0U; i < list->len; ++i) {
            nph_view_contact_record(w, m, &w->contacts.data[list->data[i]], &v->contacts[nc++], &again);
        }
        const NphArrayU32 *jl = nph_view_joint_list(w, c);
        v->joint_color_counts[c] = jl->len;
        for (u32 i = 0U; i < jl->len; ++i) {
            nph_view_joint_record(w, m, &w->joints.data[jl->data[i]], &v->joints[nj++], &again);
        }
    }
    v->contact_count = nc;
    v->joint_count = nj;
    return again == fixed ? 0 : 1;
}

// Writes a solved view back into the world: what phys_solve's stages write (finalize_body,
// store_group, the joints' impulses and block bits) and the finalize pass's box refresh. The
// view must have been exported from this world since its last change.
static inline NphResult nph_view_import(NphPhysicsWorld *w, const NphGpuWorldView *v, f32 dt)
{
    if (v->body_count != w->awake_bodies.len) {
        return NPH_RESULT_INVALID_STATE;
    }
    for (u32 i = 0U; i < v->body_count; ++i) {
        PhysBody *b = &w->bodies.data[w->awake_bodies.data[i]];
        const NphGpuBody *o = &v->bodies[i];
        b->center = nph_dvec3(o->center[0], o->center[1], o->center[2]);
        b->origin = nph_dvec3(o->origin[0], o->origin[1], o->origin[2]);
        memcpy(&b->rotation, o->rotation, sizeof o->rotation);
        memcpy(&b->linear_velocity, o->linear_velocity, sizeof o->linear_velocity);
        memcpy(&b->angular_velocity, o->angular_velocity, sizeof o->angular_velocity);
        b->force = nph_vec3_zero();
        b->torque = nph_vec3_zero();
        b->sleep_time = o->sleep_time;
        phys_body_refresh_boxes(w, b);
    }
    u32 nc = 0U;
    u32 nj = 0U;
    for (u32 c = 0U; c <= PHYS_GRAPH_COLORS; ++c) {
        const NphArrayU32 *list = nph_view_contact_list(w, c);
        for (u32 i = 0U; i < list->len; ++i) {
            PhysContact *ct = &w->contacts.data[list->data[i]];
            const NphGpuContact *o = &v->contacts[nc++];
            ct->flags = (ct->flags & ~(u32)PHYS_CONTACT_HIT) | (o->flags & PHYS_CONTACT_HIT);
            for (u32 k = 0U; k < ct->point_count; ++k) {
                PhysContactPoint *p = &ct->points[k];
                p->normal_impulse = o->points[k].normal_impulse;
                p->max_normal_impulse = o->points[k].max_normal_impulse;
                p->relative_velocity = o->points[k].relative_velocity;
                memcpy(&p->tangent_impulse, o->points[k].tangent_impulse,
                       sizeof o->points[k].tangent_impulse);
            }
        }
        const NphArrayU32 *jl = nph_view_joint_list(w, c);
        for (u32 i = 0U; i < jl->len; ++i) {
            PhysJoint *j = &w->joints.data[jl->data[i]];
            const NphGpuJoint *o = &v->joints[nj++];
            memcpy(&j->linear_impulse, o->linear_impulse, sizeof o->linear_impulse);
            memcpy(&j->angular_impulse, o->angular_impulse, sizeof o->angular_impulse);
            memcpy(&j->friction_impulse, o->friction_impulse, sizeof o->friction_impulse);
            j->lower_impulse = o->lower_impulse;
            j->upper_impulse = o->upper_impulse;
            j->swing_impulse = o->swing_impulse;
            j->motor_impulse = o->motor_impulse;
            j->spring_impulse = o->spring_impulse;
            memcpy(j->axis_impulse, o->axis_impulse, sizeof o->axis_impulse);
            j->flags = (j->flags & ~(u32)NPH_VIEW_JOINT_BLOCKS) | (o->flags & NPH_VIEW_JOINT_BLOCKS);
        }
    }
    w->last_substep = dt / (f32)w->desc.substeps;
    return NPH_RESULT_OK;
}

// The packed records of nph_gpu_phys_solve_packed, gathered straight from the world: the fields
// the stage reads.
static inline void nph_view_body_input(const PhysBody *b, NphGpuBodyInput *o)
{
    o->center[0] = b->center.x;
    o->center[1] = b->center.y;
    o->center[2] = b->center.z;
    memcpy(o->rotation, &b->rotation, sizeof o->rotation);
    memcpy(o->local_center, &b->local_center, sizeof o->local_center);
    memcpy(o->linear_velocity, &b->linear_velocity, sizeof o->linear_velocity);
    memcpy(o->angular_velocity, &b->angular_velocity, sizeof o->angular_velocity);
    memcpy(o->force, &b->force, sizeof o->force);
    memcpy(o->torque, &b->torque, sizeof o->torque);
    memcpy(o->inertia, &b->inertia, sizeof o->inertia);
    memcpy(o->inv_inertia, &b->inv_inertia, sizeof o->inv_inertia);
    o->inv_mass = b->inv_mass;
    o->linear_damping = b->linear_damping;
    o->angular_damping = b->angular_damping;
    o->gravity_scale = b->gravity_scale;
    o->sleep_threshold = b->sleep_threshold;
    o->sleep_time = b->sleep_time;
    o->max_extent = b->max_extent;
    o->type = b->type;
    o->flags = b->flags;
    o->locks = b->locks;
    o->pad = 0U;
}

static inline void nph_view_contact_input(const NphPhysicsWorld *w, NphViewMap *m, const PhysContact *c,
                                          NphGpuContactInput *o, u32 *fixed_count)
{
    memset(o, 0, sizeof *o);
    o->body_a = nph_view_index(w, m, c->body_a, fixed_count);
    o->body_b = nph_view_index(w, m, c->body_b, fixed_count);
    o->flags = c->flags & (PHYS_CONTACT_HIT | PHYS_CONTACT_HIT_EVENTS);
    o->point_count = c->point_count;
    memcpy(o->normal, &c->normal, sizeof o->normal);
    o->friction = c->friction;
    o->restitution = c->restitution;
    for (u32 k = 0U; k < c->point_count; ++k) {
        const PhysContactPoint *p = &c->points[k];
        NphGpuContactPointInput *q = &o->points[k];
        memcpy(q->anchor_a, &p->anchor_a, sizeof q->anchor_a);
        memcpy(q->anchor_b, &p->anchor_b, sizeof q->anchor_b);
        q->separation = p->separation;
        q->normal_impulse = p->normal_impulse;
        memcpy(q->tangent_impulse, &p->tangent_impulse, sizeof q->tangent_impulse);
        q->id = p->id;
    }
}

// Fills the packed input (its arrays sized by nph_view_sizes with the same map; joints and fixed
// bodies as whole records). Returns 0, or 1 when the world changed since the sizes were taken.
static inline int nph_view_export_packed(const NphPhysicsWorld *w, NphViewMap *m, NphGpuBodyInput *bodies,
                                         NphGpuBody *fixed_bodies, NphGpuContactInput *contacts,
                                         NphGpuJoint *joints, NphGpuPackedInput *in)
{
    u32 fixed = 0U;
    if (nph_view_map_fixed(w, m, &fixed) != NPH_RESULT_OK) {
        return 1;
    }
    memset(in, 0, sizeof *in);
    in->bodies = bodies;
    in->fixed_bodies = fixed_bodies;
    in->contacts = contacts;
    in->joints = joints;
    in->body_count = w->awake_bodies.len;
    for (u32 i = 0U; i < w->awake_bodies.len; ++i) {
        nph_view_body_input(&w->bodies.data[w->awake_bodies.data[i]], &bodies[i]);
    }
    in->fixed_count = fixed;
    for (u32 i = 0U; i < fixed; ++i) {
        nph_view_body_record(&w->bodies.data[m->fixed_slots[i]], &fixed_bodies[i]);
    }
    u32 nc = 0U;
    u32 nj = 0U;
    u32 again = fixed;
    for (u32 c = 0U; c <= PHYS_GRAPH_COLORS; ++c) {
        const NphArrayU32 *list = nph_view_contact_list(w, c);
        in->contact_color_counts[c] = list->len;
        for (u32 i = 0U; i < list->len; ++i) {
            nph_view_contact_input(w, m, &w->contacts.data[list->data[i]], &contacts[nc++], &again);
        }
        const NphArrayU32 *jl = nph_view_joint_list(w, c);
        in->joint_color_counts[c] = jl->len;
        for (u32 i = 0U; i < jl->len; ++i) {
            nph_view_joint_record(w, m, &w->joints.data[jl->data[i]], &joints[nj++], &again);
        }
    }
    in->contact_count = nc;
    in->joint_count = nj;
    return again == fixed ? 0 : 1;
}

// Writes the packed outputs back into the world, as nph_view_import does the whole records'.
static inline NphResult nph_view_import_packed(NphPhysicsWorld *w, const NphGpuPackedOutput *out,
                                               u32 body_count, f32 dt)
{
    if (body_count != w->awake_bodies.len) {
        return NPH_RESULT_INVALID_STATE;
    }
    for (u32 i = 0U; i < body_count; ++i) {
        PhysBody *b = &w->bodies.data[w->awake_bodies.data[i]];
        const NphGpuBodyOutput *o = &out->bodies[i];
        b->center = nph_dvec3(o->center[0], o->center[1], o->center[2]);
        b->origin = nph_dvec3(o->origin[0], o->origin[1], o->origin[2]);
        memcpy(&b->rotation, o->rotation, sizeof o->rotation);
        memcpy(&b->linear_velocity, o->linear_velocity, sizeof o->linear_velocity);
        memcpy(&b->angular_velocity, o->angular_velocity, sizeof o->angular_velocity);
        b->force = nph_vec3_zero();
        b->torque = nph_vec3_zero();
        b->sleep_time = o->sleep_time;
        phys_body_refresh_boxes(w, b);
    }
    u32 nc = 0U;
    u32 nj = 0U;
    for (u32 c = 0U; c <= PHYS_GRAPH_COLORS; ++c) {
        const NphArrayU32 *list = nph_view_contact_list(w, c);
        for (u32 i = 0U; i < list->len; ++i) {
            PhysContact *ct = &w->contacts.data[list->data[i]];
            const NphGpuContactOutput *o = &out->contacts[nc++];
            ct->flags = (ct->flags & ~(u32)PHYS_CONTACT_HIT) | (o->flags & PHYS_CONTACT_HIT);
            for (u32 k = 0U; k < ct->point_count; ++k) {
                PhysContactPoint *p = &ct->points[k];
                p->normal_impulse = o->points[k].normal_impulse;
                p->max_normal_impulse = o->points[k].max_normal_impulse;
                p->relative_velocity = o->points[k].relative_velocity;
                memcpy(&p->tangent_impulse, o->points[k].tangent_impulse,
                       sizeof o->points[k].tangent_impulse);
            }
        }
        const NphArrayU32 *jl = nph_view_joint_list(w, c);
        for (u32 i = 0U; i < jl->len; ++i) {
            PhysJoint *j = &w->joints.data[jl->data[i]];
            const NphGpuJointOutput *o = &out->joints[nj++];
            memcpy(&j->linear_impulse, o->linear_impulse, sizeof o->linear_impulse);
            memcpy(&j->angular_impulse, o->angular_impulse, sizeof o->angular_impulse);
            memcpy(&j->friction_impulse, o->friction_impulse, sizeof o->friction_impulse);
            j->lower_impulse = o->lower_impulse;
            j->upper_impulse = o->upper_impulse;
            j->swing_impulse = o->swing_impulse;
            j->motor_impulse = o->motor_impulse;
            j->spring_impulse = o->spring_impulse;
            memcpy(j->axis_impulse, o->axis_impulse, sizeof o->axis_impulse);
            j->flags = (j->flags & ~(u32)NPH_VIEW_JOINT_BLOCKS) | (o->flags & NPH_VIEW_JOINT_BLOCKS);
        }
    }
    w->last_substep = dt / (f32)w->desc.substeps;
    return NPH_RESULT_OK;
}

// The finalize pass's proxy growth (solver.c:867-878) for one awake body: shapes whose boxes
// left their proxies get them enlarged and pushed onto the move buffer.
static inline NphResult nph_view_grow_proxies(NphPhysicsWorld *w, PhysBody *b)
{
    if ((b->flags & PHYS_BODY_ENLARGED) == 0U) {
        return NPH_RESULT_OK;
    }
    b->flags &= ~(u32)PHYS_BODY_ENLARGED;
    for (u32 s = b->shape_head; s != PHYS_NULL; s = w->shapes.data[s].next) {
        PhysShape *shape = &w->shapes.data[s];
        if ((shape->flags & PHYS_SHAPE_ENLARGED) != 0U) {
            shape->flags &= ~(u32)PHYS_SHAPE_ENLARGED;
            nph_aabb_tree_enlarge_proxy(&w->trees[shape->tree], shape->proxy, shape->fat_aabb);
            NPH_TRY(phys_move_buffer_push(w, s));
        }
    }
    return NPH_RESULT_OK;
}

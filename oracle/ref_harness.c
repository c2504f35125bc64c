// SPDX-License-Identifier: Apache-2.0
//
// TEST INFRASTRUCTURE (the oracle), never the product: a white-box harness around the
// reference engine's physics, compiled together with the reference's own sources
// (oracle/Makefile) into oracle/_ref/libnphref.so. Only the tests, the smoke check and the
// bench's CPU-baseline leg load it.
//
// It builds reference worlds (bodies and shapes through the public API; joints through
// nph_physics_joint_create; synthetic manifolds injected into the world's contact array
// and coloured by the reference's own phys_graph_add, island.c:77), runs the reference's
// stages one by one (phys_update_pairs, phys_collide, phys_solve; world.c:332-346), and
// converts between the world and the solver-stage view of include/nepheline_b200.h:
//
//   export  the solver stage's inputs and outputs as NphGpuWorldView records, in the
//           reference's solver order (awake list; colours 0..23, then the overflow);
//   import  a view solved elsewhere back into the world, with what the reference's
//           finalize pass does beside the solver arithmetic (phys_body_refresh_boxes,
//           solver.c:351-369; growing the proxies of moved shapes, solver.c:867-878).
//
// All arithmetic of the step is the reference's: the harness only copies fields.

#include <nepheline/core/alloc.h>
#include <nepheline/core/hash.h>
#include <nepheline/jobs/jobs.h>
#include <nepheline/physics/body.h>
#include <nepheline/physics/joint.h>
#include <nepheline/physics/shape.h>
#include <nepheline/physics/world.h>

#include "world_internal.h"

#include "nepheline_b200.h"
#include "world_view.h" // the binding's world <-> view conversion (nepheline_b200/binding)

#include <stdlib.h>
#include <string.h>

#define REF_API __attribute__((visibility("default")))

enum { REF_CONSTRAINT_JOINT = 0, REF_CONSTRAINT_CONTACT = 1 };

typedef struct RefWorld {
    NphPhysicsWorld *w;
    NphJobSystem *js;
    NphPhysicsBody *bodies; // by creation index
    u32 body_count;
    u32 body_cap;
    u32 *kinds; // insertion order of constraints: kind and record index
    u32 *records;
    u32 constraint_count;
    u32 constraint_cap;
    NphViewMap map; // the last view's fixed bodies
} RefWorld;

static void *grow(void *p, u32 *cap, u32 need, size_t elem)
{
    if (need <= *cap) {
        return p;
    }
    u32 c = *cap > 0U ? *cap : 64U;
    while (c < need) {
        c *= 2U;
    }
    void *q = realloc(p, (size_t)c * elem);
    if (q == NULL) {
        abort();
    }
    *cap = c;
    return q;
}

REF_API RefWorld *nphref_world_create(const NphGpuWorldParams *p, u32 enable_sleep, u32 workers)
{
    NphPhysicsWorldDesc d = nph_physics_world_desc_default();
    d.alloc = nph_allocator_system();
    d.gravity = nph_vec3(p->gravity[0], p->gravity[1], p->gravity[2]);
    d.solver = (NphPhysicsSolver)p->solver;
    d.substeps = p->substeps;
    d.contact_hertz = p->contact_hertz;
    d.contact_damping_ratio = p->contact_damping_ratio;
    d.contact_push_max_velocity = p->contact_push_max_velocity;
    d.restitution_threshold = p->restitution_threshold;
    d.max_linear_speed = p->max_linear_speed;
    d.joint_hertz = p->joint_hertz;
    d.joint_damping_ratio = p->joint_damping_ratio;
    d.enable_continuous = p->enable_continuous != 0U ? 1 : 0;
    d.enable_sleep = enable_sleep != 0U ? 1 : 0;
    RefWorld *r = (RefWorld *)calloc(1, sizeof *r);
    if (r == NULL || nph_physics_world_create(&d, &r->w) != NPH_RESULT_OK) {
        free(r);
        return NULL;
    }
    if (workers != 0U) {
        NphJobSystemDesc jd;
        memset(&jd, 0, sizeof jd);
        jd.alloc = nph_allocator_system();
        jd.worker_count = workers == PHYS_NULL ? 0U : workers; // 0: logical cores - 1
        jd.pinning = NPH_JOB_PIN_NEVER;
        if (nph_job_system_create(&jd, &r->js) != NPH_RESULT_OK) {
            r->js = NULL;
        }
    }
    return r;
}

REF_API void nphref_world_destroy(RefWorld *r)
{
    if (r == NULL) {
        return;
    }
    nph_physics_world_destroy(r->w);
    if (r->js != NULL) {
        nph_job_system_destroy(r->js);
    }
    free(r->bodies);
    free(r->kinds);
    free(r->records);
    nph_view_map_release(&r->map);
    free(r);
}

REF_API u32 nphref_worker_count(const RefWorld *r)
{
    return r->js != NULL ? nph_job_system_worker_count(r->js) : 0U;
}

// The white-box knob of the reference's determinism tests (world_internal.h:653).
REF_API void nphref_force_participants(RefWorld *r, u32 participants)
{
    r->w->forced_participants = participants;
}

static u32 push_body(RefWorld *r, NphPhysicsBody b)
{
    r->bodies = (NphPhysicsBody *)grow(r->bodies, &r->body_cap, r->body_count + 1U, sizeof *r->bodies);
    r->bodies[r->body_count] = b;
    return r->body_count++;
}

static void push_constraint(RefWorld *r, u32 kind, u32 record)
{
    u32 cap = r->constraint_cap;
    r->kinds = (u32 *)grow(r->kinds, &cap, r->constraint_count + 1U, sizeof(u32));
    cap = r->constraint_cap;
    r->records = (u32 *)grow(r->records, &cap, r->constraint_count + 1U, sizeof(u32));
    r->constraint_cap = cap;
    r->kinds[r->constraint_count] = kind;
    r->records[r->constraint_count] = record;
    r->constraint_count += 1U;
}

// shape: 0 none, 1 box (dims = half extents), 2 sphere (dims[0] = radius), 3 capsule
// (dims[0] = half height, dims[1] = radius). flags: bit 0 gyroscopic, bit 1 sleep enabled,
// bit 2 bullet. Returns the body's creation index, or PHYS_NULL.
REF_API u32 nphref_add_body(RefWorld *r, u32 type, const f64 position[3], const f32 rotation[4],
                            const f32 velocity[3], const f32 angular_velocity[3], u32 shape,
                            const f32 dims[3], f32 density, f32 friction, f32 restitution,
                            u32 flags)
{
    NphPhysicsBodyDesc bd = nph_physics_body_desc_default();
    bd.type = (NphPhysicsBodyType)type;
    bd.position = nph_dvec3(position[0], position[1], position[2]);
    bd.rotation = nph_quat(rotation[0], rotation[1], rotation[2], rotation[3]);
    bd.linear_velocity = nph_vec3(velocity[0], velocity[1], velocity[2]);
    bd.angular_velocity = nph_vec3(angular_velocity[0], angular_velocity[1], angular_velocity[2]);
    bd.gyroscopic = (flags & 1U) != 0U ? 1 : 0;
    bd.enable_sleep = (flags & 2U) != 0U ? 1 : 0;
    bd.bullet = (flags & 4U) != 0U ? 1 : 0;
    NphPhysicsBody b;
    if (nph_physics_body_create(r->w, &bd, &b) != NPH_RESULT_OK) {
        return PHYS_NULL;
    }
    if (shape != 0U) {
        NphPhysicsGeometry g;
        if (shape == 1U) {
            g = nph_physics_geometry_box(nph_vec3(dims[0], dims[1], dims[2]));
        } else if (shape == 2U) {
            g = nph_physics_geometry_sphere(dims[0]);
        } else {
            g = nph_physics_geometry_capsule(dims[0], dims[1]);
        }
        NphPhysicsShapeDesc sd = nph_physics_shape_desc_default(g);
        sd.density = density;
        sd.friction = friction;
        sd.restitution = restitution;
        sd.hit_events = (flags & 8U) != 0U ? 1 : 0;
        NphPhysicsShape s;
        if (nph_physics_shape_create(r->w, b, &sd, &s) != NPH_RESULT_OK) {
            return PHYS_NULL;
        }
    }
    return push_body(r, b);
}

// Sets a shapeless body's mass, centre of mass (body frame) and inertia (column-major).
REF_API void nphref_set_mass(RefWorld *r, u32 body, f32 mass, const f32 center[3],
                             const f32 inertia[9])
{
    NphPhysicsMassData m;
    memset(&m, 0, sizeof m);
    m.mass = mass;
    m.center = nph_vec3(center[0], center[1], center[2]);
    memcpy(&m.inertia, inertia, sizeof m.inertia);
    nph_physics_body_set_mass_data(r->w, r->bodies[body], &m);
}

// A joint between two bodies given by creation index; the record's body fields are ignored.
REF_API u32 nphref_add_joint(RefWorld *r, const NphGpuJoint *j, u32 body_a, u32 body_b)
{
    NphPhysicsJointDesc d = nph_physics_joint_desc_default((NphPhysicsJointType)j->type,
                                                           r->bodies[body_a], r->bodies[body_b]);
    d.frame_a.position = nph_vec3(j->frame_a_position[0], j->frame_a_position[1],
                                  j->frame_a_position[2]);
    d.frame_a.rotation = nph_quat(j->frame_a_rotation[0], j->frame_a_rotation[1],
                                  j->frame_a_rotation[2], j->frame_a_rotation[3]);
    d.frame_b.position = nph_vec3(j->frame_b_position[0], j->frame_b_position[1],
                                  j->frame_b_position[2]);
    d.frame_b.rotation = nph_quat(j->frame_b_rotation[0], j->frame_b_rotation[1],
                                  j->frame_b_rotation[2], j->frame_b_rotation[3]);
    if (j->type == NPH_GPU_JOINT_BALL) {
        d.ball.enable_swing_limit = (b32)j->u.ball.enable_swing_limit;
        d.ball.swing_y = j->u.ball.swing_y;
        d.ball.swing_z = j->u.ball.swing_z;
        d.ball.enable_twist_limit = (b32)j->u.ball.enable_twist_limit;
        d.ball.twist_lower = j->u.ball.twist_lower;
        d.ball.twist_upper = j->u.ball.twist_upper;
        d.ball.friction_torque = j->u.ball.friction_torque;
    } else if (j->type == NPH_GPU_JOINT_HINGE) {
        d.hinge.enable_limit = (b32)j->u.hinge.enable_limit;
        d.hinge.lower = j->u.hinge.lower;
        d.hinge.upper = j->u.hinge.upper;
        d.hinge.enable_motor = (b32)j->u.hinge.enable_motor;
        d.hinge.motor_speed = j->u.hinge.motor_speed;
        d.hinge.max_motor_torque = j->u.hinge.max_motor_torque;
        d.hinge.enable_spring = (b32)j->u.hinge.enable_spring;
        d.hinge.spring_hertz = j->u.hinge.spring_hertz;
        d.hinge.spring_damping_ratio = j->u.hinge.spring_damping_ratio;
        d.hinge.spring_target = j->u.hinge.spring_target;
    } else if (j->type == NPH_GPU_JOINT_SLIDER) {
        d.slider.enable_limit = (b32)j->u.slider.enable_limit;
        d.slider.lower = j->u.slider.lower;
        d.slider.upper = j->u.slider.upper;
        d.slider.enable_motor = (b32)j->u.slider.enable_motor;
        d.slider.motor_speed = j->u.slider.motor_speed;
        d.slider.max_motor_force = j->u.slider.max_motor_force;
        d.slider.enable_spring = (b32)j->u.slider.enable_spring;
        d.slider.spring_hertz = j->u.slider.spring_hertz;
        d.slider.spring_damping_ratio = j->u.slider.spring_damping_ratio;
        d.slider.spring_target = j->u.slider.spring_target;
    } else if (j->type == NPH_GPU_JOINT_DISTANCE) {
        d.distance.length = j->u.distance.length;
        d.distance.enable_limit = (b32)j->u.distance.enable_limit;
        d.distance.min_length = j->u.distance.min_length;
        d.distance.max_length = j->u.distance.max_length;
        d.distance.enable_spring = (b32)j->u.distance.enable_spring;
        d.distance.spring_hertz = j->u.distance.spring_hertz;
        d.distance.spring_damping_ratio = j->u.distance.spring_damping_ratio;
        d.distance.enable_motor = (b32)j->u.distance.enable_motor;
        d.distance.motor_speed = j->u.distance.motor_speed;
        d.distance.max_motor_force = j->u.distance.max_motor_force;
    } else if (j->type == NPH_GPU_JOINT_D6) {
        for (u32 i = 0U; i < NPH_PHYSICS_D6_AXES; ++i) {
            const NphGpuD6Axis *x = &j->u.d6[i];
            NphPhysicsD6Axis *y = &d.d6.axes[i];
            y->motion = (NphPhysicsAxisMotion)x->motion;
            y->lower = x->lower;
            y->upper = x->upper;
            y->enable_motor = (b32)x->enable_motor;
            y->motor_speed = x->motor_speed;
            y->max_motor_force = x->max_motor_force;
            y->enable_spring = (b32)x->enable_spring;
            y->spring_hertz = x->spring_hertz;
            y->spring_damping_ratio = x->spring_damping_ratio;
            y->spring_target = x->spring_target;
        }
    }
    NphPhysicsJoint out;
    if (nph_physics_joint_create(r->w, &d, &out) != NPH_RESULT_OK) {
        return PHYS_NULL;
    }
    const u32 slot = phys_handle_slot(out.value);
    push_constraint(r, REF_CONSTRAINT_JOINT, slot);
    return slot;
}

// A touching manifold between two bodies (creation indices in the record's body fields),
// placed in the world's contact array and added to the constraint graph by the reference's
// phys_graph_add (island.c:77). For solver-only scenes: the bodies have no shapes, so no
// narrow phase ever replaces the manifold.
REF_API u32 nphref_inject_contact(RefWorld *r, const NphGpuContact *in)
{
    NphPhysicsWorld *w = r->w;
    PhysContact *c = NPH_ARRAY_PUSH_SLOT(&w->contacts);
    if (c == NULL) {
        return PHYS_NULL;
    }
    const u32 index = w->contacts.len - 1U;
    memset(c, 0, sizeof *c);
    c->shape_a = 0U;
    c->shape_b = 0U;
    c->body_a = phys_handle_slot(r->bodies[in->body_a].value);
    c->body_b = phys_handle_slot(r->bodies[in->body_b].value);
    c->flags = PHYS_CONTACT_TOUCHING | (in->flags & (NPH_GPU_CONTACT_HIT | NPH_GPU_CONTACT_HIT_EVENTS));
    c->parent = PHYS_NULL;
    c->child = PHYS_NULL;
    c->prev[0] = c->prev[1] = PHYS_NULL;
    c->next[0] = c->next[1] = PHYS_NULL;
    c->color = PHYS_NULL;
    c->color_slot = PHYS_NULL;
    c->island = PHYS_NULL;
    c->island_prev = PHYS_NULL;
    c->island_next = PHYS_NULL;
    c->awake_slot = PHYS_NULL;
    c->friction = in->friction;
    c->restitution = in->restitution;
    c->normal = nph_vec3(in->normal[0], in->normal[1], in->normal[2]);
    c->point_count = in->point_count;
    for (u32 k = 0U; k < in->point_count; ++k) {
        const NphGpuContactPoint *p = &in->points[k];
        PhysContactPoint *q = &c->points[k];
        q->anchor_a = nph_vec3(p->anchor_a[0], p->anchor_a[1], p->anchor_a[2]);
        q->anchor_b = nph_vec3(p->anchor_b[0], p->anchor_b[1], p->anchor_b[2]);
        q->separation = p->separation;
        q->id = p->id;
        q->normal_impulse = p->normal_impulse;
        q->max_normal_impulse = p->max_normal_impulse;
        q->tangent_impulse = nph_vec3(p->tangent_impulse[0], p->tangent_impulse[1],
                                      p->tangent_impulse[2]);
        q->relative_velocity = p->relative_velocity;
    }
    if (phys_graph_add(w, index) != NPH_RESULT_OK) {
        return PHYS_NULL;
    }
    push_constraint(r, REF_CONSTRAINT_CONTACT, index);
    return index;
}

// The world step's stages before and after the solver (world.c:332-339, 355-366).
REF_API int nphref_collide(RefWorld *r)
{
    NphResult res = phys_update_pairs(r->w, r->js);
    if (res == NPH_RESULT_OK) {
        res = phys_collide(r->w, r->js);
    }
    return (int)res;
}

REF_API int nphref_solve(RefWorld *r, f32 dt)
{
    r->w->step_dt = dt;
    NPH_ARRAY_CLEAR(&r->w->hit_events); // as the world step does before its stages (world.c:320)
    NPH_ARRAY_CLEAR(&r->w->move_events);
    return (int)phys_solve(r->w, dt, r->js);
}

// The hit events of the last solve (solver.c:919-960), in their order: approach speed, world
// point and normal; returns how many there are (at most `cap` written).
REF_API u32 nphref_hit_events(const RefWorld *r, u32 cap, f32 *approach, f64 *point, f32 *normal)
{
    const u32 n = r->w->hit_events.len;
    for (u32 i = 0U; i < n && i < cap; ++i) {
        const NphPhysicsContactHitEvent *e = &r->w->hit_events.data[i];
        approach[i] = e->approach_speed;
        point[3U * i + 0U] = e->point.x;
        point[3U * i + 1U] = e->point.y;
        point[3U * i + 2U] = e->point.z;
        normal[3U * i + 0U] = e->normal.x;
        normal[3U * i + 1U] = e->normal.y;
        normal[3U * i + 2U] = e->normal.z;
    }
    return n;
}

REF_API void nphref_set_hit_threshold(RefWorld *r, f32 speed) { nph_physics_world_set_hit_threshold(r->w, speed); }

REF_API int nphref_finish(RefWorld *r)
{
    NphResult res = phys_island_merge_pending(r->w);
    if (res == NPH_RESULT_OK && r->w->desc.enable_sleep != 0) {
        res = phys_island_sleep_and_split(r->w);
    }
    return (int)res;
}

// The island stage in its two halves (world.c:350-358), for a caller that decides between them:
// the merge of the step's links, then sleep and split.
REF_API int nphref_merge_islands(RefWorld *r)
{
    return (int)phys_island_merge_pending(r->w);
}

REF_API int nphref_sleep_islands(RefWorld *r)
{
    return r->w->desc.enable_sleep != 0 ? (int)phys_island_sleep_and_split(r->w) : 0;
}

// The islands as the sleep decision reads them (island.c:675-735), after the merge: per awake
// body (awake-list order: the view's) the place of its island in the awake-island list, or
// PHYS_NULL for a body in no island (kinematic); per awake island its record index and its
// constraint_remove_count. Returns the awake-island count (arrays of `cap` islands).
REF_API u32 nphref_island_view(const RefWorld *r, u32 *island_of, u32 *island_ids, u32 *removed, u32 cap)
{
    const NphPhysicsWorld *w = r->w;
    const u32 n = w->awake_islands.len;
    for (u32 k = 0U; k < n && k < cap; ++k) {
        island_ids[k] = w->awake_islands.data[k];
        removed[k] = w->islands.data[w->awake_islands.data[k]].constraint_remove_count;
    }
    for (u32 i = 0U; i < w->awake_bodies.len; ++i) {
        const PhysBody *b = &w->bodies.data[w->awake_bodies.data[i]];
        island_of[i] = b->island != PHYS_NULL ? w->islands.data[b->island].awake_slot : PHYS_NULL;
    }
    return n;
}

// An island record's constraint_remove_count and whether it is live and awake.
REF_API void nphref_island_state(const RefWorld *r, u32 island, u32 *removed, u32 *awake)
{
    const PhysIsland *is = &r->w->islands.data[island];
    *removed = is->constraint_remove_count;
    *awake = is->live != 0U && is->awake != 0U ? 1U : 0U;
}

// The creation index of each awake body, in awake-list order.
REF_API void nphref_awake_creation_ids(const RefWorld *r, u32 *out)
{
    const NphPhysicsWorld *w = r->w;
    for (u32 c = 0U; c < r->body_count; ++c) {
        const PhysBody *b = phys_body(w, r->bodies[c]);
        if (b != NULL && b->awake_slot != PHYS_NULL) {
            out[b->awake_slot] = c;
        }
    }
}

REF_API int nphref_step(RefWorld *r, f32 dt)
{
    return (int)nph_physics_world_step(r->w, dt, r->js);
}

REF_API u64 nphref_hash(const RefWorld *r)
{
    return nph_physics_world_hash(r->w);
}

REF_API double nphref_last_solve_ms(const RefWorld *r)
{
    return r->w->stats.solve_ms;
}

REF_API u32 nphref_body_count(const RefWorld *r)
{
    return r->body_count;
}

// A body's state by creation index: centre, origin, rotation, velocities, sleep time, flags.
REF_API void nphref_body_state(const RefWorld *r, u32 body, f64 center[3], f64 origin[3],
                               f32 rotation[4], f32 v[3], f32 w[3], f32 *sleep_time, u32 *flags)
{
    const PhysBody *b = phys_body(r->w, r->bodies[body]);
    center[0] = b->center.x;
    center[1] = b->center.y;
    center[2] = b->center.z;
    origin[0] = b->origin.x;
    origin[1] = b->origin.y;
    origin[2] = b->origin.z;
    memcpy(rotation, &b->rotation, sizeof(f32) * 4U);
    memcpy(v, &b->linear_velocity, sizeof(f32) * 3U);
    memcpy(w, &b->angular_velocity, sizeof(f32) * 3U);
    *sleep_time = b->sleep_time;
    *flags = b->flags;
}

// ---------------------------------------------------------------------------
// The colouring, in insertion order
// ---------------------------------------------------------------------------

REF_API u32 nphref_constraint_count(const RefWorld *r)
{
    return r->constraint_count;
}

// Per constraint in insertion order: its bodies' slots, which are dynamic (bit 0 A, bit 1 B),
// and the colour and slot the reference gave it (PHYS_GRAPH_OVERFLOW = 24).
REF_API void nphref_constraints(const RefWorld *r, u32 *body_a, u32 *body_b, u8 *dynamic_bits,
                                u32 *color, u32 *slot)
{
    const NphPhysicsWorld *w = r->w;
    for (u32 i = 0U; i < r->constraint_count; ++i) {
        u32 a;
        u32 b;
        if (r->kinds[i] == REF_CONSTRAINT_JOINT) {
            const PhysJoint *j = &w->joints.data[r->records[i]];
            a = j->body_a;
            b = j->body_b;
            color[i] = j->color;
            slot[i] = j->color_slot;
        } else {
            const PhysContact *c = &w->contacts.data[r->records[i]];
            a = c->body_a;
            b = c->body_b;
            color[i] = c->color;
            slot[i] = c->color_slot;
        }
        body_a[i] = a;
        body_b[i] = b;
        dynamic_bits[i] = (u8)((w->bodies.data[a].type == NPH_PHYSICS_BODY_DYNAMIC ? 1U : 0U) |
                               (w->bodies.data[b].type == NPH_PHYSICS_BODY_DYNAMIC ? 2U : 0U));
    }
}

REF_API u32 nphref_body_slots(const RefWorld *r)
{
    return r->w->bodies.len;
}

// ---------------------------------------------------------------------------
// World <-> view (the conversion is the binding's, nepheline_b200/binding/world_view.h)
// ---------------------------------------------------------------------------

// The sizes a view of the world needs.
REF_API void nphref_view_sizes(RefWorld *r, u32 *bodies, u32 *fixed, u32 *contacts, u32 *joints)
{
    if (nph_view_sizes(r->w, &r->map, bodies, fixed, contacts, joints) != NPH_RESULT_OK) {
        abort();
    }
}

// Fills a view whose arrays the caller sized by nphref_view_sizes.
REF_API int nphref_export(RefWorld *r, NphGpuWorldView *v) { return nph_view_export(r->w, &r->map, v); }

// Writes a solved view back into the world: what phys_solve's stages write
// (finalize_body, store_group, the joints' impulses), then the finalize pass's box refresh
// and the growth of moved proxies (solver.c:351-369, 867-878). The view must have been
// exported from this world since its last change.
REF_API int nphref_import(RefWorld *r, const NphGpuWorldView *v, f32 dt)
{
    NphPhysicsWorld *w = r->w;
    NphResult res = nph_view_import(w, v, dt);
    for (u32 i = 0U; res == NPH_RESULT_OK && i < w->awake_bodies.len; ++i) {
        res = nph_view_grow_proxies(w, &w->bodies.data[w->awake_bodies.data[i]]);
    }
    return (int)res;
}

// The world's statistics the scenes report.
REF_API void nphref_stats(const RefWorld *r, u32 *touching, u32 *points, u32 *colors_used,
                          u32 *overflow, u32 *awake)
{
    const NphPhysicsStats s = nph_physics_world_stats(r->w);
    *touching = s.touching_contacts;
    *points = s.manifold_points;
    *colors_used = s.colors_used;
    *overflow = s.overflow_constraints;
    *awake = s.awake_bodies;
}

// ---------------------------------------------------------------------------
// Bulk scene building (solver-only scenes of shapeless bodies)
// ---------------------------------------------------------------------------

// Dynamic (or the record's type) shapeless bodies at the records' centres, with the records'
// rotation, velocities, damping, gravity scale, sleep settings and mass properties (`mass`
// per body; the record's inertia, column-major, and local centre). Returns the first
// creation index, or PHYS_NULL.
REF_API u32 nphref_add_shapeless_bodies(RefWorld *r, u32 n, const NphGpuBody *recs,
                                        const f32 *mass)
{
    const u32 first = r->body_count;
    for (u32 i = 0U; i < n; ++i) {
        const NphGpuBody *o = &recs[i];
        NphPhysicsBodyDesc bd = nph_physics_body_desc_default();
        bd.type = (NphPhysicsBodyType)o->type;
        const NphQuat q = nph_quat(o->rotation[0], o->rotation[1], o->rotation[2], o->rotation[3]);
        const NphVec3 lc = nph_vec3(o->local_center[0], o->local_center[1], o->local_center[2]);
        bd.position = nph_dvec3_add_vec3(nph_dvec3(o->center[0], o->center[1], o->center[2]),
                                         nph_vec3_neg(nph_quat_rotate(q, lc)));
        bd.rotation = q;
        bd.linear_velocity = nph_vec3(o->linear_velocity[0], o->linear_velocity[1],
                                      o->linear_velocity[2]);
        bd.angular_velocity = nph_vec3(o->angular_velocity[0], o->angular_velocity[1],
                                       o->angular_velocity[2]);
        bd.linear_damping = o->linear_damping;
        bd.angular_damping = o->angular_damping;
        bd.gravity_scale = o->gravity_scale;
        bd.sleep_threshold = o->sleep_threshold;
        bd.locks = o->locks;
        bd.enable_sleep = (o->flags & NPH_GPU_BODY_ENABLE_SLEEP) != 0U ? 1 : 0;
        bd.gyroscopic = (o->flags & NPH_GPU_BODY_GYROSCOPIC) != 0U ? 1 : 0;
        bd.bullet = (o->flags & NPH_GPU_BODY_BULLET) != 0U ? 1 : 0;
        NphPhysicsBody b;
        if (nph_physics_body_create(r->w, &bd, &b) != NPH_RESULT_OK) {
            return PHYS_NULL;
        }
        const u32 index = push_body(r, b);
        if (o->type == NPH_GPU_BODY_DYNAMIC) {
            nphref_set_mass(r, index, mass[i], o->local_center, o->inertia);
        }
        if (o->force[0] != 0.0F || o->force[1] != 0.0F || o->force[2] != 0.0F) {
            nph_physics_body_apply_force_at_center(
                r->w, b, nph_vec3(o->force[0], o->force[1], o->force[2]));
        }
        if (o->torque[0] != 0.0F || o->torque[1] != 0.0F || o->torque[2] != 0.0F) {
            nph_physics_body_apply_torque(r->w, b,
                                          nph_vec3(o->torque[0], o->torque[1], o->torque[2]));
        }
    }
    return first;
}

// Joints in insertion order; the records' body fields are creation indices.
REF_API u32 nphref_add_joints(RefWorld *r, u32 n, const NphGpuJoint *recs)
{
    for (u32 i = 0U; i < n; ++i) {
        if (nphref_add_joint(r, &recs[i], recs[i].body_a, recs[i].body_b) == PHYS_NULL) {
            return PHYS_NULL;
        }
    }
    return n;
}

// Manifolds in insertion order; the records' body fields are creation indices.
REF_API u32 nphref_inject_contacts(RefWorld *r, u32 n, const NphGpuContact *recs)
{
    if (NPH_ARRAY_RESERVE(&r->w->contacts, r->w->contacts.len + n) != NPH_RESULT_OK) {
        return PHYS_NULL;
    }
    for (u32 i = 0U; i < n; ++i) {
        if (nphref_inject_contact(r, &recs[i]) == PHYS_NULL) {
            return PHYS_NULL;
        }
    }
    return n;
}

// Sets every dynamic awake body's velocities (by creation index) between steps.
REF_API void nphref_set_velocity(RefWorld *r, u32 body, const f32 v[3], const f32 w[3])
{
    nph_physics_body_set_linear_velocity(r->w, r->bodies[body], nph_vec3(v[0], v[1], v[2]));
    nph_physics_body_set_angular_velocity(r->w, r->bodies[body], nph_vec3(w[0], w[1], w[2]));
}

/* The reference's narrow phase for `count` pairs of convex shapes (nph_physics_collide,
 * collide.c:524-535), in the device library's records. */
REF_API void nphref_collide_pairs(const NphGpuShape *a, const NphGpuPose *pa, const NphGpuShape *b,
                                  const NphGpuPose *pb, const float *spec, uint32_t count,
                                  NphGpuManifold *out)
{
    for (uint32_t i = 0U; i < count; ++i) {
        NphPhysicsGeometry g[2];
        const NphGpuShape *sh[2] = {&a[i], &b[i]};
        for (uint32_t k = 0U; k < 2U; ++k) {
            const NphGpuShape *s = sh[k];
            if (s->type == NPH_GPU_SHAPE_SPHERE) {
                g[k] = nph_physics_geometry_sphere(s->dims[0]);
            } else if (s->type == NPH_GPU_SHAPE_CAPSULE) {
                g[k] = nph_physics_geometry_capsule(s->dims[0], s->dims[1]);
            } else {
                g[k] = nph_physics_geometry_box(nph_vec3(s->dims[0], s->dims[1], s->dims[2]));
            }
        }
        const NphPhysicsPose p0 = nph_physics_pose(
            nph_vec3(pa[i].position[0], pa[i].position[1], pa[i].position[2]),
            nph_quat(pa[i].rotation[0], pa[i].rotation[1], pa[i].rotation[2], pa[i].rotation[3]));
        const NphPhysicsPose p1 = nph_physics_pose(
            nph_vec3(pb[i].position[0], pb[i].position[1], pb[i].position[2]),
            nph_quat(pb[i].rotation[0], pb[i].rotation[1], pb[i].rotation[2], pb[i].rotation[3]));
        NphPhysicsManifold m;
        memset(&m, 0, sizeof m);
        nph_physics_collide(&g[0], p0, &g[1], p1, spec[i], NULL, &m);
        memset(&out[i], 0, sizeof out[i]);
        out[i].normal[0] = m.normal.x;
        out[i].normal[1] = m.normal.y;
        out[i].normal[2] = m.normal.z;
        out[i].point_count = m.point_count;
        for (uint32_t k = 0U; k < m.point_count; ++k) {
            out[i].points[k].point[0] = m.points[k].point.x;
            out[i].points[k].point[1] = m.points[k].point.y;
            out[i].points[k].point[2] = m.points[k].point.z;
            out[i].points[k].separation = m.points[k].separation;
            out[i].points[k].id = m.points[k].id;
        }
    }
}

// SPDX-License-Identifier: Apache-2.0
//
// The binding that puts the device solver behind the reference engine's world step: compiled
// into the engine's physics library beside its own sources, with world.c compiled as
//
//     cc ... -Dphys_solve=phys_solve_dispatch -c engine/physics/src/world.c
//
// so the solver stage's one call (world.c:346) comes here, with no edit to the engine's
// sources. phys_solve_dispatch does what phys_solve (solver.c:961-1105) does, in its order:
// the stage's arithmetic on the device (nph_gpu_phys_solve_packed over the world's packed
// records: only the fields the stage reads go up, only those it writes come back), its results
// written back into the world (finalize_body, store_group, the joints' impulses, the box
// refresh), then the host work after the arithmetic: post_finalize (solver.c:847-917: driven
// joints keep their bodies awake, the CCD flags cleared, enlarged proxies grown, one move event
// per awake body, moving kinematic bodies waking what they touch) and hit_events
// (solver.c:919-960, the hits found on the device from its resident records).
//
// Settings the device solver does not run (XPBD, continuous collision) return
// NPH_RESULT_UNSUPPORTED from the step: there is no fallback to the CPU stage. With no solver
// attached (nph_gpu_binding_attach), the engine's own phys_solve runs: the engine chooses its
// solver stage once, before stepping, as it chooses its SIMD kernels (world.c:132).

#include "world_view.h"

#include <nepheline/physics/world.h>
#include <nepheline/platform/time.h>

// The packed records' arrays, kept between steps and grown as the world grows.
typedef struct Binding {
    NphGpuSolver *solver;
    NphViewMap map;
    NphGpuBodyInput *bodies;
    NphGpuBody *fixed;
    NphGpuContactInput *contacts;
    NphGpuJoint *joints;
    NphGpuBodyOutput *out_bodies;
    NphGpuContactOutput *out_contacts;
    NphGpuJointOutput *out_joints;
    NphGpuHitEvent *hits;
    u32 body_cap, fixed_cap, contact_cap, joint_cap, out_body_cap, out_contact_cap, out_joint_cap, hit_cap;
} Binding;

static Binding g_binding;

// Attaches the device solver every following world step uses as its solver stage (NULL: the
// engine's own stage). One thread steps the world, as for the engine (world.h:45-46).
void nph_gpu_binding_attach(NphGpuSolver *solver) { g_binding.solver = solver; }

// Frees the arrays the binding keeps.
void nph_gpu_binding_release(void)
{
    nph_view_map_release(&g_binding.map);
    free(g_binding.bodies);
    free(g_binding.fixed);
    free(g_binding.contacts);
    free(g_binding.joints);
    free(g_binding.out_bodies);
    free(g_binding.out_contacts);
    free(g_binding.out_joints);
    free(g_binding.hits);
    memset(&g_binding, 0, sizeof g_binding);
}

NphResult phys_solve(NphPhysicsWorld *w, f32 dt, NphJobSystem *js); // the engine's own stage
NphResult phys_solve_dispatch(NphPhysicsWorld *w, f32 dt, NphJobSystem *js);

static NphResult reserve(void **p, u32 *cap, u32 need, size_t elem)
{
    if (need <= *cap) {
        return NPH_RESULT_OK;
    }
    const u32 c = need + need / 2U + 16U;
    void *q = realloc(*p, (size_t)c * elem);
    if (q == NULL) {
        return NPH_RESULT_OUT_OF_MEMORY;
    }
    *p = q;
    *cap = c;
    return NPH_RESULT_OK;
}

static NphGpuWorldParams params_from_desc(const NphPhysicsWorldDesc *d)
{
    NphGpuWorldParams p;
    memset(&p, 0, sizeof p);
    p.gravity[0] = d->gravity.x;
    p.gravity[1] = d->gravity.y;
    p.gravity[2] = d->gravity.z;
    p.solver = (uint32_t)d->solver;
    p.substeps = d->substeps;
    p.contact_hertz = d->contact_hertz;
    p.contact_damping_ratio = d->contact_damping_ratio;
    p.contact_push_max_velocity = d->contact_push_max_velocity;
    p.restitution_threshold = d->restitution_threshold;
    p.max_linear_speed = d->max_linear_speed;
    p.joint_hertz = d->joint_hertz;
    p.joint_damping_ratio = d->joint_damping_ratio;
    p.enable_continuous = d->enable_continuous != 0 ? 1U : 0U;
    return p;
}

// post_finalize (solver.c:847-917) after the device's write-back. The device already reset the
// sleep clocks of awake bodies on driven joints; the host does it again for every body a
// driven joint names, fixed bodies included, as the reference does.
static NphResult post_finalize(NphPhysicsWorld *w)
{
    for (u32 c = 0U; c <= PHYS_GRAPH_COLORS; ++c) {
        const NphArrayU32 *jl = nph_view_joint_list(w, c);
        for (u32 i = 0U; i < jl->len; ++i) {
            const PhysJoint *j = &w->joints.data[jl->data[i]];
            if (phys_joint_is_driven(j)) {
                w->bodies.data[j->body_a].sleep_time = 0.0F;
                w->bodies.data[j->body_b].sleep_time = 0.0F;
            }
        }
    }
    NPH_TRY(NPH_ARRAY_RESERVE(&w->move_events, w->awake_bodies.len));
    w->stats.swept_bodies = 0U;
    w->stats.impact_bodies = 0U;
    for (u32 i = 0U; i < w->awake_bodies.len; ++i) {
        PhysBody *b = &w->bodies.data[w->awake_bodies.data[i]];
        b->flags &= ~(u32)(PHYS_BODY_SWEPT | PHYS_BODY_IMPACT | PHYS_BODY_FAST);
        NPH_TRY(nph_view_grow_proxies(w, b));
        NphPhysicsBodyMoveEvent e;
        e.body = (NphPhysicsBody){b->handle};
        e.fell_asleep = 0U;
        e.user_data = b->user_data;
        e.position = b->origin;
        e.rotation = b->rotation;
        e.linear_velocity = b->linear_velocity;
        e.angular_velocity = b->angular_velocity;
        b->move_event = w->move_events.len;
        NPH_TRY(NPH_ARRAY_PUSH(&w->move_events, e));
    }
    for (u32 i = 0U; i < w->awake_bodies.len; ++i) {
        const PhysBody *b = &w->bodies.data[w->awake_bodies.data[i]];
        if (b->type != NPH_PHYSICS_BODY_KINEMATIC || b->sleep_time > 0.0F) {
            continue;
        }
        for (u32 key = b->contact_head; key != PHYS_NULL;) {
            const PhysContact *c = &w->contacts.data[key >> 1U];
            const u32 other = (key & 1U) == 0U ? c->body_b : c->body_a;
            key = c->next[key & 1U];
            if ((c->flags & PHYS_CONTACT_TOUCHING) != 0U &&
                (w->bodies.data[other].flags & PHYS_BODY_AWAKE) == 0U) {
                NPH_TRY(phys_wake_body(w, other));
            }
        }
        for (u32 key = b->joint_head; key != PHYS_NULL;) {
            const PhysJoint *j = &w->joints.data[key >> 1U];
            const u32 other = (key & 1U) == 0U ? j->body_b : j->body_a;
            key = j->next[key & 1U];
            if ((w->bodies.data[other].flags & PHYS_BODY_AWAKE) == 0U) {
                NPH_TRY(phys_wake_body(w, other));
            }
        }
    }
    return NPH_RESULT_OK;
}

// hit_events (solver.c:919-960) from the device's scan: each event's manifold is the view's
// contact record in colour order, which is the order the colour lists give here.
static NphResult push_hits(NphPhysicsWorld *w, const NphGpuHitEvent *hits, u32 count)
{
    u32 cursor = 0U;
    u32 base = 0U;
    for (u32 c = 0U; c <= PHYS_GRAPH_COLORS && cursor < count; ++c) {
        const NphArrayU32 *list = nph_view_contact_list(w, c);
        while (cursor < count && hits[cursor].contact < base + list->len) {
            const NphGpuHitEvent *h = &hits[cursor++];
            const PhysContact *contact = &w->contacts.data[list->data[h->contact - base]];
            NphPhysicsContactHitEvent e;
            e.shape_a = phys_shape_handle(w, contact->shape_a);
            e.shape_b = phys_shape_handle(w, contact->shape_b);
            e.point = nph_dvec3_add_vec3(w->bodies.data[contact->body_a].center,
                                         contact->points[h->point].anchor_a);
            e.normal = contact->normal;
            e.approach_speed = h->approach_speed;
            NPH_TRY(NPH_ARRAY_PUSH(&w->hit_events, e));
        }
        base += list->len;
    }
    return NPH_RESULT_OK;
}

NphResult phys_solve_dispatch(NphPhysicsWorld *w, f32 dt, NphJobSystem *js)
{
    Binding *g = &g_binding;
    if (g->solver == NULL) {
        return phys_solve(w, dt, js);
    }
    if (w->desc.solver == NPH_PHYSICS_SOLVER_XPBD || w->desc.enable_continuous != 0) {
        return NPH_RESULT_UNSUPPORTED;
    }
    if (w->awake_bodies.len == 0U) {
        return NPH_RESULT_OK;
    }
    u32 nb = 0U, nf = 0U, nc = 0U, nj = 0U;
    NPH_TRY(nph_view_sizes(w, &g->map, &nb, &nf, &nc, &nj));
    NPH_TRY(reserve((void **)&g->bodies, &g->body_cap, nb, sizeof(NphGpuBodyInput)));
    NPH_TRY(reserve((void **)&g->fixed, &g->fixed_cap, nf, sizeof(NphGpuBody)));
    NPH_TRY(reserve((void **)&g->contacts, &g->contact_cap, nc, sizeof(NphGpuContactInput)));
    NPH_TRY(reserve((void **)&g->joints, &g->joint_cap, nj, sizeof(NphGpuJoint)));
    NPH_TRY(reserve((void **)&g->out_bodies, &g->out_body_cap, nb, sizeof(NphGpuBodyOutput)));
    NPH_TRY(reserve((void **)&g->out_contacts, &g->out_contact_cap, nc, sizeof(NphGpuContactOutput)));
    NPH_TRY(reserve((void **)&g->out_joints, &g->out_joint_cap, nj, sizeof(NphGpuJointOutput)));
    NPH_TRY(reserve((void **)&g->hits, &g->hit_cap, nc, sizeof(NphGpuHitEvent)));
    NphGpuPackedInput in;
    if (nph_view_export_packed(w, &g->map, g->bodies, g->fixed, g->contacts, g->joints, &in) != 0) {
        return NPH_RESULT_INVALID_STATE;
    }
    NphGpuPackedOutput out;
    out.bodies = g->out_bodies;
    out.contacts = g->out_contacts;
    out.joints = g->out_joints;
    const NphGpuWorldParams p = params_from_desc(&w->desc);
    const NphGpuResult r = nph_gpu_phys_solve_packed(g->solver, &p, dt, &in, &out);
    if (r != NPH_GPU_OK) {
        return (NphResult)r; // the world is untouched: the step did not happen
    }
    NPH_TRY(nph_view_import_packed(w, &out, in.body_count, dt));
    w->stats.workers = 1U;
    const u64 t = nph_time_now_ns();
    NPH_TRY(post_finalize(w));
    u32 hits = 0U;
    NPH_TRY((NphResult)nph_gpu_world_hit_events(g->solver, w->hit_threshold, g->hits, g->hit_cap, &hits));
    NPH_TRY(push_hits(w, g->hits, hits < g->hit_cap ? hits : g->hit_cap));
    w->stats.finalize_ms = (f64)(nph_time_now_ns() - t) * 1e-6;
    return NPH_RESULT_OK;
}

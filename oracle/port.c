// SPDX-License-Identifier: Apache-2.0
//
// TEST INFRASTRUCTURE (the oracle), never the product: the CPU restatement of the reference's
// solver stage (port_impl.h) instantiated in FP32 (bit-exact with the reference, checked
// against oracle/_ref/libnphref.so) and in FP64 (the error baseline), with the write-back of
// phys_solve's results into the view: finalize_body (solver.c:304-349), store_group
// (solver.c:475-499), the joints' impulses, and the driven joints' sleep reset of
// post_finalize (solver.c:851-857).

#include "nepheline_b200.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PORT_API __attribute__((visibility("default")))

// d6_config (joint_solver.c:399-421): a 6-DOF joint's axes, or a slider's (translation X
// free or limited with the slider's drives, the rest locked).
static void port_axes(const NphGpuJoint *j, NphGpuD6Axis out[NPH_GPU_D6_AXES])
{
    if (j->type == NPH_GPU_JOINT_D6) {
        memcpy(out, j->u.d6, sizeof j->u.d6);
        return;
    }
    memset(out, 0, sizeof(NphGpuD6Axis) * NPH_GPU_D6_AXES);
    const NphGpuSliderJoint *sl = &j->u.slider;
    out[0].motion = sl->enable_limit != 0U ? NPH_GPU_AXIS_LIMITED : NPH_GPU_AXIS_FREE;
    out[0].lower = sl->lower;
    out[0].upper = sl->upper;
    out[0].enable_motor = sl->enable_motor;
    out[0].motor_speed = sl->motor_speed;
    out[0].max_motor_force = sl->max_motor_force;
    out[0].enable_spring = sl->enable_spring;
    out[0].spring_hertz = sl->spring_hertz;
    out[0].spring_damping_ratio = sl->spring_damping_ratio;
    out[0].spring_target = sl->spring_target;
}

// all_locked (joint_solver.c:423-431).
static int port_all_locked(const NphGpuD6Axis *ax, unsigned first, unsigned count)
{
    for (unsigned i = first; i < first + count; ++i) {
        if (ax[i].motion != NPH_GPU_AXIS_LOCKED) {
            return 0;
        }
    }
    return 1;
}

#define REAL float
#define SUF _f32
#define SQRT sqrtf
#define ATAN2 atan2f
#define ABS fabsf
#include "port_impl.h"
#undef REAL
#undef SUF
#undef SQRT
#undef ATAN2
#undef ABS

#define REAL double
#define SUF _f64
#define SQRT sqrt
#define ATAN2 atan2
#define ABS fabs
#include "port_impl.h"
#undef REAL
#undef SUF
#undef SQRT
#undef ATAN2
#undef ABS

// Checks what the reference asserts or relies on: indices in range, 1..4 points, colour
// counts that add up, supported joint types and settings.
static int check_view(const NphGpuWorldParams *wp, const NphGpuWorldView *v)
{
    if (wp == NULL || v == NULL || wp->substeps == 0U ||
        (wp->solver != NPH_GPU_SOLVER_SOFT_STEP && wp->solver != NPH_GPU_SOLVER_TGS)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    const unsigned total = v->body_count + v->fixed_count;
    unsigned nc = 0U;
    unsigned nj = 0U;
    for (unsigned c = 0U; c < NPH_GPU_COLOR_SLOTS; ++c) {
        nc += v->contact_color_counts[c];
        nj += v->joint_color_counts[c];
    }
    if (nc != v->contact_count || nj != v->joint_count) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    for (unsigned i = 0U; i < v->contact_count; ++i) {
        const NphGpuContact *c = &v->contacts[i];
        if (c->body_a >= total || c->body_b >= total || c->point_count < 1U ||
            c->point_count > NPH_GPU_MAX_POINTS) {
            return NPH_GPU_INVALID_ARGUMENT;
        }
    }
    for (unsigned i = 0U; i < v->joint_count; ++i) {
        const NphGpuJoint *j = &v->joints[i];
        if (j->body_a >= total || j->body_b >= total) {
            return NPH_GPU_INVALID_ARGUMENT;
        }
        if (j->type > NPH_GPU_JOINT_D6) {
            return NPH_GPU_UNSUPPORTED;
        }
        if (j->type == NPH_GPU_JOINT_D6) {
            for (unsigned a = 0U; a < NPH_GPU_D6_AXES; ++a) {
                if (j->u.d6[a].motion > NPH_GPU_AXIS_FREE) {
                    return NPH_GPU_INVALID_ARGUMENT;
                }
            }
        }
    }
    if (wp->enable_continuous != 0U) {
        return NPH_GPU_UNSUPPORTED;
    }
    return NPH_GPU_OK;
}

// phys_joint_is_driven (joint_solver.c:1410-1434).
static int joint_is_driven(const NphGpuJoint *j)
{
    if (j->type == NPH_GPU_JOINT_HINGE) {
        return j->u.hinge.enable_motor != 0U && j->u.hinge.motor_speed != 0.0F &&
               j->u.hinge.max_motor_torque > 0.0F;
    }
    if (j->type == NPH_GPU_JOINT_DISTANCE) {
        return j->u.distance.enable_motor != 0U && j->u.distance.motor_speed != 0.0F &&
               j->u.distance.max_motor_force > 0.0F;
    }
    if (j->type == NPH_GPU_JOINT_SLIDER || j->type == NPH_GPU_JOINT_D6) {
        NphGpuD6Axis ax[NPH_GPU_D6_AXES];
        port_axes(j, ax);
        for (unsigned i = 0U; i < NPH_GPU_D6_AXES; ++i) {
            if (ax[i].motion != NPH_GPU_AXIS_LOCKED && ax[i].enable_motor != 0U &&
                ax[i].motor_speed != 0.0F && ax[i].max_motor_force > 0.0F) {
                return 1;
            }
        }
    }
    return 0;
}

// The FP32 write-back of a step into the view (finalize, store, joints, driven sleep reset).
static void write_back_f32(const Result_f32 *rp, float dt, NphGpuWorldView *v);

// The FP32 solve, in place on the view, as the device library's nph_gpu_phys_solve.
PORT_API int nph_port32_solve(const NphGpuWorldParams *wp, float dt, NphGpuWorldView *v)
{
    const int bad = check_view(wp, v);
    if (bad != NPH_GPU_OK) {
        return bad;
    }
    Result_f32 r;
    const int res = run_f32(wp, dt, v, &r);
    if (res != NPH_GPU_OK) {
        return res;
    }
    write_back_f32(&r, dt, v);
    return NPH_GPU_OK;
}

// The residual-driven mode (nph_gpu_world_converge) in FP32, the residual in double: residuals[0..passes], 1 + max_passes doubles.
PORT_API int nph_port32_converge(const NphGpuWorldParams *wp, float dt, const NphGpuWorldView *v,
                                 const float *init, double tol, unsigned max_passes, double ref,
                                 double *residuals, unsigned *passes, unsigned *cold, float *impulses)
{
    const int bad = check_view(wp, v);
    if (bad != NPH_GPU_OK) {
        return bad;
    }
    if (wp->solver != NPH_GPU_SOLVER_SOFT_STEP) {
        return NPH_GPU_UNSUPPORTED; // the residual-driven mode is the soft step's
    }
    return converge_f32(wp, dt, v, init, tol, max_passes, ref, residuals, passes, cold, impulses);
}

// The contact update's warm start for pairs of convex shapes (contact.c:332-380, 516-565),
// contact by contact: `old` last step's record of the pair (point_count 0 for a pair that
// starts touching), `fresh` the narrow phase's manifold (impulses zero); `out` the manifold
// with the pair and flags of the old record and the impulses its points carry over: by
// feature id first (the first old point with the id, claimed or not), then, when a point found
// no id and an old point is left, the nearest unclaimed old point in point order, its anchors
// within 2 x the linear slop on both bodies (the larger of the two squared distances).
PORT_API int nph_port_warm_update(const NphGpuContact *old, const NphGpuContact *fresh, unsigned count,
                                  NphGpuContact *out)
{
    const float reach = 2.0F * 0.005F;
    for (unsigned g = 0U; g < count; ++g) {
        const NphGpuContact *o = &old[g];
        NphGpuContact c = fresh[g];
        const unsigned oc = o->point_count, nc = c.point_count;
        if (oc > NPH_GPU_MAX_POINTS || nc > NPH_GPU_MAX_POINTS) {
            return NPH_GPU_INVALID_ARGUMENT;
        }
        c.body_a = o->body_a;
        c.body_b = o->body_b;
        c.flags = o->flags;
        unsigned taken = 0U, open = 0U;
        for (unsigned i = 0U; i < nc; ++i) {
            unsigned k = oc;
            for (unsigned q = 0U; q < oc && k == oc; ++q) {
                k = o->points[q].id == c.points[i].id ? q : oc;
            }
            if (k == oc) {
                open |= 1U << i;
                continue;
            }
            c.points[i].normal_impulse = o->points[k].normal_impulse;
            memcpy(c.points[i].tangent_impulse, o->points[k].tangent_impulse, sizeof(float) * 3U);
            taken |= 1U << k;
        }
        const unsigned all = (1U << oc) - 1U;
        for (unsigned i = 0U; i < nc && open != 0U && taken != all; ++i) {
            if ((open & (1U << i)) == 0U) {
                continue;
            }
            unsigned pick = NPH_GPU_NULL;
            float nearest = reach * reach;
            for (unsigned q = 0U; q < oc; ++q) {
                if ((taken >> q) & 1U) {
                    continue;
                }
                float da = 0.0F, db = 0.0F;
                {
                    const float x = o->points[q].anchor_a[0] - c.points[i].anchor_a[0];
                    const float y = o->points[q].anchor_a[1] - c.points[i].anchor_a[1];
                    const float z = o->points[q].anchor_a[2] - c.points[i].anchor_a[2];
                    da = x * x + y * y + z * z;
                }
                {
                    const float x = o->points[q].anchor_b[0] - c.points[i].anchor_b[0];
                    const float y = o->points[q].anchor_b[1] - c.points[i].anchor_b[1];
                    const float z = o->points[q].anchor_b[2] - c.points[i].anchor_b[2];
                    db = x * x + y * y + z * z;
                }
                const float d = da > db ? da : db;
                if (d < nearest) {
                    nearest = d;
                    pick = q;
                }
            }
            if (pick != NPH_GPU_NULL) {
                c.points[i].normal_impulse = o->points[pick].normal_impulse;
                memcpy(c.points[i].tangent_impulse, o->points[pick].tangent_impulse, sizeof(float) * 3U);
                taken |= 1U << pick;
            }
        }
        out[g] = c;
    }
    return NPH_GPU_OK;
}

static void write_back_f32(const Result_f32 *rp, float dt, NphGpuWorldView *v)
{
    Result_f32 r = *rp;
    // finalize_body (solver.c:304-349). Recomputed from the FP32 prepare: q0 is the record's.
    for (unsigned i = 0U; i < r.n; ++i) {
        NphGpuBody *b = &v->bodies[i];
        const Body_f32 *sb = &r.bodies[i];
        const Q4_f32 q0 = q4_load_f32(b->rotation);
        b->linear_velocity[0] = sb->v.x;
        b->linear_velocity[1] = sb->v.y;
        b->linear_velocity[2] = sb->v.z;
        b->angular_velocity[0] = sb->w.x;
        b->angular_velocity[1] = sb->w.y;
        b->angular_velocity[2] = sb->w.z;
        const Q4_f32 q = q_normalize_f32(q_mul_f32(sb->dq, q0));
        b->rotation[0] = q.x;
        b->rotation[1] = q.y;
        b->rotation[2] = q.z;
        b->rotation[3] = q.w;
        b->center[0] = b->center[0] + (double)sb->dp.x;
        b->center[1] = b->center[1] + (double)sb->dp.y;
        b->center[2] = b->center[2] + (double)sb->dp.z;
        const V3_f32 rc = rotate_f32(q, v3_load_f32(b->local_center));
        b->origin[0] = b->center[0] + (double)(-rc.x);
        b->origin[1] = b->center[1] + (double)(-rc.y);
        b->origin[2] = b->center[2] + (double)(-rc.z);
        memset(b->force, 0, sizeof b->force);
        memset(b->torque, 0, sizeof b->torque);
        const float speed = max_f32(length_f32(sb->v), b->max_extent * length_f32(sb->w));
        if ((b->flags & NPH_GPU_BODY_ENABLE_SLEEP) == 0U || speed > b->sleep_threshold) {
            b->sleep_time = 0.0F;
        } else {
            b->sleep_time += dt;
        }
    }
    // store_group (solver.c:475-499).
    for (unsigned i = 0U; i < v->contact_count; ++i) {
        NphGpuContact *c = &v->contacts[i];
        const Manifold_f32 *m = &r.m[i];
        c->flags = m->impacted ? (c->flags | NPH_GPU_CONTACT_HIT) : (c->flags & ~NPH_GPU_CONTACT_HIT);
        for (unsigned k = 0U; k < c->point_count; ++k) {
            const Point_f32 *p = &m->p[k];
            NphGpuContactPoint *cp = &c->points[k];
            cp->normal_impulse = p->normal_impulse;
            cp->max_normal_impulse = p->max_normal_impulse;
            cp->relative_velocity = p->relative_velocity;
            const V3_f32 t = add_f32(scale_f32(m->t1, p->tangent_impulse[0]),
                                     scale_f32(m->t2, p->tangent_impulse[1]));
            cp->tangent_impulse[0] = t.x;
            cp->tangent_impulse[1] = t.y;
            cp->tangent_impulse[2] = t.z;
        }
    }
    for (unsigned i = 0U; i < v->joint_count; ++i) {
        NphGpuJoint *jr = &v->joints[i];
        const Joint_f32 *j = &r.j[i];
        jr->linear_impulse[0] = j->linear_impulse.x;
        jr->linear_impulse[1] = j->linear_impulse.y;
        jr->linear_impulse[2] = j->linear_impulse.z;
        jr->angular_impulse[0] = j->angular_impulse.x;
        jr->angular_impulse[1] = j->angular_impulse.y;
        jr->angular_impulse[2] = j->angular_impulse.z;
        jr->friction_impulse[0] = j->friction_impulse.x;
        jr->friction_impulse[1] = j->friction_impulse.y;
        jr->friction_impulse[2] = j->friction_impulse.z;
        jr->lower_impulse = j->lower_impulse;
        jr->upper_impulse = j->upper_impulse;
        jr->swing_impulse = j->swing_impulse;
        jr->motor_impulse = j->motor_impulse;
        jr->spring_impulse = j->spring_impulse;
        for (unsigned a = 0U; a < NPH_GPU_D6_AXES; ++a) {
            for (unsigned k = 0U; k < 4U; ++k) {
                jr->axis_impulse[a][k] = j->axis_impulse[a][k];
            }
        }
        jr->flags = j->flags;
    }
    // post_finalize (solver.c:851-857): a driven joint keeps its bodies awake.
    for (unsigned i = 0U; i < v->joint_count; ++i) {
        const NphGpuJoint *jr = &v->joints[i];
        if (joint_is_driven(jr)) {
            if (jr->body_a < v->body_count) {
                v->bodies[jr->body_a].sleep_time = 0.0F;
            }
            if (jr->body_b < v->body_count) {
                v->bodies[jr->body_b].sleep_time = 0.0F;
            }
        }
    }
    free(r.bodies);
    free(r.m);
    free(r.j);
}

// What the FP64 step returns: the same results as the FP32 write-back, in double.
typedef struct NphPort64Out {
    double *linear_velocity;       // 3 per body
    double *angular_velocity;      // 3 per body
    double *rotation;              // 4 per body
    double *center;                // 3 per body
    double *normal_impulse;        // 4 per contact
    double *max_normal_impulse;    // 4 per contact
    double *tangent_impulse;       // 12 per contact (world)
    double *relative_velocity;     // 4 per contact
    double *joint_linear_impulse;  // 3 per joint
    double *joint_angular_impulse; // 3 per joint
} NphPort64Out;

// The FP64 re-run of the same step: the view is read only.
PORT_API int nph_port64_solve(const NphGpuWorldParams *wp, float dt, const NphGpuWorldView *v,
                              NphPort64Out *out)
{
    const int bad = check_view(wp, v);
    if (bad != NPH_GPU_OK) {
        return bad;
    }
    Result_f64 r;
    const int res = run_f64(wp, dt, v, &r);
    if (res != NPH_GPU_OK) {
        return res;
    }
    for (unsigned i = 0U; i < r.n; ++i) {
        const NphGpuBody *b = &v->bodies[i];
        const Body_f64 *sb = &r.bodies[i];
        const Q4_f64 q = q_normalize_f64(q_mul_f64(sb->dq, q4_load_f64(b->rotation)));
        const double vv[3] = {sb->v.x, sb->v.y, sb->v.z};
        const double ww[3] = {sb->w.x, sb->w.y, sb->w.z};
        const double qq[4] = {q.x, q.y, q.z, q.w};
        const double cc[3] = {b->center[0] + sb->dp.x, b->center[1] + sb->dp.y,
                              b->center[2] + sb->dp.z};
        memcpy(&out->linear_velocity[3 * i], vv, sizeof vv);
        memcpy(&out->angular_velocity[3 * i], ww, sizeof ww);
        memcpy(&out->rotation[4 * i], qq, sizeof qq);
        memcpy(&out->center[3 * i], cc, sizeof cc);
    }
    for (unsigned i = 0U; i < v->contact_count; ++i) {
        const Manifold_f64 *m = &r.m[i];
        for (unsigned k = 0U; k < 4U; ++k) {
            const Point_f64 *p = &m->p[k];
            const int has = k < m->point_count;
            out->normal_impulse[4 * i + k] = has ? p->normal_impulse : 0.0;
            out->max_normal_impulse[4 * i + k] = has ? p->max_normal_impulse : 0.0;
            out->relative_velocity[4 * i + k] = has ? p->relative_velocity : 0.0;
            const V3_f64 t = add_f64(scale_f64(m->t1, p->tangent_impulse[0]),
                                     scale_f64(m->t2, p->tangent_impulse[1]));
            out->tangent_impulse[12 * i + 3 * k + 0] = has ? t.x : 0.0;
            out->tangent_impulse[12 * i + 3 * k + 1] = has ? t.y : 0.0;
            out->tangent_impulse[12 * i + 3 * k + 2] = has ? t.z : 0.0;
        }
    }
    for (unsigned i = 0U; i < v->joint_count; ++i) {
        const Joint_f64 *j = &r.j[i];
        out->joint_linear_impulse[3 * i + 0] = j->linear_impulse.x;
        out->joint_linear_impulse[3 * i + 1] = j->linear_impulse.y;
        out->joint_linear_impulse[3 * i + 2] = j->linear_impulse.z;
        out->joint_angular_impulse[3 * i + 0] = j->angular_impulse.x;
        out->joint_angular_impulse[3 * i + 1] = j->angular_impulse.y;
        out->joint_angular_impulse[3 * i + 2] = j->angular_impulse.z;
    }
    free(r.bodies);
    free(r.m);
    free(r.j);
    return NPH_GPU_OK;
}

// Sequential first-fit colouring of constraints inserted in order into an empty graph
// (graph_pick_color, island.c:34-56; graph_set_bodies, island.c:58-75), with each
// constraint's slot in its colour's list: its contact list, or its joint list for a
// constraint whose bit 2 of `dynamic_bits` is set (island.c:77-88, 106-118).
PORT_API int nph_port_graph_color(const unsigned *body_a, const unsigned *body_b,
                                  const unsigned char *dynamic_bits, unsigned count,
                                  unsigned body_slots, unsigned *out_color, unsigned *out_slot)
{
    const size_t words = ((size_t)body_slots + 63U) / 64U;
    unsigned long long *bits =
        (unsigned long long *)calloc(words * NPH_GPU_COLORS + 1U, sizeof(unsigned long long));
    if (bits == NULL) {
        return NPH_GPU_OUT_OF_MEMORY;
    }
    unsigned lens[2][NPH_GPU_COLOR_SLOTS]; // the colours' contact lists and joint lists
    memset(lens, 0, sizeof lens);
#define TEST(c, b) ((bits[(size_t)(c) * words + (b) / 64U] >> ((b) % 64U)) & 1ULL)
#define SET(c, b) (bits[(size_t)(c) * words + (b) / 64U] |= 1ULL << ((b) % 64U))
    for (unsigned i = 0U; i < count; ++i) {
        const unsigned a = body_a[i];
        const unsigned b = body_b[i];
        const int da = (dynamic_bits[i] & 1U) != 0U;
        const int db = (dynamic_bits[i] & 2U) != 0U;
        unsigned color = NPH_GPU_OVERFLOW;
        if (da && db) {
            for (unsigned k = 0U; k < NPH_GPU_DYNAMIC_COLORS; ++k) {
                if (!TEST(k, a) && !TEST(k, b)) {
                    color = k;
                    break;
                }
            }
        } else {
            const unsigned body = da ? a : b;
            for (unsigned k = 1U; k < NPH_GPU_COLORS; ++k) {
                if (!TEST(k, body)) {
                    color = k;
                    break;
                }
            }
        }
        if (color != NPH_GPU_OVERFLOW) {
            if (da) {
                SET(color, a);
            }
            if (db) {
                SET(color, b);
            }
        }
        out_color[i] = color;
        out_slot[i] = lens[(dynamic_bits[i] & 4U) != 0U ? 1 : 0][color]++;
    }
#undef TEST
#undef SET
    free(bits);
    return NPH_GPU_OK;
}

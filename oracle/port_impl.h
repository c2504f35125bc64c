// SPDX-License-Identifier: Apache-2.0
//
// TEST INFRASTRUCTURE (the oracle), never the product. A CPU restatement of the reference's
// soft-step solver stage (phys_solve, engine/physics/src/solver.c:961-1105) over the
// NphGpuWorldView records of include/nepheline_b200.h, one constraint at a time in the
// reference's pass order. Every formula keeps the reference's operation order and rounding
// (no FMA contraction, IEEE division and square root), so the FP32 instance agrees with the
// reference bit for bit; the FP64 instance is the same step in double precision, the error
// baseline of every FP32 result.
//
// Included twice by port.c, with REAL float or double and SUF the name suffix.
//
// Where the reference runs eight contacts per call (solver_impl.h), this runs one; a
// manifold's row loops run over its own points. Two decisions of the reference depend on the
// eight-lane group a manifold falls in (its colour's list cut in eights, build_groups,
// solver.c:810-843): the impact sweeps and the restitution sweeps run when the group's largest
// point count is above one (solver_impl.h:533, 637), and the TGS-style warm-start share of a
// hit lane also visits the group's points the lane lacks, whose anchors are zero
// (solver_impl.h:210-235). Each manifold carries its group's point count for both. Rows past
// a lane's own points change no value otherwise (zero masses): at most the sign of a zero.

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SUF)
#define R(x) ((REAL)(x))

typedef struct FN(V3) {
    REAL x, y, z;
} FN(V3);
typedef struct FN(Q4) {
    REAL x, y, z, w;
} FN(Q4);
typedef struct FN(M3) {
    FN(V3) c[3]; // columns
} FN(M3);

#define V3 FN(V3)
#define Q4 FN(Q4)
#define M3 FN(M3)

static inline V3 FN(v3)(REAL x, REAL y, REAL z)
{
    V3 r = {x, y, z};
    return r;
}
static inline V3 FN(v3_load)(const float *p)
{
    return FN(v3)(R(p[0]), R(p[1]), R(p[2]));
}
static inline Q4 FN(q4_load)(const float *p)
{
    Q4 q = {R(p[0]), R(p[1]), R(p[2]), R(p[3])};
    return q;
}
static inline V3 FN(add)(V3 a, V3 b) { return FN(v3)(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 FN(sub)(V3 a, V3 b) { return FN(v3)(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 FN(scale)(V3 a, REAL s) { return FN(v3)(a.x * s, a.y * s, a.z * s); }
static inline V3 FN(neg)(V3 a) { return FN(v3)(-a.x, -a.y, -a.z); }
// vec.h:292-295: a + b s.
static inline V3 FN(mul_add)(V3 a, V3 b, REAL s)
{
    return FN(v3)(a.x + b.x * s, a.y + b.y * s, a.z + b.z * s);
}
// vec.h:300-303.
static inline REAL FN(dot)(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// vec.h:305-308.
static inline V3 FN(cross)(V3 a, V3 b)
{
    return FN(v3)(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline REAL FN(min)(REAL a, REAL b) { return a < b ? a : b; } // scalar.h:67, _mm_min_ps
static inline REAL FN(max)(REAL a, REAL b) { return a > b ? a : b; } // scalar.h:71, _mm_max_ps
static inline REAL FN(abs)(REAL a) { return ABS(a); }
static inline REAL FN(length)(V3 a) { return SQRT(FN(dot)(a, a)); }
// vec.h:326-331: v / sqrt(|v|^2), as two rounded operations (scalar.h:181-184).
static inline V3 FN(normalize)(V3 a) { return FN(scale)(a, R(1) / SQRT(FN(dot)(a, a))); }

static inline Q4 FN(q_identity)(void)
{
    Q4 q = {R(0), R(0), R(0), R(1)};
    return q;
}
// quat.h:70-76.
static inline Q4 FN(q_mul)(Q4 a, Q4 b)
{
    Q4 r = {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
            a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
    return r;
}
static inline Q4 FN(q_conj)(Q4 q)
{
    Q4 r = {-q.x, -q.y, -q.z, q.w};
    return r;
}
static inline Q4 FN(q_scale)(Q4 q, REAL s)
{
    Q4 r = {q.x * s, q.y * s, q.z * s, q.w * s};
    return r;
}
static inline REAL FN(q_dot)(Q4 a, Q4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
// quat.h:102-107.
static inline Q4 FN(q_normalize)(Q4 q) { return FN(q_scale)(q, R(1) / SQRT(FN(q_dot)(q, q))); }
// quat.h:109-113.
static inline Q4 FN(q_normalize_or_identity)(Q4 q)
{
    const REAL len_sq = FN(q_dot)(q, q);
    return len_sq > R(0) ? FN(q_scale)(q, R(1) / SQRT(len_sq)) : FN(q_identity)();
}
// quat.h:156-163: v + 2 w (u x v) + 2 u x (u x v).
static inline V3 FN(rotate)(Q4 q, V3 v)
{
    const V3 u = FN(v3)(q.x, q.y, q.z);
    const V3 t = FN(scale)(FN(cross)(u, v), R(2));
    return FN(add)(FN(add)(v, FN(scale)(t, q.w)), FN(cross)(u, t));
}
// quat.h:234-239.
static inline Q4 FN(q_integrate)(Q4 q, V3 omega, REAL dt)
{
    const Q4 w = {omega.x, omega.y, omega.z, R(0)};
    const Q4 dq = FN(q_scale)(FN(q_mul)(w, q), R(0.5F) * dt);
    Q4 s = {q.x + dq.x, q.y + dq.y, q.z + dq.z, q.w + dq.w};
    return FN(q_normalize_or_identity)(s);
}
// quat.h:171-185: the rotated basis vectors.
static inline V3 FN(axis_x)(Q4 q)
{
    return FN(v3)(R(1) - R(2) * (q.y * q.y + q.z * q.z), R(2) * (q.x * q.y + q.w * q.z),
                  R(2) * (q.x * q.z - q.w * q.y));
}
static inline V3 FN(axis_y)(Q4 q)
{
    return FN(v3)(R(2) * (q.x * q.y - q.w * q.z), R(1) - R(2) * (q.x * q.x + q.z * q.z),
                  R(2) * (q.y * q.z + q.w * q.x));
}
static inline V3 FN(axis_z)(Q4 q)
{
    return FN(v3)(R(2) * (q.x * q.z + q.w * q.y), R(2) * (q.y * q.z - q.w * q.x),
                  R(1) - R(2) * (q.x * q.x + q.y * q.y));
}
// mat.h:103-107.
static inline V3 FN(m_mul_v)(M3 m, V3 v)
{
    return FN(add)(FN(add)(FN(scale)(m.c[0], v.x), FN(scale)(m.c[1], v.y)), FN(scale)(m.c[2], v.z));
}
static inline M3 FN(m_mul)(M3 a, M3 b)
{
    M3 r = {{FN(m_mul_v)(a, b.c[0]), FN(m_mul_v)(a, b.c[1]), FN(m_mul_v)(a, b.c[2])}};
    return r;
}
static inline M3 FN(m_transpose)(M3 m)
{
    M3 r = {{FN(v3)(m.c[0].x, m.c[1].x, m.c[2].x), FN(v3)(m.c[0].y, m.c[1].y, m.c[2].y),
             FN(v3)(m.c[0].z, m.c[1].z, m.c[2].z)}};
    return r;
}
static inline M3 FN(m_zero)(void)
{
    M3 r = {{FN(v3)(R(0), R(0), R(0)), FN(v3)(R(0), R(0), R(0)), FN(v3)(R(0), R(0), R(0))}};
    return r;
}
static inline M3 FN(m_load)(const float *p)
{
    M3 r = {{FN(v3_load)(p), FN(v3_load)(p + 3), FN(v3_load)(p + 6)}};
    return r;
}
static inline REAL FN(comp)(V3 v, unsigned i) { return i == 0U ? v.x : (i == 1U ? v.y : v.z); }
static inline V3 FN(without)(V3 v, unsigned axis)
{
    if (axis == 0U) {
        v.x = R(0);
    } else if (axis == 1U) {
        v.y = R(0);
    } else {
        v.z = R(0);
    }
    return v;
}

// ---------------------------------------------------------------------------------------
// Step state
// ---------------------------------------------------------------------------------------

typedef struct FN(Soft) {
    REAL bias_rate, mass_scale, impulse_scale;
} FN(Soft);

// solver.c:48-65.
static FN(Soft) FN(make_soft)(REAL hertz, REAL zeta, REAL h)
{
    FN(Soft) s;
    if (hertz <= R(0)) {
        s.bias_rate = R(0);
        s.mass_scale = R(1);
        s.impulse_scale = R(0);
        return s;
    }
    const REAL omega = R(2.0F) * R(3.14159265F) * hertz;
    const REAL a1 = R(2) * zeta + h * omega;
    const REAL a2 = h * omega * a1;
    const REAL a3 = R(1) / (R(1) + a2);
    s.bias_rate = omega / a1;
    s.mass_scale = a2 * a3;
    s.impulse_scale = a3;
    return s;
}

typedef struct FN(Body) { // PhysSolverBody, world_internal.h:387-398
    V3 v, w, dp;
    Q4 dq;
} FN(Body);

typedef struct FN(Param) { // PhysSolverParams, world_internal.h:403-417
    V3 linear_accel;
    REAL linear_damping;
    V3 angular_accel;
    REAL angular_damping;
    M3 inv_inertia;
    M3 inertia_local;
    Q4 q0;
    REAL max_angular_speed_sq, max_linear_speed_sq;
    unsigned flags, locks;
    REAL inv_mass;
} FN(Param);

enum { FN(PARAM_DYNAMIC) = 1, FN(PARAM_GYROSCOPIC) = 2 };

typedef struct FN(Point) { // PhysPointLanes, world_internal.h:460-479, one lane
    V3 ra, rb;
    REAL adjusted_separation, normal_mass, normal_impulse, max_normal_impulse, relative_velocity;
    REAL tangent_mass[3];
    REAL tangent_impulse[2];
    V3 ang_a[3], ang_b[3]; // I^-1 (r x axis) for the normal, tangent 1, tangent 2
} FN(Point);

typedef struct FN(Manifold) { // PhysContactLanes, world_internal.h:430-458, one lane
    unsigned ia, ib, write_a, write_b, point_count, group_points, impact, impacted;
    REAL ma, mb, friction, restitution;
    V3 n, t1, t2;
    FN(Soft) soft;
    FN(Point) p[4];
} FN(Manifold);

typedef struct FN(Joint) { // the step data of PhysJoint, world_internal.h:317-329
    unsigned type, sa, sb, write_a, write_b;
    REAL ma, mb;
    M3 ia, ib;
    V3 anchor_a, anchor_b, delta_center;
    Q4 frame_q_a, frame_q_b;
    FN(Soft) spring_soft;
    V3 linear_impulse, angular_impulse, friction_impulse;
    REAL lower_impulse, upper_impulse, swing_impulse, motor_impulse, spring_impulse;
    REAL axis_impulse[NPH_GPU_D6_AXES][4]; // PHYS_ROW_* per axis (distance: axis 0)
    unsigned flags;                        // the record's flags with this step's blocks
    NphGpuD6Axis ax[NPH_GPU_D6_AXES];      // a slider's or 6-DOF joint's axes (d6_config)
    const NphGpuJoint *rec;
} FN(Joint);

typedef struct FN(Step) { // StepContext, solver.c:67-85
    REAL dt, h, inv_h, push_max, restitution_threshold;
    FN(Soft) contact_soft, static_soft, joint_soft;
    REAL slop;           // TGS's linear slop (solver.c:1016); 0 for the soft step
    unsigned scale_hits; // TGS: a hit scales the next warm start (solver.c:411-416)
    unsigned solver;     // the stage list (solver.c:1036-1060)
    unsigned dummy;
    FN(Body) *bodies;
    FN(Param) *params;
    FN(Manifold) *m;
    FN(Joint) *j;
    unsigned color_first[NPH_GPU_COLOR_SLOTS], joint_first[NPH_GPU_COLOR_SLOTS];
} FN(Step);

// ---------------------------------------------------------------------------------------
// Bodies
// ---------------------------------------------------------------------------------------

// solver.c:103-117.
static M3 FN(lock_inertia)(M3 m, unsigned locks)
{
    for (unsigned axis = 0U; axis < 3U; ++axis) {
        if ((locks & (NPH_GPU_LOCK_ANGULAR_X << axis)) == 0U) {
            continue;
        }
        m.c[axis] = FN(v3)(R(0), R(0), R(0));
        for (unsigned k = 0U; k < 3U; ++k) {
            m.c[k] = FN(without)(m.c[k], axis);
        }
    }
    return m;
}

// solver.c:123-129 (on the FP32 inertia as stored).
static int FN(isotropic)(const float *m)
{
    const float tol = 1e-6F * (fabsf(m[0]) + fabsf(m[4]) + fabsf(m[8]));
    return fabsf(m[4] - m[0]) <= tol && fabsf(m[8] - m[0]) <= tol && fabsf(m[1]) <= tol &&
           fabsf(m[2]) <= tol && fabsf(m[5]) <= tol;
}

// solver.c:131-168.
static void FN(prepare_body)(FN(Step) *s, const NphGpuWorldParams *wp, const NphGpuBody *b,
                             unsigned i)
{
    FN(Body) *sb = &s->bodies[i];
    FN(Param) *p = &s->params[i];
    memset(sb, 0, sizeof *sb);
    memset(p, 0, sizeof *p);
    sb->v = FN(v3_load)(b->linear_velocity);
    sb->w = FN(v3_load)(b->angular_velocity);
    sb->dq = FN(q_identity)();
    p->q0 = FN(q4_load)(b->rotation);
    p->locks = b->locks;
    const REAL max_rotation = R(0.25F * 3.14159265F) * s->inv_h;
    p->max_angular_speed_sq = max_rotation * max_rotation;
    p->max_linear_speed_sq = R(wp->max_linear_speed) * R(wp->max_linear_speed);
    if (b->type == NPH_GPU_BODY_DYNAMIC) {
        p->flags = FN(PARAM_DYNAMIC);
        if ((b->flags & NPH_GPU_BODY_GYROSCOPIC) != 0U && !FN(isotropic)(b->inertia)) {
            p->flags |= FN(PARAM_GYROSCOPIC);
        }
        const V3 g = FN(v3_load)(wp->gravity);
        p->linear_accel =
            FN(add)(FN(scale)(g, R(b->gravity_scale)), FN(scale)(FN(v3_load)(b->force), R(b->inv_mass)));
        const Q4 q = FN(q4_load)(b->rotation);
        M3 r;
        r.c[0] = FN(axis_x)(q);
        r.c[1] = FN(axis_y)(q);
        r.c[2] = FN(axis_z)(q);
        p->inv_inertia = FN(lock_inertia)(
            FN(m_mul)(FN(m_mul)(r, FN(m_load)(b->inv_inertia)), FN(m_transpose)(r)), b->locks);
        p->angular_accel = FN(m_mul_v)(p->inv_inertia, FN(v3_load)(b->torque));
        p->inertia_local = FN(m_load)(b->inertia);
        p->linear_damping = R(1) / (R(1) + s->h * R(b->linear_damping));
        p->angular_damping = R(1) / (R(1) + s->h * R(b->angular_damping));
        p->inv_mass = R(b->inv_mass);
    }
}

// solver.c:176-202.
static V3 FN(gyroscopic)(V3 w_world, Q4 q, M3 inertia, REAL h)
{
    const V3 w = FN(rotate)(FN(q_conj)(q), w_world);
    const V3 iw = FN(m_mul_v)(inertia, w);
    const V3 f = FN(scale)(FN(cross)(w, iw), h);
    const V3 e[3] = {FN(v3)(R(1), R(0), R(0)), FN(v3)(R(0), R(1), R(0)), FN(v3)(R(0), R(0), R(1))};
    V3 j[3];
    for (unsigned k = 0U; k < 3U; ++k) {
        j[k] = FN(mul_add)(inertia.c[k],
                           FN(sub)(FN(cross)(w, inertia.c[k]), FN(cross)(iw, e[k])), h);
    }
    const V3 c12 = FN(cross)(j[1], j[2]);
    const REAL det = FN(dot)(j[0], c12);
    if (!(det > R(0))) {
        return w_world;
    }
    const REAL inv_det = R(1) / det;
    const V3 x = FN(v3)(FN(dot)(f, c12) * inv_det, FN(dot)(j[0], FN(cross)(f, j[2])) * inv_det,
                        FN(dot)(j[0], FN(cross)(j[1], f)) * inv_det);
    return FN(rotate)(q, FN(sub)(w, x));
}

static V3 FN(lock_linear)(V3 v, unsigned locks)
{
    if ((locks & NPH_GPU_LOCK_LINEAR_X) != 0U) v.x = R(0);
    if ((locks & NPH_GPU_LOCK_LINEAR_Y) != 0U) v.y = R(0);
    if ((locks & NPH_GPU_LOCK_LINEAR_Z) != 0U) v.z = R(0);
    return v;
}
static V3 FN(lock_angular)(V3 w, unsigned locks)
{
    if ((locks & NPH_GPU_LOCK_ANGULAR_X) != 0U) w.x = R(0);
    if ((locks & NPH_GPU_LOCK_ANGULAR_Y) != 0U) w.y = R(0);
    if ((locks & NPH_GPU_LOCK_ANGULAR_Z) != 0U) w.z = R(0);
    return w;
}

// solver.c:232-259.
static void FN(integrate_velocity)(FN(Step) *s, unsigned i)
{
    const FN(Param) *p = &s->params[i];
    if ((p->flags & FN(PARAM_DYNAMIC)) == 0U) {
        return;
    }
    FN(Body) *sb = &s->bodies[i];
    const REAL h = s->h;
    V3 v = FN(scale)(FN(mul_add)(sb->v, p->linear_accel, h), p->linear_damping);
    V3 av = FN(scale)(FN(mul_add)(sb->w, p->angular_accel, h), p->angular_damping);
    if ((p->flags & FN(PARAM_GYROSCOPIC)) != 0U) {
        av = FN(gyroscopic)(av, FN(q_mul)(sb->dq, p->q0), p->inertia_local, h);
    }
    const REAL v_sq = FN(dot)(v, v);
    if (v_sq > p->max_linear_speed_sq) {
        v = FN(scale)(v, SQRT(p->max_linear_speed_sq / v_sq));
    }
    const REAL w_sq = FN(dot)(av, av);
    if (w_sq > p->max_angular_speed_sq) {
        av = FN(scale)(av, SQRT(p->max_angular_speed_sq / w_sq));
    }
    sb->v = FN(lock_linear)(v, p->locks);
    sb->w = FN(lock_angular)(av, p->locks);
}

// solver.c:261-270.
static void FN(integrate_position)(FN(Step) *s, unsigned i)
{
    const FN(Param) *p = &s->params[i];
    FN(Body) *sb = &s->bodies[i];
    sb->v = FN(lock_linear)(sb->v, p->locks);
    sb->w = FN(lock_angular)(sb->w, p->locks);
    sb->dp = FN(mul_add)(sb->dp, sb->v, s->h);
    sb->dq = FN(q_integrate)(sb->dq, sb->w, s->h);
}

// ---------------------------------------------------------------------------------------
// Contacts (solver.c:394-499; solver_impl.h:107-668)
// ---------------------------------------------------------------------------------------

// vec.h:460-469.
static V3 FN(perpendicular)(V3 n)
{
    const V3 a = FN(v3)(FN(abs)(n.x), FN(abs)(n.y), FN(abs)(n.z));
    const V3 axis = (a.x <= a.y && a.x <= a.z) ? FN(v3)(R(1), R(0), R(0))
                    : (a.y <= a.z)             ? FN(v3)(R(0), R(1), R(0))
                                               : FN(v3)(R(0), R(0), R(1));
    return FN(normalize)(FN(cross)(n, axis));
}

// solver_impl.h:121-142: vB + wB x rB - (vA + wA x rA).
static V3 FN(relative_velocity)(const FN(Body) *a, const FN(Body) *b, V3 ra, V3 rb)
{
    const V3 ca = FN(cross)(a->w, ra);
    const V3 cb = FN(cross)(b->w, rb);
    return FN(sub)(FN(add)(b->v, cb), FN(add)(a->v, ca));
}

// solver_impl.h:147-168.
static void FN(apply)(FN(Body) *a, FN(Body) *b, REAL ma, REAL mb, REAL lambda, V3 axis, V3 ang_a,
                      V3 ang_b)
{
    const REAL la = ma * lambda;
    const REAL lb = mb * lambda;
    a->v.x = a->v.x - la * axis.x;
    a->v.y = a->v.y - la * axis.y;
    a->v.z = a->v.z - la * axis.z;
    b->v.x = b->v.x + lb * axis.x;
    b->v.y = b->v.y + lb * axis.y;
    b->v.z = b->v.z + lb * axis.z;
    a->w.x = a->w.x - lambda * ang_a.x;
    a->w.y = a->w.y - lambda * ang_a.y;
    a->w.z = a->w.z - lambda * ang_a.z;
    b->w.x = b->w.x + lambda * ang_b.x;
    b->w.y = b->w.y + lambda * ang_b.y;
    b->w.z = b->w.z + lambda * ang_b.z;
}

// prepare_group (solver.c:394-473) and the prepare kernel (solver_impl.h:276-385), one lane.
static void FN(prepare_manifold)(FN(Step) *s, const NphGpuContact *c, unsigned body_count,
                                 const NphGpuBody *bodies, const NphGpuBody *fixed,
                                 FN(Manifold) *m, unsigned group_points)
{
    memset(m, 0, sizeof *m);
    const NphGpuBody *ba = c->body_a < body_count ? &bodies[c->body_a] : &fixed[c->body_a - body_count];
    const NphGpuBody *bb = c->body_b < body_count ? &bodies[c->body_b] : &fixed[c->body_b - body_count];
    const int dyn_a = ba->type == NPH_GPU_BODY_DYNAMIC;
    const int dyn_b = bb->type == NPH_GPU_BODY_DYNAMIC;
    m->ia = c->body_a < body_count ? c->body_a : s->dummy;
    m->ib = c->body_b < body_count ? c->body_b : s->dummy;
    m->write_a = (unsigned)dyn_a;
    m->write_b = (unsigned)dyn_b;
    m->ma = dyn_a ? R(ba->inv_mass) : R(0);
    m->mb = dyn_b ? R(bb->inv_mass) : R(0);
    const M3 ii_a = dyn_a ? s->params[m->ia].inv_inertia : FN(m_zero)();
    const M3 ii_b = dyn_b ? s->params[m->ib].inv_inertia : FN(m_zero)();
    m->n = FN(v3_load)(c->normal);
    m->t1 = FN(perpendicular)(m->n);
    m->t2 = FN(cross)(m->n, m->t1);
    m->friction = R(c->friction);
    m->restitution = R(c->restitution);
    m->soft = (!dyn_a || !dyn_b) ? s->static_soft : s->contact_soft;
    m->impacted = (c->flags & NPH_GPU_CONTACT_HIT) != 0U;
    m->point_count = c->point_count;
    m->group_points = group_points;
    const FN(Body) *a = &s->bodies[m->ia];
    const FN(Body) *b = &s->bodies[m->ib];
    const REAL mass = m->ma + m->mb;
    const V3 axes[3] = {m->n, m->t1, m->t2};
    m->impact = 0U;
    for (unsigned k = 0U; k < c->point_count; ++k) {
        FN(Point) *p = &m->p[k];
        const NphGpuContactPoint *cp = &c->points[k];
        p->ra = FN(v3_load)(cp->anchor_a);
        p->rb = FN(v3_load)(cp->anchor_b);
        p->normal_impulse = R(cp->normal_impulse);
        const REAL gap = FN(dot)(FN(sub)(p->rb, p->ra), m->n);
        p->adjusted_separation = R(cp->separation) - gap;
        V3 rxa[3];
        V3 rxb[3];
        for (unsigned x = 0U; x < 3U; ++x) {
            rxa[x] = FN(cross)(p->ra, axes[x]);
            rxb[x] = FN(cross)(p->rb, axes[x]);
            p->ang_a[x] = FN(m_mul_v)(ii_a, rxa[x]);
            p->ang_b[x] = FN(m_mul_v)(ii_b, rxb[x]);
        }
        const REAL kn = mass + FN(dot)(rxa[0], p->ang_a[0]) + FN(dot)(rxb[0], p->ang_b[0]);
        p->normal_mass = kn > R(0) ? R(1) / kn : R(0);
        const REAL k11 = mass + FN(dot)(rxa[1], p->ang_a[1]) + FN(dot)(rxb[1], p->ang_b[1]);
        const REAL k22 = mass + FN(dot)(rxa[2], p->ang_a[2]) + FN(dot)(rxb[2], p->ang_b[2]);
        const REAL k12 = FN(dot)(rxa[1], p->ang_a[2]) + FN(dot)(rxb[1], p->ang_b[2]);
        const REAL det = k11 * k22 - k12 * k12;
        const REAL inv = det > R(0) ? R(1) / det : R(0);
        p->tangent_mass[0] = k22 * inv;
        p->tangent_mass[1] = -k12 * inv;
        p->tangent_mass[2] = k11 * inv;
        const V3 dv = FN(relative_velocity)(a, b, p->ra, p->rb);
        p->relative_velocity = FN(dot)(dv, m->n);
        const V3 ti = FN(v3_load)(cp->tangent_impulse);
        p->tangent_impulse[0] = FN(dot)(ti, m->t1);
        p->tangent_impulse[1] = FN(dot)(ti, m->t2);
        p->max_normal_impulse = R(0);
        if (p->relative_velocity < -R(1.0F)) { // PHYS_IMPACT_SPEED, world_internal.h:382
            m->impact = 1U;
        }
    }
}

// solver_impl.h:181-258, one lane.
static void FN(warm_start)(FN(Step) *s, FN(Manifold) *m)
{
    FN(Body) a = s->bodies[m->ia];
    FN(Body) b = s->bodies[m->ib];
    if (m->impacted) {
        FN(Body) a1 = a;
        FN(Body) b1 = b;
        for (unsigned k = 0U; k < m->point_count; ++k) {
            const FN(Point) *p = &m->p[k];
            FN(apply)(&a1, &b1, m->ma, m->mb, p->normal_impulse, m->n, p->ang_a[0], p->ang_b[0]);
            FN(apply)(&a1, &b1, m->ma, m->mb, p->tangent_impulse[0], m->t1, p->ang_a[1], p->ang_b[1]);
            FN(apply)(&a1, &b1, m->ma, m->mb, p->tangent_impulse[1], m->t2, p->ang_a[2], p->ang_b[2]);
        }
        REAL share = R(1);
        for (unsigned k = 0U; k < m->group_points; ++k) {
            // Points of the group this lane lacks have zero anchors.
            const V3 zero = FN(v3)(R(0), R(0), R(0));
            const V3 ra = k < m->point_count ? m->p[k].ra : zero;
            const V3 rb = k < m->point_count ? m->p[k].rb : zero;
            const REAL before = FN(dot)(FN(relative_velocity)(&a, &b, ra, rb), m->n);
            const REAL after = FN(dot)(FN(relative_velocity)(&a1, &b1, ra, rb), m->n);
            const REAL allowed = FN(max)(before, R(0));
            const int pushed = after > allowed;
            const REAL part = (allowed - before) / (pushed ? after - before : R(1));
            share = FN(min)(share, pushed ? part : R(1));
        }
        for (unsigned k = 0U; k < m->point_count; ++k) {
            FN(Point) *p = &m->p[k];
            p->normal_impulse = p->normal_impulse * share;
            p->tangent_impulse[0] = p->tangent_impulse[0] * share;
            p->tangent_impulse[1] = p->tangent_impulse[1] * share;
        }
        m->impacted = 0U;
    }
    for (unsigned k = 0U; k < m->point_count; ++k) {
        const FN(Point) *p = &m->p[k];
        FN(apply)(&a, &b, m->ma, m->mb, p->normal_impulse, m->n, p->ang_a[0], p->ang_b[0]);
        FN(apply)(&a, &b, m->ma, m->mb, p->tangent_impulse[0], m->t1, p->ang_a[1], p->ang_b[1]);
        FN(apply)(&a, &b, m->ma, m->mb, p->tangent_impulse[1], m->t2, p->ang_a[2], p->ang_b[2]);
    }
    if (m->write_a) {
        s->bodies[m->ia].v = a.v;
        s->bodies[m->ia].w = a.w;
    }
    if (m->write_b) {
        s->bodies[m->ib].v = b.v;
        s->bodies[m->ib].w = b.w;
    }
}

// solver_impl.h:400-421.
static void FN(friction_circle)(REAL vt1, REAL vt2, REAL limit, REAL *new1, REAL *new2)
{
    const REAL len = SQRT(*new1 * *new1 + *new2 * *new2);
    const int over = len > limit;
    const REAL slip = SQRT(vt1 * vt1 + vt2 * vt2);
    const int sliding = over && slip > R(0);
    const REAL r = limit / (over ? len : R(1));
    const REAL stop_share = r / (over ? len : R(1));
    const REAL slip_share = (R(1) - r) / (sliding ? slip : R(1));
    const REAL d1 = stop_share * *new1 - slip_share * vt1;
    const REAL d2 = stop_share * *new2 - slip_share * vt2;
    const REAL dlen = SQRT(d1 * d1 + d2 * d2);
    const REAL to_edge = limit / (sliding ? dlen : R(1));
    if (sliding) {
        *new1 = d1 * to_edge;
        *new2 = d2 * to_edge;
    } else if (over) {
        *new1 = *new1 * r;
        *new2 = *new2 * r;
    }
}

// solver_impl.h:446-464.
static REAL FN(separation)(const FN(Body) *a, const FN(Body) *b, const FN(Point) *p, V3 n)
{
    const V3 pa = FN(rotate)(a->dq, p->ra);
    const V3 pb = FN(rotate)(b->dq, p->rb);
    const V3 d = FN(v3)((b->dp.x - a->dp.x) + (pb.x - pa.x), (b->dp.y - a->dp.y) + (pb.y - pa.y),
                        (b->dp.z - a->dp.z) + (pb.z - pa.z));
    return FN(dot)(d, n) + p->adjusted_separation;
}

// solver_impl.h:471-482 (the soft step's slop is zero).
static void FN(normal_row)(REAL sep, REAL inv_h, REAL slop, REAL soft_bias, REAL min_bias,
                           REAL soft_mass, REAL soft_impulse, REAL *bias, REAL *mass_scale,
                           REAL *impulse_scale)
{
    const int apart = sep > R(0);
    const REAL overlap = FN(min)(sep + slop, R(0));
    *bias = apart ? sep * inv_h : FN(max)(soft_bias * overlap, min_bias);
    *mass_scale = apart ? R(1) : soft_mass;
    *impulse_scale = apart ? R(0) : soft_impulse;
}

// solver_impl.h:484-602, one lane.
static void FN(solve)(FN(Step) *s, FN(Manifold) *m, int use_bias)
{
    FN(Body) a = s->bodies[m->ia];
    FN(Body) b = s->bodies[m->ib];
    const REAL min_bias = -s->push_max;
    const REAL soft_bias = use_bias ? m->soft.bias_rate : R(0);
    const REAL soft_mass = use_bias ? m->soft.mass_scale : R(1);
    const REAL soft_impulse = use_bias ? m->soft.impulse_scale : R(0);
    for (unsigned k = 0U; k < m->point_count; ++k) {
        FN(Point) *p = &m->p[k];
        REAL bias;
        REAL mass_scale;
        REAL impulse_scale;
        FN(normal_row)(FN(separation)(&a, &b, p, m->n), s->inv_h, s->slop, soft_bias, min_bias,
                       soft_mass, soft_impulse, &bias, &mass_scale, &impulse_scale);
        const REAL vn = FN(dot)(FN(relative_velocity)(&a, &b, p->ra, p->rb), m->n);
        const REAL row = p->normal_mass * mass_scale;
        const REAL acc = p->normal_impulse;
        const REAL impulse = -(row * (vn + bias)) - impulse_scale * acc;
        const REAL total = FN(max)(acc + impulse, R(0));
        const REAL delta = total - acc;
        p->normal_impulse = total;
        p->max_normal_impulse = FN(max)(p->max_normal_impulse, total);
        FN(apply)(&a, &b, m->ma, m->mb, delta, m->n, p->ang_a[0], p->ang_b[0]);
    }
    if (s->scale_hits != 0U && m->impact) {
        m->impacted = 1U; // solver_impl.h:528-532
    }
    if (m->group_points > 1U && m->impact) {
        REAL row_bias[4];
        REAL row_mass[4];
        REAL row_soft[4];
        for (unsigned k = 0U; k < m->point_count; ++k) {
            REAL mass_scale;
            FN(normal_row)(FN(separation)(&a, &b, &m->p[k], m->n), s->inv_h, s->slop, soft_bias,
                           min_bias, soft_mass, soft_impulse, &row_bias[k], &mass_scale,
                           &row_soft[k]);
            row_mass[k] = m->p[k].normal_mass * mass_scale;
        }
        for (unsigned sweep = 0U; sweep < 7U; ++sweep) { // PHYS_IMPACT_SWEEPS
            for (unsigned k = 0U; k < m->point_count; ++k) {
                FN(Point) *p = &m->p[k];
                const REAL vn = FN(dot)(FN(relative_velocity)(&a, &b, p->ra, p->rb), m->n);
                const REAL acc = p->normal_impulse;
                const REAL impulse = -(row_mass[k] * (vn + row_bias[k])) - row_soft[k] * acc;
                const REAL total = FN(max)(acc + impulse, R(0));
                const REAL delta = total - acc;
                p->normal_impulse = total;
                p->max_normal_impulse = FN(max)(p->max_normal_impulse, total);
                FN(apply)(&a, &b, m->ma, m->mb, delta, m->n, p->ang_a[0], p->ang_b[0]);
            }
        }
    }
    for (unsigned k = 0U; k < m->point_count; ++k) {
        FN(Point) *p = &m->p[k];
        const V3 dv = FN(relative_velocity)(&a, &b, p->ra, p->rb);
        const REAL vt1 = FN(dot)(dv, m->t1);
        const REAL vt2 = FN(dot)(dv, m->t2);
        const REAL old1 = p->tangent_impulse[0];
        const REAL old2 = p->tangent_impulse[1];
        REAL new1 = old1 - (p->tangent_mass[0] * vt1 + p->tangent_mass[1] * vt2);
        REAL new2 = old2 - (p->tangent_mass[1] * vt1 + p->tangent_mass[2] * vt2);
        FN(friction_circle)(vt1, vt2, m->friction * p->normal_impulse, &new1, &new2);
        p->tangent_impulse[0] = new1;
        p->tangent_impulse[1] = new2;
        FN(apply)(&a, &b, m->ma, m->mb, new1 - old1, m->t1, p->ang_a[1], p->ang_b[1]);
        FN(apply)(&a, &b, m->ma, m->mb, new2 - old2, m->t2, p->ang_a[2], p->ang_b[2]);
    }
    if (m->write_a) {
        s->bodies[m->ia].v = a.v;
        s->bodies[m->ia].w = a.w;
    }
    if (m->write_b) {
        s->bodies[m->ib].v = b.v;
        s->bodies[m->ib].w = b.w;
    }
}

// solver_impl.h:611-668, one lane.
static void FN(restitution)(FN(Step) *s, FN(Manifold) *m)
{
    int loaded[4] = {0, 0, 0, 0};
    int bounced = 0;
    for (unsigned k = 0U; k < m->point_count; ++k) {
        loaded[k] = m->p[k].relative_velocity < -s->restitution_threshold &&
                    m->p[k].max_normal_impulse > R(0);
        bounced |= loaded[k];
    }
    if (!bounced) {
        return;
    }
    if (s->scale_hits != 0U) {
        m->impacted = 1U; // solver_impl.h:662-665
    }
    FN(Body) a = s->bodies[m->ia];
    FN(Body) b = s->bodies[m->ib];
    const unsigned sweeps = m->group_points > 1U ? 8U : 1U;
    for (unsigned sweep = 0U; sweep < sweeps; ++sweep) {
        for (unsigned k = 0U; k < m->point_count; ++k) {
            if (!loaded[k]) {
                continue;
            }
            FN(Point) *p = &m->p[k];
            const REAL vn = FN(dot)(FN(relative_velocity)(&a, &b, p->ra, p->rb), m->n);
            const REAL acc = p->normal_impulse;
            const REAL impulse = -(p->normal_mass * (vn + m->restitution * p->relative_velocity));
            const REAL total = FN(max)(acc + impulse, R(0));
            const REAL delta = total - acc;
            p->normal_impulse = acc + delta;
            p->max_normal_impulse = FN(max)(p->max_normal_impulse, acc + delta);
            FN(apply)(&a, &b, m->ma, m->mb, delta, m->n, p->ang_a[0], p->ang_b[0]);
        }
    }
    if (m->write_a) {
        s->bodies[m->ia].v = a.v;
        s->bodies[m->ia].w = a.w;
    }
    if (m->write_b) {
        s->bodies[m->ib].v = b.v;
        s->bodies[m->ib].w = b.w;
    }
}

// ---------------------------------------------------------------------------------------
// Joints: ball and hinge (joint_solver.c)
// ---------------------------------------------------------------------------------------

typedef struct FN(JState) { // joint_solver.c:114-133
    FN(Body) *a, *b;
    V3 ra, rb;
    Q4 qa, qb;
} FN(JState);

static FN(JState) FN(joint_state)(FN(Step) *s, const FN(Joint) *j)
{
    FN(JState) st;
    st.a = &s->bodies[j->sa];
    st.b = &s->bodies[j->sb];
    st.ra = FN(rotate)(st.a->dq, j->anchor_a);
    st.rb = FN(rotate)(st.b->dq, j->anchor_b);
    st.qa = FN(q_mul)(st.a->dq, j->frame_q_a);
    st.qb = FN(q_mul)(st.b->dq, j->frame_q_b);
    return st;
}

// joint_solver.c:32-42.
static V3 FN(solve3)(const V3 k[3], V3 b)
{
    const V3 c12 = FN(cross)(k[1], k[2]);
    const REAL det = FN(dot)(k[0], c12);
    if (!(det > R(0))) {
        return FN(v3)(R(0), R(0), R(0));
    }
    const REAL inv = R(1) / det;
    return FN(v3)(FN(dot)(b, c12) * inv, FN(dot)(k[0], FN(cross)(b, k[2])) * inv,
                  FN(dot)(k[0], FN(cross)(k[1], b)) * inv);
}

// joint_solver.c:46-57.
static void FN(point_mass)(const FN(Joint) *j, V3 ra, V3 rb, V3 k[3])
{
    const V3 e[3] = {FN(v3)(R(1), R(0), R(0)), FN(v3)(R(0), R(1), R(0)), FN(v3)(R(0), R(0), R(1))};
    const REAL m = j->ma + j->mb;
    for (unsigned c = 0U; c < 3U; ++c) {
        const V3 ta = FN(m_mul_v)(j->ia, FN(cross)(ra, e[c]));
        const V3 tb = FN(m_mul_v)(j->ib, FN(cross)(rb, e[c]));
        k[c] = FN(sub)(FN(sub)(FN(scale)(e[c], m), FN(cross)(ra, ta)), FN(cross)(rb, tb));
    }
}

// joint_solver.c:60-65.
static void FN(angular_mass)(const FN(Joint) *j, V3 k[3])
{
    for (unsigned c = 0U; c < 3U; ++c) {
        k[c] = FN(add)(j->ia.c[c], j->ib.c[c]);
    }
}

// joint_solver.c:68-73.
static REAL FN(axial_mass)(const FN(Joint) *j, V3 axis)
{
    const REAL k = FN(dot)(axis, FN(m_mul_v)(j->ia, axis)) + FN(dot)(axis, FN(m_mul_v)(j->ib, axis));
    return k > R(0) ? R(1) / k : R(0);
}

// joint_solver.c:77-84.
static REAL FN(twist_angle)(Q4 qa, Q4 qb)
{
    Q4 r = FN(q_mul)(FN(q_conj)(qa), qb);
    if (r.w < R(0)) {
        r.x = -r.x;
        r.y = -r.y;
        r.z = -r.z;
        r.w = -r.w;
    }
    return R(2) * ATAN2(r.x, r.w);
}

// joint_solver.c:86-96.
static REAL FN(unwind)(REAL a)
{
    const REAL pi = R(3.14159265F);
    if (a > pi) {
        return a - R(2) * pi;
    }
    if (a < -pi) {
        return a + R(2) * pi;
    }
    return a;
}

// joint_solver.c:136-148.
static void FN(apply_linear)(const FN(Joint) *j, FN(JState) *st, V3 p)
{
    if (j->write_a) {
        st->a->v = FN(mul_add)(st->a->v, p, -j->ma);
        st->a->w = FN(sub)(st->a->w, FN(m_mul_v)(j->ia, FN(cross)(st->ra, p)));
    }
    if (j->write_b) {
        st->b->v = FN(mul_add)(st->b->v, p, j->mb);
        st->b->w = FN(add)(st->b->w, FN(m_mul_v)(j->ib, FN(cross)(st->rb, p)));
    }
}

// joint_solver.c:151-159.
static void FN(apply_angular)(const FN(Joint) *j, FN(JState) *st, V3 l)
{
    if (j->write_a) {
        st->a->w = FN(sub)(st->a->w, FN(m_mul_v)(j->ia, l));
    }
    if (j->write_b) {
        st->b->w = FN(add)(st->b->w, FN(m_mul_v)(j->ib, l));
    }
}

static V3 FN(relative_angular)(const FN(JState) *st) { return FN(sub)(st->b->w, st->a->w); }

// joint_solver.c:178-204.
static void FN(solve_angular_limit)(FN(Step) *s, FN(Joint) *j, FN(JState) *st, V3 axis, REAL c,
                                    REAL *accumulated, int use_bias)
{
    REAL bias = R(0);
    REAL mass_scale = R(1);
    REAL impulse_scale = R(0);
    if (c > R(0)) {
        bias = c * s->inv_h;
    } else if (use_bias) {
        bias = s->joint_soft.bias_rate * c;
        mass_scale = s->joint_soft.mass_scale;
        impulse_scale = s->joint_soft.impulse_scale;
    }
    const REAL cdot = -FN(dot)(FN(relative_angular)(st), axis);
    const REAL impulse =
        -FN(axial_mass)(j, axis) * mass_scale * (cdot + bias) - impulse_scale * *accumulated;
    const REAL total = FN(max)(*accumulated + impulse, R(0));
    const REAL delta = total - *accumulated;
    *accumulated = total;
    FN(apply_angular)(j, st, FN(scale)(axis, -delta));
}

// joint_solver.c:207-230.
static void FN(solve_point)(FN(Step) *s, FN(Joint) *j, FN(JState) *st, int use_bias)
{
    const V3 va = FN(add)(st->a->v, FN(cross)(st->a->w, st->ra));
    const V3 vb = FN(add)(st->b->v, FN(cross)(st->b->w, st->rb));
    const V3 cdot = FN(sub)(vb, va);
    V3 bias = FN(v3)(R(0), R(0), R(0));
    REAL mass_scale = R(1);
    REAL impulse_scale = R(0);
    if (use_bias) {
        const V3 c = FN(add)(FN(add)(FN(sub)(st->b->dp, st->a->dp), FN(sub)(st->rb, st->ra)),
                             j->delta_center);
        bias = FN(scale)(c, s->joint_soft.bias_rate);
        mass_scale = s->joint_soft.mass_scale;
        impulse_scale = s->joint_soft.impulse_scale;
    }
    V3 k[3];
    FN(point_mass)(j, st->ra, st->rb, k);
    const V3 x = FN(solve3)(k, FN(add)(cdot, bias));
    const V3 impulse = FN(sub)(FN(scale)(x, -mass_scale), FN(scale)(j->linear_impulse, impulse_scale));
    j->linear_impulse = FN(add)(j->linear_impulse, impulse);
    FN(apply_linear)(j, st, impulse);
}

// joint_solver.c:264-301.
static void FN(solve_axis_lock)(FN(Step) *s, FN(Joint) *j, FN(JState) *st, int use_bias)
{
    const V3 p1 = FN(axis_y)(st->qa);
    const V3 p2 = FN(axis_z)(st->qa);
    const V3 dw = FN(relative_angular)(st);
    REAL c1 = R(0);
    REAL c2 = R(0);
    REAL mass_scale = R(1);
    REAL impulse_scale = R(0);
    if (use_bias) {
        const V3 e = FN(cross)(FN(axis_x)(st->qa), FN(axis_x)(st->qb));
        c1 = s->joint_soft.bias_rate * FN(dot)(e, p1);
        c2 = s->joint_soft.bias_rate * FN(dot)(e, p2);
        mass_scale = s->joint_soft.mass_scale;
        impulse_scale = s->joint_soft.impulse_scale;
    }
    const V3 ip1 = FN(add)(FN(m_mul_v)(j->ia, p1), FN(m_mul_v)(j->ib, p1));
    const V3 ip2 = FN(add)(FN(m_mul_v)(j->ia, p2), FN(m_mul_v)(j->ib, p2));
    const REAL k11 = FN(dot)(p1, ip1);
    const REAL k12 = FN(dot)(p1, ip2);
    const REAL k22 = FN(dot)(p2, ip2);
    const REAL det = k11 * k22 - k12 * k12;
    if (!(det > R(0))) {
        return;
    }
    const REAL inv = R(1) / det;
    const REAL b1 = FN(dot)(dw, p1) + c1;
    const REAL b2 = FN(dot)(dw, p2) + c2;
    const REAL x1 = (k22 * b1 - k12 * b2) * inv;
    const REAL x2 = (k11 * b2 - k12 * b1) * inv;
    const REAL i1 = -mass_scale * x1 - impulse_scale * j->angular_impulse.x;
    const REAL i2 = -mass_scale * x2 - impulse_scale * j->angular_impulse.y;
    j->angular_impulse.x += i1;
    j->angular_impulse.y += i2;
    FN(apply_angular)(j, st, FN(add)(FN(scale)(p1, i1), FN(scale)(p2, i2)));
}

// joint_solver.c:303-336.
static void FN(solve_hinge)(FN(Step) *s, FN(Joint) *j, FN(JState) *st, int use_bias)
{
    const NphGpuHingeJoint *h = &j->rec->u.hinge;
    const V3 axis = FN(axis_x)(st->qa);
    const int need_angle = (h->enable_spring != 0U && use_bias) || h->enable_limit != 0U;
    const REAL angle = need_angle ? FN(twist_angle)(st->qa, st->qb) : R(0);
    const REAL mass = FN(axial_mass)(j, axis);
    if (h->enable_spring != 0U && use_bias) {
        const FN(Soft) *soft = &j->spring_soft;
        const REAL c = FN(unwind)(angle - R(h->spring_target));
        const REAL cdot = FN(dot)(FN(relative_angular)(st), axis);
        const REAL impulse = -soft->mass_scale * mass * (cdot + soft->bias_rate * c) -
                             soft->impulse_scale * j->spring_impulse;
        j->spring_impulse += impulse;
        FN(apply_angular)(j, st, FN(scale)(axis, impulse));
    }
    if (h->enable_motor != 0U) {
        const REAL cdot = FN(dot)(FN(relative_angular)(st), axis) - R(h->motor_speed);
        const REAL max_impulse = s->h * R(h->max_motor_torque);
        const REAL old = j->motor_impulse;
        const REAL v = old - mass * cdot;
        j->motor_impulse = v < -max_impulse ? -max_impulse : (v > max_impulse ? max_impulse : v);
        FN(apply_angular)(j, st, FN(scale)(axis, j->motor_impulse - old));
    }
    if (h->enable_limit != 0U) {
        FN(solve_angular_limit)(s, j, st, FN(neg)(axis), angle - R(h->lower), &j->lower_impulse,
                                use_bias);
        FN(solve_angular_limit)(s, j, st, axis, R(h->upper) - angle, &j->upper_impulse, use_bias);
    }
    FN(solve_axis_lock)(s, j, st, use_bias);
}

// joint_solver.c:341-358.
static void FN(solve_swing)(FN(Step) *s, FN(Joint) *j, FN(JState) *st, int use_bias)
{
    const NphGpuBallJoint *bj = &j->rec->u.ball;
    const V3 xa = FN(axis_x)(st->qa);
    const V3 xb = FN(axis_x)(st->qb);
    const V3 n = FN(cross)(xa, xb);
    const REAL sin_phi = FN(length)(n);
    if (!(sin_phi > R(1e-6F))) {
        return;
    }
    const V3 axis = FN(scale)(n, R(1) / sin_phi);
    const V3 local = FN(rotate)(FN(q_conj)(st->qa), axis);
    const REAL ey = local.y / R(bj->swing_y);
    const REAL ez = local.z / R(bj->swing_z);
    const REAL limit = R(1) / SQRT(ey * ey + ez * ez);
    const REAL phi = ATAN2(sin_phi, FN(dot)(xa, xb));
    FN(solve_angular_limit)(s, j, st, axis, limit - phi, &j->swing_impulse, use_bias);
}

// joint_solver.c:360-394.
static void FN(solve_ball)(FN(Step) *s, FN(Joint) *j, FN(JState) *st, int use_bias)
{
    const NphGpuBallJoint *bj = &j->rec->u.ball;
    if (R(bj->friction_torque) > R(0)) {
        V3 k[3];
        FN(angular_mass)(j, k);
        const V3 x = FN(solve3)(k, FN(relative_angular)(st));
        const V3 old = j->friction_impulse;
        V3 total = FN(sub)(old, x);
        const REAL max_impulse = s->h * R(bj->friction_torque);
        const REAL len_sq = FN(dot)(total, total);
        if (len_sq > max_impulse * max_impulse) {
            total = FN(scale)(total, max_impulse / SQRT(len_sq));
        }
        j->friction_impulse = total;
        FN(apply_angular)(j, st, FN(sub)(total, old));
    }
    if (bj->enable_swing_limit != 0U) {
        FN(solve_swing)(s, j, st, use_bias);
    }
    if (bj->enable_twist_limit != 0U) {
        const V3 sum = FN(add)(FN(axis_x)(st->qa), FN(axis_x)(st->qb));
        const REAL len = FN(length)(sum);
        if (len > R(1e-3F)) {
            const V3 axis = FN(scale)(sum, R(1) / len);
            const REAL twist = FN(twist_angle)(st->qa, st->qb);
            FN(solve_angular_limit)(s, j, st, FN(neg)(axis), twist - R(bj->twist_lower),
                                    &j->lower_impulse, use_bias);
            FN(solve_angular_limit)(s, j, st, axis, R(bj->twist_upper) - twist, &j->upper_impulse,
                                    use_bias);
        }
    }
}

// ---------------------------------------------------------------------------------------
// Joints: fixed, slider, 6-DOF and distance (joint_solver.c:232-262, 395-720)
// ---------------------------------------------------------------------------------------

// joint_solver.c:232-262.
static void FN(solve_rotation_lock)(FN(Step) *s, FN(Joint) *j, FN(JState) *st, int use_bias)
{
    const V3 cdot = FN(relative_angular)(st);
    V3 bias = FN(v3)(R(0), R(0), R(0));
    REAL mass_scale = R(1);
    REAL impulse_scale = R(0);
    if (use_bias) {
        Q4 e = FN(q_mul)(st->qb, FN(q_conj)(st->qa));
        if (e.w < R(0)) {
            e.x = -e.x;
            e.y = -e.y;
            e.z = -e.z;
            e.w = -e.w;
        }
        bias = FN(scale)(FN(v3)(e.x, e.y, e.z), R(2) * s->joint_soft.bias_rate);
        mass_scale = s->joint_soft.mass_scale;
        impulse_scale = s->joint_soft.impulse_scale;
    }
    V3 k[3];
    FN(angular_mass)(j, k);
    const V3 x = FN(solve3)(k, FN(add)(cdot, bias));
    const V3 impulse = FN(sub)(FN(scale)(x, -mass_scale), FN(scale)(j->angular_impulse, impulse_scale));
    j->angular_impulse = FN(add)(j->angular_impulse, impulse);
    FN(apply_angular)(j, st, impulse);
}

// joint_solver.c:480-509.
typedef struct FN(Row) {
    V3 u, ca, cb;
    REAL mass;
} FN(Row);

static FN(Row) FN(row_make)(const FN(Joint) *j, V3 u, V3 ca, V3 cb)
{
    FN(Row) r;
    r.u = u;
    r.ca = ca;
    r.cb = cb;
    const REAL k = (j->ma + j->mb) * FN(dot)(u, u) + FN(dot)(ca, FN(m_mul_v)(j->ia, ca)) +
                   FN(dot)(cb, FN(m_mul_v)(j->ib, cb));
    r.mass = k > R(0) ? R(1) / k : R(0);
    return r;
}

static FN(Row) FN(linear_row)(const FN(Joint) *j, const FN(JState) *st, V3 d, V3 u)
{
    return FN(row_make)(j, u, FN(cross)(FN(add)(st->ra, d), u), FN(cross)(st->rb, u));
}

static FN(Row) FN(angular_row)(const FN(Joint) *j, V3 axis)
{
    return FN(row_make)(j, FN(v3)(R(0), R(0), R(0)), axis, axis);
}

// joint_solver.c:511-530.
static REAL FN(row_speed)(const FN(JState) *st, const FN(Row) *r)
{
    return FN(dot)(FN(sub)(st->b->v, st->a->v), r->u) + FN(dot)(st->b->w, r->cb) -
           FN(dot)(st->a->w, r->ca);
}

static void FN(row_apply)(const FN(Joint) *j, FN(JState) *st, const FN(Row) *r, REAL lambda)
{
    if (j->write_a) {
        st->a->v = FN(mul_add)(st->a->v, r->u, -j->ma * lambda);
        st->a->w = FN(sub)(st->a->w, FN(m_mul_v)(j->ia, FN(scale)(r->ca, lambda)));
    }
    if (j->write_b) {
        st->b->v = FN(mul_add)(st->b->v, r->u, j->mb * lambda);
        st->b->w = FN(add)(st->b->w, FN(m_mul_v)(j->ib, FN(scale)(r->cb, lambda)));
    }
}

// joint_solver.c:531-549.
static void FN(row_lock)(FN(Step) *s, const FN(Joint) *j, FN(JState) *st, const FN(Row) *r, REAL c,
                         REAL *accumulated, int use_bias)
{
    REAL bias = R(0);
    REAL mass_scale = R(1);
    REAL impulse_scale = R(0);
    if (use_bias) {
        bias = s->joint_soft.bias_rate * c;
        mass_scale = s->joint_soft.mass_scale;
        impulse_scale = s->joint_soft.impulse_scale;
    }
    const REAL impulse =
        -r->mass * mass_scale * (FN(row_speed)(st, r) + bias) - impulse_scale * *accumulated;
    *accumulated += impulse;
    FN(row_apply)(j, st, r, impulse);
}

// joint_solver.c:550-562 with limit_soft (178-190).
static void FN(row_limit)(FN(Step) *s, const FN(Joint) *j, FN(JState) *st, const FN(Row) *r, REAL c,
                          REAL sign, REAL *accumulated, int use_bias)
{
    REAL bias = R(0);
    REAL mass_scale = R(1);
    REAL impulse_scale = R(0);
    if (c > R(0)) {
        bias = c * s->inv_h;
    } else if (use_bias) {
        bias = s->joint_soft.bias_rate * c;
        mass_scale = s->joint_soft.mass_scale;
        impulse_scale = s->joint_soft.impulse_scale;
    }
    const REAL impulse = -r->mass * mass_scale * (sign * FN(row_speed)(st, r) + bias) -
                         impulse_scale * *accumulated;
    const REAL total = FN(max)(*accumulated + impulse, R(0));
    const REAL delta = total - *accumulated;
    *accumulated = total;
    FN(row_apply)(j, st, r, sign * delta);
}

// joint_solver.c:564-571.
static void FN(row_motor)(const FN(Joint) *j, FN(JState) *st, const FN(Row) *r, REAL speed,
                          REAL max_impulse, REAL *accumulated)
{
    const REAL old = *accumulated;
    const REAL v = old - r->mass * (FN(row_speed)(st, r) - speed);
    *accumulated = v < -max_impulse ? -max_impulse : (v > max_impulse ? max_impulse : v);
    FN(row_apply)(j, st, r, *accumulated - old);
}

// joint_solver.c:573-585.
static void FN(row_spring)(FN(Step) *s, const FN(Joint) *j, FN(JState) *st, const FN(Row) *r, REAL c,
                           float hertz, float zeta, REAL *accumulated)
{
    const FN(Soft) soft = FN(make_soft)(R(hertz), R(zeta), s->h);
    const REAL impulse = -soft.mass_scale * r->mass * (FN(row_speed)(st, r) + soft.bias_rate * c) -
                         soft.impulse_scale * *accumulated;
    *accumulated += impulse;
    FN(row_apply)(j, st, r, impulse);
}

// vec.h:337-350.
static V3 FN(normalize_or)(V3 v, V3 fallback)
{
    const REAL len_sq = FN(dot)(v, v);
    if (len_sq > R(0) && len_sq <= R(3.40282347e38F)) {
        return FN(scale)(v, R(1) / SQRT(len_sq));
    }
    if (!(len_sq > R(3.40282347e38F)) || !isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) {
        return fallback;
    }
    const REAL m = FN(max)(ABS(v.x), FN(max)(ABS(v.y), ABS(v.z)));
    const V3 u = FN(scale)(v, R(1) / m);
    return FN(scale)(u, R(1) / SQRT(FN(dot)(u, u)));
}

// joint_solver.c:432-470.
typedef struct FN(AxesNow) {
    V3 d;
    V3 axis[NPH_GPU_D6_AXES];
    REAL value[NPH_GPU_D6_AXES];
} FN(AxesNow);

static FN(AxesNow) FN(axes_of)(Q4 qa, Q4 qb, V3 d)
{
    FN(AxesNow) n;
    n.d = d;
    n.axis[0] = FN(axis_x)(qa);
    n.axis[1] = FN(axis_y)(qa);
    n.axis[2] = FN(axis_z)(qa);
    for (unsigned i = 0U; i < 3U; ++i) {
        n.value[i] = FN(dot)(d, n.axis[i]);
    }
    Q4 r = FN(q_mul)(FN(q_conj)(qa), qb);
    if (r.w < R(0)) {
        r.x = -r.x;
        r.y = -r.y;
        r.z = -r.z;
        r.w = -r.w;
    }
    n.value[3] = R(2) * ATAN2(r.x, r.w);
    const REAL tl = SQRT(r.x * r.x + r.w * r.w);
    Q4 twist = FN(q_identity)();
    if (tl > R(1e-9F)) {
        twist.x = r.x / tl;
        twist.y = R(0);
        twist.z = R(0);
        twist.w = r.w / tl;
    }
    const Q4 swing = FN(q_mul)(r, FN(q_conj)(twist));
    n.value[4] = R(2) * ATAN2(swing.y, swing.w);
    n.value[5] = R(2) * ATAN2(swing.z, swing.w);
    n.axis[3] = FN(normalize_or)(FN(add)(n.axis[0], FN(axis_x)(qb)), n.axis[0]);
    n.axis[4] = n.axis[1];
    n.axis[5] = n.axis[2];
    return n;
}

// joint_solver.c:471-476.
static V3 FN(anchor_offset)(const FN(Joint) *j, const FN(JState) *st)
{
    return FN(add)(FN(add)(FN(sub)(st->b->dp, st->a->dp), FN(sub)(st->rb, st->ra)), j->delta_center);
}

static FN(Row) FN(axis_row)(const FN(Joint) *j, const FN(JState) *st, const FN(AxesNow) *n, unsigned i)
{
    return i < 3U ? FN(linear_row)(j, st, n->d, n->axis[i]) : FN(angular_row)(j, n->axis[i]);
}

// joint_solver.c:597-652.
static void FN(solve_axes)(FN(Step) *s, FN(Joint) *j, FN(JState) *st, int use_bias)
{
    const NphGpuD6Axis *ax = j->ax;
    const FN(AxesNow) n = FN(axes_of)(st->qa, st->qb, FN(anchor_offset)(j, st));
    for (unsigned i = 0U; i < NPH_GPU_D6_AXES; ++i) {
        const NphGpuD6Axis *a = &ax[i];
        if (a->motion == NPH_GPU_AXIS_LOCKED) {
            continue;
        }
        REAL *imp = j->axis_impulse[i];
        const FN(Row) r = FN(axis_row)(j, st, &n, i);
        if (a->enable_spring != 0U && use_bias) {
            const REAL e = n.value[i] - R(a->spring_target);
            FN(row_spring)(s, j, st, &r, i >= 3U ? FN(unwind)(e) : e, a->spring_hertz,
                           a->spring_damping_ratio, &imp[NPH_GPU_ROW_SPRING]);
        }
        if (a->enable_motor != 0U) {
            FN(row_motor)(j, st, &r, R(a->motor_speed), s->h * R(a->max_motor_force),
                          &imp[NPH_GPU_ROW_MOTOR]);
        }
        if (a->motion == NPH_GPU_AXIS_LIMITED) {
            FN(row_limit)(s, j, st, &r, n.value[i] - R(a->lower), R(1), &imp[NPH_GPU_ROW_LOCK], use_bias);
            FN(row_limit)(s, j, st, &r, R(a->upper) - n.value[i], R(-1), &imp[NPH_GPU_ROW_UPPER],
                          use_bias);
        }
    }
    if (port_all_locked(ax, 3U, 3U)) {
        FN(solve_rotation_lock)(s, j, st, use_bias);
    } else {
        const int swings = port_all_locked(ax, 4U, 2U);
        if (swings) {
            FN(solve_axis_lock)(s, j, st, use_bias);
        }
        for (unsigned i = 3U; i < NPH_GPU_D6_AXES; ++i) {
            if (ax[i].motion == NPH_GPU_AXIS_LOCKED && (i == 3U || !swings)) {
                const FN(Row) r = FN(angular_row)(j, n.axis[i]);
                FN(row_lock)(s, j, st, &r, n.value[i], &j->axis_impulse[i][NPH_GPU_ROW_LOCK], use_bias);
            }
        }
    }
    if (port_all_locked(ax, 0U, 3U)) {
        FN(solve_point)(s, j, st, use_bias);
    } else {
        for (unsigned i = 0U; i < 3U; ++i) {
            if (ax[i].motion == NPH_GPU_AXIS_LOCKED) {
                const FN(Row) r = FN(linear_row)(j, st, n.d, n.axis[i]);
                FN(row_lock)(s, j, st, &r, n.value[i], &j->axis_impulse[i][NPH_GPU_ROW_LOCK], use_bias);
            }
        }
    }
}

// joint_solver.c:654-682.
static void FN(warm_axes)(FN(Joint) *j, FN(JState) *st)
{
    const NphGpuD6Axis *ax = j->ax;
    const FN(AxesNow) n = FN(axes_of)(st->qa, st->qb, FN(anchor_offset)(j, st));
    const int rotation_block = port_all_locked(ax, 3U, 3U);
    const int swing_block = !rotation_block && port_all_locked(ax, 4U, 2U);
    const int point_block = port_all_locked(ax, 0U, 3U);
    for (unsigned i = 0U; i < NPH_GPU_D6_AXES; ++i) {
        const REAL *imp = j->axis_impulse[i];
        const REAL total = imp[NPH_GPU_ROW_LOCK] - imp[NPH_GPU_ROW_UPPER] + imp[NPH_GPU_ROW_MOTOR] +
                           imp[NPH_GPU_ROW_SPRING];
        if (total != R(0)) {
            const FN(Row) r = FN(axis_row)(j, st, &n, i);
            FN(row_apply)(j, st, &r, total);
        }
    }
    if (rotation_block) {
        FN(apply_angular)(j, st, j->angular_impulse);
    } else if (swing_block) {
        FN(apply_angular)(j, st, FN(add)(FN(scale)(FN(axis_y)(st->qa), j->angular_impulse.x),
                                         FN(scale)(FN(axis_z)(st->qa), j->angular_impulse.y)));
    }
    if (point_block) {
        FN(apply_linear)(j, st, j->linear_impulse);
    }
}

// joint_solver.c:683-707.
static void FN(solve_distance)(FN(Step) *s, FN(Joint) *j, FN(JState) *st, int use_bias)
{
    const NphGpuDistanceJoint *dj = &j->rec->u.distance;
    const V3 d = FN(anchor_offset)(j, st);
    const REAL len = FN(length)(d);
    if (!(len > R(1e-6F))) {
        return;
    }
    const FN(Row) r = FN(linear_row)(j, st, d, FN(scale)(d, R(1) / len));
    REAL *imp = j->axis_impulse[0];
    if (dj->enable_spring != 0U && use_bias) {
        FN(row_spring)(s, j, st, &r, len - R(dj->length), dj->spring_hertz, dj->spring_damping_ratio,
                       &imp[NPH_GPU_ROW_SPRING]);
    }
    if (dj->enable_motor != 0U) {
        FN(row_motor)(j, st, &r, R(dj->motor_speed), s->h * R(dj->max_motor_force),
                      &imp[NPH_GPU_ROW_MOTOR]);
    }
    if (dj->enable_limit != 0U) {
        FN(row_limit)(s, j, st, &r, len - R(dj->min_length), R(1), &imp[NPH_GPU_ROW_LOCK], use_bias);
        FN(row_limit)(s, j, st, &r, R(dj->max_length) - len, R(-1), &imp[NPH_GPU_ROW_UPPER], use_bias);
    } else if (dj->enable_spring == 0U) {
        FN(row_lock)(s, j, st, &r, len - R(dj->length), &imp[NPH_GPU_ROW_LOCK], use_bias);
    }
}

// joint_solver.c:709-720.
static void FN(warm_distance)(FN(Joint) *j, FN(JState) *st)
{
    const V3 d = FN(anchor_offset)(j, st);
    const REAL len = FN(length)(d);
    const REAL *imp = j->axis_impulse[0];
    const REAL total = imp[NPH_GPU_ROW_LOCK] - imp[NPH_GPU_ROW_UPPER] + imp[NPH_GPU_ROW_MOTOR] +
                       imp[NPH_GPU_ROW_SPRING];
    if (len > R(1e-6F) && total != R(0)) {
        const FN(Row) r = FN(linear_row)(j, st, d, FN(scale)(d, R(1) / len));
        FN(row_apply)(j, st, &r, total);
    }
}

// joint_solver.c:726-824, every type.
static void FN(prepare_joint)(FN(Step) *s, const NphGpuJoint *jr, unsigned body_count,
                              const NphGpuBody *bodies, const NphGpuBody *fixed, FN(Joint) *j)
{
    memset(j, 0, sizeof *j);
    j->rec = jr;
    j->type = jr->type;
    const NphGpuBody *a = jr->body_a < body_count ? &bodies[jr->body_a] : &fixed[jr->body_a - body_count];
    const NphGpuBody *b = jr->body_b < body_count ? &bodies[jr->body_b] : &fixed[jr->body_b - body_count];
    const int dyn_a = a->type == NPH_GPU_BODY_DYNAMIC;
    const int dyn_b = b->type == NPH_GPU_BODY_DYNAMIC;
    j->sa = jr->body_a < body_count ? jr->body_a : s->dummy;
    j->sb = jr->body_b < body_count ? jr->body_b : s->dummy;
    j->write_a = (unsigned)dyn_a;
    j->write_b = (unsigned)dyn_b;
    j->ma = dyn_a ? R(a->inv_mass) : R(0);
    j->mb = dyn_b ? R(b->inv_mass) : R(0);
    j->ia = dyn_a ? s->params[j->sa].inv_inertia : FN(m_zero)();
    j->ib = dyn_b ? s->params[j->sb].inv_inertia : FN(m_zero)();
    const Q4 qa = FN(q4_load)(a->rotation);
    const Q4 qb = FN(q4_load)(b->rotation);
    j->anchor_a = FN(rotate)(qa, FN(sub)(FN(v3_load)(jr->frame_a_position), FN(v3_load)(a->local_center)));
    j->anchor_b = FN(rotate)(qb, FN(sub)(FN(v3_load)(jr->frame_b_position), FN(v3_load)(b->local_center)));
    // nph_dvec3_relative (vec.h:991-994): the 64-bit difference, rounded to 32 bits.
    j->delta_center = FN(v3)(R(b->center[0] - a->center[0]), R(b->center[1] - a->center[1]),
                             R(b->center[2] - a->center[2]));
    j->frame_q_a = FN(q_mul)(qa, FN(q4_load)(jr->frame_a_rotation));
    j->frame_q_b = FN(q_mul)(qb, FN(q4_load)(jr->frame_b_rotation));
    j->linear_impulse = FN(v3_load)(jr->linear_impulse);
    j->angular_impulse = FN(v3_load)(jr->angular_impulse);
    j->friction_impulse = FN(v3_load)(jr->friction_impulse);
    j->lower_impulse = R(jr->lower_impulse);
    j->upper_impulse = R(jr->upper_impulse);
    j->swing_impulse = R(jr->swing_impulse);
    j->motor_impulse = R(jr->motor_impulse);
    j->spring_impulse = R(jr->spring_impulse);
    for (unsigned a = 0U; a < NPH_GPU_D6_AXES; ++a) {
        for (unsigned k = 0U; k < 4U; ++k) {
            j->axis_impulse[a][k] = R(jr->axis_impulse[a][k]);
        }
    }
    j->flags = jr->flags;
    if (jr->type == NPH_GPU_JOINT_HINGE) {
        const NphGpuHingeJoint *h = &jr->u.hinge;
        if (h->enable_limit == 0U) {
            j->lower_impulse = R(0);
            j->upper_impulse = R(0);
        }
        if (h->enable_motor == 0U) {
            j->motor_impulse = R(0);
        }
        if (h->enable_spring == 0U) {
            j->spring_impulse = R(0);
        }
        j->spring_soft = FN(make_soft)(h->enable_spring != 0U ? R(h->spring_hertz) : R(0),
                                       R(h->spring_damping_ratio), s->h);
    } else if (jr->type == NPH_GPU_JOINT_DISTANCE) {
        const NphGpuDistanceJoint *dj = &jr->u.distance;
        REAL *imp = j->axis_impulse[0];
        if (dj->enable_limit == 0U) {
            imp[NPH_GPU_ROW_UPPER] = R(0);
            if (dj->enable_spring != 0U) {
                imp[NPH_GPU_ROW_LOCK] = R(0);
            }
        }
        if (dj->enable_motor == 0U) {
            imp[NPH_GPU_ROW_MOTOR] = R(0);
        }
        if (dj->enable_spring == 0U) {
            imp[NPH_GPU_ROW_SPRING] = R(0);
        }
    } else if (jr->type == NPH_GPU_JOINT_SLIDER || jr->type == NPH_GPU_JOINT_D6) {
        port_axes(jr, j->ax);
        for (unsigned a = 0U; a < NPH_GPU_D6_AXES; ++a) {
            REAL *imp = j->axis_impulse[a];
            const unsigned motion = j->ax[a].motion;
            if (motion != NPH_GPU_AXIS_LIMITED) {
                imp[NPH_GPU_ROW_UPPER] = R(0);
            }
            if (motion == NPH_GPU_AXIS_FREE) {
                imp[NPH_GPU_ROW_LOCK] = R(0);
            }
            if (motion == NPH_GPU_AXIS_LOCKED || j->ax[a].enable_motor == 0U) {
                imp[NPH_GPU_ROW_MOTOR] = R(0);
            }
            if (motion == NPH_GPU_AXIS_LOCKED || j->ax[a].enable_spring == 0U) {
                imp[NPH_GPU_ROW_SPRING] = R(0);
            }
        }
        const int rotation = port_all_locked(j->ax, 3U, 3U);
        const int swing = !rotation && port_all_locked(j->ax, 4U, 2U);
        const int point = port_all_locked(j->ax, 0U, 3U);
        const unsigned blocks = (rotation ? NPH_GPU_JOINT_BLOCK_ROTATION : 0U) |
                                (swing ? NPH_GPU_JOINT_BLOCK_SWING : 0U) |
                                (point ? NPH_GPU_JOINT_BLOCK_POINT : 0U);
        const unsigned angular = NPH_GPU_JOINT_BLOCK_ROTATION | NPH_GPU_JOINT_BLOCK_SWING;
        const unsigned all = angular | NPH_GPU_JOINT_BLOCK_POINT;
        if ((j->flags & angular) != (blocks & angular)) {
            j->angular_impulse = FN(v3)(R(0), R(0), R(0));
        }
        if ((j->flags & NPH_GPU_JOINT_BLOCK_POINT) != (blocks & NPH_GPU_JOINT_BLOCK_POINT)) {
            j->linear_impulse = FN(v3)(R(0), R(0), R(0));
        }
        j->flags = (j->flags & ~all) | blocks;
    } else if (jr->type == NPH_GPU_JOINT_BALL) {
        const NphGpuBallJoint *bj = &jr->u.ball;
        if (bj->enable_swing_limit == 0U) {
            j->swing_impulse = R(0);
        }
        if (bj->enable_twist_limit == 0U) {
            j->lower_impulse = R(0);
            j->upper_impulse = R(0);
        }
        if (!(bj->friction_torque > 0.0F)) {
            j->friction_impulse = FN(v3)(R(0), R(0), R(0));
        }
    }
}

// joint_solver.c:855-868.
static void FN(joint_warm_start)(FN(Step) *s, FN(Joint) *j)
{
    FN(JState) st = FN(joint_state)(s, j);
    if (j->type == NPH_GPU_JOINT_SLIDER || j->type == NPH_GPU_JOINT_D6) {
        FN(warm_axes)(j, &st);
        return;
    }
    if (j->type == NPH_GPU_JOINT_DISTANCE) {
        FN(warm_distance)(j, &st);
        return;
    }
    // phys_joint_angular_impulse (joint_solver.c:826-853): the fixed joint's world vector.
    V3 angular = j->angular_impulse;
    if (j->type == NPH_GPU_JOINT_HINGE) {
        angular = FN(add)(FN(scale)(FN(axis_y)(st.qa), j->angular_impulse.x),
                          FN(scale)(FN(axis_z)(st.qa), j->angular_impulse.y));
        const REAL axial = j->lower_impulse - j->upper_impulse + j->motor_impulse + j->spring_impulse;
        angular = FN(mul_add)(angular, FN(axis_x)(st.qa), axial);
    } else if (j->type == NPH_GPU_JOINT_BALL) {
        angular = j->friction_impulse;
        const V3 xa = FN(axis_x)(st.qa);
        const V3 xb = FN(axis_x)(st.qb);
        const V3 n = FN(cross)(xa, xb);
        const REAL sin_phi = FN(length)(n);
        if (j->swing_impulse != R(0) && sin_phi > R(1e-6F)) {
            angular = FN(mul_add)(angular, n, -j->swing_impulse / sin_phi);
        }
        const V3 sum = FN(add)(xa, xb);
        const REAL len = FN(length)(sum);
        if (len > R(1e-3F)) {
            angular = FN(mul_add)(angular, sum, (j->lower_impulse - j->upper_impulse) / len);
        }
    }
    FN(apply_angular)(j, &st, angular);
    FN(apply_linear)(j, &st, j->linear_impulse);
}

// joint_solver.c:870-897.
static void FN(joint_solve)(FN(Step) *s, FN(Joint) *j, int use_bias)
{
    FN(JState) st = FN(joint_state)(s, j);
    switch (j->type) {
    case NPH_GPU_JOINT_BALL:
        FN(solve_ball)(s, j, &st, use_bias);
        break;
    case NPH_GPU_JOINT_HINGE:
        FN(solve_hinge)(s, j, &st, use_bias);
        break;
    case NPH_GPU_JOINT_FIXED:
        FN(solve_rotation_lock)(s, j, &st, use_bias);
        break;
    case NPH_GPU_JOINT_SLIDER:
    case NPH_GPU_JOINT_D6:
        FN(solve_axes)(s, j, &st, use_bias);
        return;
    default: // NPH_GPU_JOINT_DISTANCE
        FN(solve_distance)(s, j, &st, use_bias);
        return;
    }
    FN(solve_point)(s, j, &st, use_bias);
}

// ---------------------------------------------------------------------------------------
// The stage list (solver.c:961-1105)
// ---------------------------------------------------------------------------------------

enum { FN(PASS_WARM) = 0, FN(PASS_SOLVE), FN(PASS_RELAX), FN(PASS_RESTITUTION) };

// push_contact_pass (solver.c:774-789): the overflow's joints, its contacts, then every
// colour's joints and contacts in order.
static void FN(contact_pass)(FN(Step) *s, const NphGpuWorldView *v, int pass)
{
    for (unsigned slot = 0U; slot < NPH_GPU_COLOR_SLOTS; ++slot) {
        const unsigned c = slot == 0U ? NPH_GPU_OVERFLOW : slot - 1U;
        if (pass != FN(PASS_RESTITUTION)) {
            for (unsigned i = 0U; i < v->joint_color_counts[c]; ++i) {
                FN(Joint) *j = &s->j[s->joint_first[c] + i];
                if (pass == FN(PASS_WARM)) {
                    FN(joint_warm_start)(s, j);
                } else {
                    FN(joint_solve)(s, j, pass == FN(PASS_SOLVE));
                }
            }
        }
        for (unsigned i = 0U; i < v->contact_color_counts[c]; ++i) {
            FN(Manifold) *m = &s->m[s->color_first[c] + i];
            if (pass == FN(PASS_WARM)) {
                FN(warm_start)(s, m);
            } else if (pass == FN(PASS_RESTITUTION)) {
                FN(restitution)(s, m);
            } else {
                FN(solve)(s, m, pass == FN(PASS_SOLVE));
            }
        }
    }
}

typedef struct FN(Result) {
    FN(Body) *bodies;
    FN(Manifold) *m;
    FN(Joint) *j;
    unsigned n;
} FN(Result);

// The step's constants and the prepare stage (solver.c:985-1041): allocates the working state.
static int FN(setup)(FN(Step) *sp, const NphGpuWorldParams *wp, float dt, const NphGpuWorldView *v)
{
    const unsigned n = v->body_count;
    FN(Step) s;
    memset(&s, 0, sizeof s);
    s.dt = R(dt);
    s.h = R(dt) / R(wp->substeps); // solver.c:986
    s.inv_h = R(1) / s.h;
    s.push_max = R(wp->contact_push_max_velocity);
    s.restitution_threshold = R(wp->restitution_threshold);
    s.dummy = n;
    const REAL contact_hertz = wp->contact_hertz > 0.0F ? R(wp->contact_hertz) : R(0.125F) * s.inv_h;
    const REAL joint_hertz = wp->joint_hertz > 0.0F ? R(wp->joint_hertz) : R(0.25F) * s.inv_h;
    const REAL hertz = FN(min)(contact_hertz, R(0.25F) * s.inv_h);
    s.contact_soft = FN(make_soft)(hertz, R(wp->contact_damping_ratio), s.h);
    s.static_soft = FN(make_soft)(R(2.0F) * hertz, R(wp->contact_damping_ratio), s.h);
    s.joint_soft = FN(make_soft)(FN(min)(joint_hertz, R(0.25F) * s.inv_h), R(wp->joint_damping_ratio), s.h);
    s.solver = wp->solver;
    if (wp->solver == NPH_GPU_SOLVER_TGS) { // solver.c:1007-1017
        const FN(Soft) hard = {R(0.2F) * s.inv_h, R(1), R(0)};
        s.contact_soft = hard;
        s.static_soft = hard;
        s.joint_soft = hard;
        s.slop = R(0.005F); // NPH_PHYSICS_LINEAR_SLOP
        s.scale_hits = 1U;
    }
    s.bodies = (FN(Body) *)calloc((size_t)n + 1U, sizeof(FN(Body)));
    s.params = (FN(Param) *)calloc((size_t)n + 1U, sizeof(FN(Param)));
    s.m = (FN(Manifold) *)calloc((size_t)v->contact_count + 1U, sizeof(FN(Manifold)));
    s.j = (FN(Joint) *)calloc((size_t)v->joint_count + 1U, sizeof(FN(Joint)));
    if (s.bodies == NULL || s.params == NULL || s.m == NULL || s.j == NULL) {
        free(s.bodies);
        free(s.params);
        free(s.m);
        free(s.j);
        return NPH_GPU_OUT_OF_MEMORY;
    }
    s.bodies[n].dq = FN(q_identity)(); // the dummy: at rest, never written
    // Offsets of the colours in the view's arrays (colours 0..23, then the overflow).
    unsigned first = 0U;
    unsigned jfirst = 0U;
    for (unsigned c = 0U; c < NPH_GPU_COLOR_SLOTS; ++c) {
        s.color_first[c] = first;
        first += v->contact_color_counts[c];
        s.joint_first[c] = jfirst;
        jfirst += v->joint_color_counts[c];
    }
    // PHYS_STAGE_PREPARE_BODIES.
    for (unsigned i = 0U; i < n; ++i) {
        FN(prepare_body)(&s, wp, &v->bodies[i], i);
    }
    // PHYS_STAGE_PREPARE_CONTACTS: joints, then the groups.
    for (unsigned i = 0U; i < v->joint_count; ++i) {
        FN(prepare_joint)(&s, &v->joints[i], n, v->bodies, v->fixed_bodies, &s.j[i]);
    }
    for (unsigned c = 0U; c < NPH_GPU_COLOR_SLOTS; ++c) {
        const unsigned per = c == NPH_GPU_OVERFLOW ? 1U : 8U; // PHYS_LANES
        const unsigned count = v->contact_color_counts[c];
        for (unsigned i = 0U; i < count; ++i) {
            const unsigned g0 = (i / per) * per;
            const unsigned g1 = g0 + per < count ? g0 + per : count;
            unsigned group_points = 0U;
            for (unsigned q = g0; q < g1; ++q) {
                const unsigned pc = v->contacts[s.color_first[c] + q].point_count;
                group_points = pc > group_points ? pc : group_points;
            }
            FN(prepare_manifold)(&s, &v->contacts[s.color_first[c] + i], n, v->bodies,
                                 v->fixed_bodies, &s.m[s.color_first[c] + i], group_points);
        }
    }
    *sp = s;
    return NPH_GPU_OK;
}

// The whole stage: returns the working state for the caller to read back (and free).
static int FN(run)(const NphGpuWorldParams *wp, float dt, const NphGpuWorldView *v, FN(Result) *out)
{
    const unsigned n = v->body_count;
    FN(Step) s;
    const int rc = FN(setup)(&s, wp, dt, v);
    if (rc != NPH_GPU_OK) {
        return rc;
    }
    for (unsigned sub = 0U; sub < wp->substeps; ++sub) {
        for (unsigned i = 0U; i < n; ++i) {
            FN(integrate_velocity)(&s, i);
        }
        FN(contact_pass)(&s, v, FN(PASS_WARM));
        FN(contact_pass)(&s, v, FN(PASS_SOLVE));
        for (unsigned i = 0U; i < n; ++i) {
            FN(integrate_position)(&s, i);
        }
        if (s.solver == NPH_GPU_SOLVER_SOFT_STEP) {
            FN(contact_pass)(&s, v, FN(PASS_RELAX));
        }
    }
    if (s.solver == NPH_GPU_SOLVER_TGS) {
        FN(contact_pass)(&s, v, FN(PASS_RELAX)); // TGS's one velocity pass without bias
    }
    FN(contact_pass)(&s, v, FN(PASS_RESTITUTION));
    free(s.params);
    out->bodies = s.bodies;
    out->m = s.m;
    out->j = s.j;
    out->n = n;
    return NPH_GPU_OK;
}

// ---------------------------------------------------------------------------------------
// The residual-driven mode that judges a warm start (no counterpart in the reference; the
// device's nph_gpu_world_converge): prepare, the first substep's velocity integration and
// warm start, then rigid passes (the relax pass) until the velocity-constraint residual
// falls to `tol` x the reference residual.
// ---------------------------------------------------------------------------------------

// The residual, in double: over points, r_n = |vn + b| where the normal impulse is positive,
// else max(-(vn + b), 0) (b = separation / h for a separated point), plus the slip |vt|
// where the friction impulse is inside the cone (|tau| < 0.999 mu lambda).
static double FN(residual)(const FN(Step) *s, unsigned count)
{
    double sum = 0.0;
    for (unsigned g = 0U; g < count; ++g) {
        const FN(Manifold) *m = &s->m[g];
        const FN(Body) *a = &s->bodies[m->ia];
        const FN(Body) *b = &s->bodies[m->ib];
        for (unsigned k = 0U; k < m->point_count; ++k) {
            const FN(Point) *p = &m->p[k];
            const REAL sep = FN(separation)(a, b, p, m->n);
            const V3 dv = FN(sub)(FN(add)(b->v, FN(cross)(b->w, p->rb)), FN(add)(a->v, FN(cross)(a->w, p->ra)));
            const double vn = (double)FN(dot)(dv, m->n) + (sep > R(0) ? (double)sep * (double)s->inv_h : 0.0);
            const double lambda = (double)p->normal_impulse;
            const double rn = lambda > 0.0 ? fabs(vn) : (vn < 0.0 ? -vn : 0.0);
            double rt = 0.0;
            const double t1 = (double)p->tangent_impulse[0], t2 = (double)p->tangent_impulse[1];
            if (sqrt(t1 * t1 + t2 * t2) < (double)m->friction * lambda * 0.999) {
                const double v1 = (double)FN(dot)(dv, m->t1), v2 = (double)FN(dot)(dv, m->t2);
                rt = v1 * v1 + v2 * v2;
            }
            sum += rn * rn + rt;
        }
    }
    return sqrt(sum);
}

// `init` (12 floats per manifold, or NULL): the starting normal, t1 and t2 impulses of cold
// points (those whose warm start is zero), per point slot 4 g + k. Writes the residual after
// the warm start and after each pass to residuals[0..passes], the passes run, the cold points
// and (when `impulses` is given) every slot's final impulses.
static int FN(converge)(const NphGpuWorldParams *wp, float dt, const NphGpuWorldView *v, const float *init,
                        double tol, unsigned max_passes, double ref, double *residuals, unsigned *passes_out,
                        unsigned *cold_out, float *impulses)
{
    const unsigned n = v->body_count;
    const unsigned count = v->contact_count;
    FN(Step) s;
    const int rc = FN(setup)(&s, wp, dt, v);
    if (rc != NPH_GPU_OK) {
        return rc;
    }
    unsigned cold = 0U;
    for (unsigned g = 0U; g < count; ++g) {
        FN(Manifold) *m = &s.m[g];
        for (unsigned k = 0U; k < m->point_count; ++k) {
            FN(Point) *p = &m->p[k];
            if (p->normal_impulse == R(0) && p->tangent_impulse[0] == R(0) && p->tangent_impulse[1] == R(0)) {
                ++cold;
                if (init != NULL) {
                    const float *q = &init[12U * g + 3U * k];
                    p->normal_impulse = R(q[0]);
                    p->tangent_impulse[0] = R(q[1]);
                    p->tangent_impulse[1] = R(q[2]);
                }
            }
        }
    }
    for (unsigned i = 0U; i < n; ++i) {
        FN(integrate_velocity)(&s, i);
    }
    FN(contact_pass)(&s, v, FN(PASS_WARM));
    double r = FN(residual)(&s, count);
    residuals[0] = r;
    const double reference = ref > 0.0 ? ref : r;
    unsigned passes = 0U;
    while (r > tol * reference && passes < max_passes) {
        FN(contact_pass)(&s, v, FN(PASS_RELAX));
        ++passes;
        r = FN(residual)(&s, count);
        residuals[passes] = r;
    }
    *passes_out = passes;
    *cold_out = cold;
    if (impulses != NULL) {
        for (unsigned g = 0U; g < count; ++g) {
            for (unsigned k = 0U; k < 4U; ++k) {
                const FN(Point) *p = &s.m[g].p[k];
                const int live = k < s.m[g].point_count;
                impulses[12U * g + 3U * k] = live ? (float)p->normal_impulse : 0.0F;
                impulses[12U * g + 3U * k + 1U] = live ? (float)p->tangent_impulse[0] : 0.0F;
                impulses[12U * g + 3U * k + 2U] = live ? (float)p->tangent_impulse[1] : 0.0F;
            }
        }
    }
    free(s.params);
    free(s.bodies);
    free(s.m);
    free(s.j);
    return NPH_GPU_OK;
}

#undef V3
#undef Q4
#undef M3
#undef FN
#undef R

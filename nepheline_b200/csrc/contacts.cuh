// SPDX-License-Identifier: Apache-2.0
//
// The contact rows of the soft step, one manifold per lane: prepare, warm start, solve and
// relax, restitution, store (engine/physics/src/solver_impl.h:107-668, solver.c:394-499).
// The reference runs eight manifolds per call in SIMD lanes; here each CUDA thread owns
// one manifold, so a warp covers 32 manifolds of one colour, which share no dynamic body.
//
// Two decisions of the reference are made per eight-lane group (its colour's list cut in
// eights, solver.c:810-843): the normal rows get seven more sweeps when any lane is an
// impact and the group's largest point count is above one (solver_impl.h:533-566), and
// restitution sweeps eight times when that count is above one (solver_impl.h:637). The
// manifold header carries the group's largest point count, so each lane decides alone.
// Rows the reference runs past a lane's own points have zero masses and change no value
// (at most the sign of a zero); the one place they matter, the share of a hit's warm start,
// visits them here too with zero anchors (solver_impl.h:210-235).
//
// A side that is not dynamic takes no impulse: its inverse mass and inertia are zero and
// its velocities are never written (write_mask, solver_impl.h:74-105), so its updates are
// skipped outright.
#pragma once

#include "layout.cuh"

namespace nph {

// solver_impl.h:121-142: vB + wB x rB - (vA + wA x rA).
NPH_D V3 rel_vel(const BodyState &a, const BodyState &b, V3 ra, V3 rb)
{
    const V3 ca = cross(a.w, ra);
    const V3 cb = cross(b.w, rb);
    return sub(add(b.v, cb), add(a.v, ca));
}

// solver_impl.h:147-168, A's half: A loses the impulse `lambda` along `axis`; `ang` is
// I_A^-1 (r_A x axis).
NPH_D void apply_a(BodyState &a, float ma, float lambda, V3 axis, V3 ang)
{
    const float la = ma * lambda;
    a.v.x = a.v.x - la * axis.x;
    a.v.y = a.v.y - la * axis.y;
    a.v.z = a.v.z - la * axis.z;
    a.w.x = a.w.x - lambda * ang.x;
    a.w.y = a.w.y - lambda * ang.y;
    a.w.z = a.w.z - lambda * ang.z;
}

// B's half: B gains it.
NPH_D void apply_b(BodyState &b, float mb, float lambda, V3 axis, V3 ang)
{
    const float lb = mb * lambda;
    b.v.x = b.v.x + lb * axis.x;
    b.v.y = b.v.y + lb * axis.y;
    b.v.z = b.v.z + lb * axis.z;
    b.w.x = b.w.x + lambda * ang.x;
    b.w.y = b.w.y + lambda * ang.y;
    b.w.z = b.w.z + lambda * ang.z;
}

// Both halves, for the sides that take results.
struct Sides {
    bool wa, wb;
    float ma, mb;
    M3 ia, ib;
};

NPH_D void apply2(const Sides &s, BodyState &a, BodyState &b, float lambda, V3 axis, V3 ra, V3 rb)
{
    if (s.wa) {
        apply_a(a, s.ma, lambda, axis, m_mul_v(s.ia, cross(ra, axis)));
    }
    if (s.wb) {
        apply_b(b, s.mb, lambda, axis, m_mul_v(s.ib, cross(rb, axis)));
    }
}

NPH_D Sides load_sides(const float4 *prm, uint32_t ia, uint32_t ib, uint32_t bits)
{
    Sides s;
    s.wa = (bits & kHdrWriteA) != 0u;
    s.wb = (bits & kHdrWriteB) != 0u;
    s.ma = 0.0f;
    s.mb = 0.0f;
    s.ia = m_zero();
    s.ib = m_zero();
    if (s.wa) {
        s.ia = load_inv_inertia(prm, ia, &s.ma);
    }
    if (s.wb) {
        s.ib = load_inv_inertia(prm, ib, &s.mb);
    }
    return s;
}

// ---------------------------------------------------------------------------------------
// Prepare: prepare_group (solver.c:394-473) and the prepare kernel (solver_impl.h:276-385)
// ---------------------------------------------------------------------------------------

// `c` is the manifold's record; `ia`/`ib` its bodies' solver slots (the dummy for bodies
// without one), `dyn_a`/`dyn_b` whether they are dynamic and `ma`/`mb` their inverse masses
// (zero unless dynamic). Writes the manifold's rows at lane g.
NPH_D void prepare_manifold(const DevSolver &S, uint32_t g, const NphGpuContact &c, uint32_t ia,
                            uint32_t ib, bool dyn_a, bool dyn_b, float ma, float mb,
                            uint32_t group_points)
{
    float unused;
    // prm holds zeros for a body that is not dynamic and for the dummy: dyn ? params : zero.
    const M3 ii_a = dyn_a ? load_inv_inertia(S.prm, ia, &unused) : m_zero();
    const M3 ii_b = dyn_b ? load_inv_inertia(S.prm, ib, &unused) : m_zero();
    const V3 n = v3(c.normal[0], c.normal[1], c.normal[2]);
    const V3 t1 = perpendicular(n);
    const V3 t2 = cross(n, t1);
    const BodyState a = load_state(S.vel, ia);
    const BodyState b = load_state(S.vel, ib);
    const float mass = ma + mb;
    const uint32_t pc = c.point_count;
    bool impact = false;
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            const NphGpuContactPoint &cp = c.points[k];
            const V3 ra = v3(cp.anchor_a[0], cp.anchor_a[1], cp.anchor_a[2]);
            const V3 rb = v3(cp.anchor_b[0], cp.anchor_b[1], cp.anchor_b[2]);
            const float gap = dot(sub(rb, ra), n);
            const float adjusted = cp.separation - gap;
            const V3 rxa_n = cross(ra, n);
            const V3 rxa_1 = cross(ra, t1);
            const V3 rxa_2 = cross(ra, t2);
            const V3 rxb_n = cross(rb, n);
            const V3 rxb_1 = cross(rb, t1);
            const V3 rxb_2 = cross(rb, t2);
            const V3 aa_n = m_mul_v(ii_a, rxa_n);
            const V3 aa_1 = m_mul_v(ii_a, rxa_1);
            const V3 aa_2 = m_mul_v(ii_a, rxa_2);
            const V3 ab_n = m_mul_v(ii_b, rxb_n);
            const V3 ab_1 = m_mul_v(ii_b, rxb_1);
            const V3 ab_2 = m_mul_v(ii_b, rxb_2);
            const float kn = mass + dot(rxa_n, aa_n) + dot(rxb_n, ab_n);
            const float normal_mass = kn > 0.0f ? 1.0f / kn : 0.0f;
            const float k11 = mass + dot(rxa_1, aa_1) + dot(rxb_1, ab_1);
            const float k22 = mass + dot(rxa_2, aa_2) + dot(rxb_2, ab_2);
            const float k12 = dot(rxa_1, aa_2) + dot(rxb_1, ab_2);
            const float det = k11 * k22 - k12 * k12;
            const float inv = det > 0.0f ? 1.0f / det : 0.0f;
            const float rv = dot(rel_vel(a, b, ra, rb), n);
            const V3 ti = v3(cp.tangent_impulse[0], cp.tangent_impulse[1], cp.tangent_impulse[2]);
            impact = impact || rv < -1.0f; // PHYS_IMPACT_SPEED, world_internal.h:382
            const uint32_t row = k * S.mcap + g;
            __stcs(&S.pa[row], f4(ra, adjusted));
            __stcs(&S.pb[row], f4(rb, normal_mass));
            __stcs(&S.pt[row], make_float4(k22 * inv, -k12 * inv, k11 * inv, rv));
            __stcs(&S.pi[row], make_float4(cp.normal_impulse, 0.0f, dot(ti, t1), dot(ti, t2)));
        }
    }
    uint32_t bits = pc | (group_points << kHdrGroupShift);
    bits |= dyn_a ? kHdrWriteA : 0u;
    bits |= dyn_b ? kHdrWriteB : 0u;
    bits |= (!dyn_a || !dyn_b) ? kHdrStaticSoft : 0u;
    bits |= impact ? kHdrImpact : 0u;
    bits |= (c.flags & NPH_GPU_CONTACT_HIT) != 0u ? kHdrImpacted : 0u;
    S.hdr[g] = make_uint4(ia, ib, bits, 0u);
}

// ---------------------------------------------------------------------------------------
// Warm start (solver_impl.h:181-258)
// ---------------------------------------------------------------------------------------

// The passes read a manifold's point rows once each and the prepare and the passes write them
// once (__ldcs / __stcs: evicted first), so the body rows every manifold of a body reads stay in
// L2 (measured 0.8 % and 0.3 % off the lattice step).

// Where a pass reads a manifold's body velocities it first calls gate(hdr): a dependency-driven
// pass (solver.cu k_pass_flow) waits there for the constraints of earlier colours on the
// bodies; a pass that runs a colour a launch reads them straight away.
struct NoGate {
    NPH_D void operator()(uint4) const {}
};

template <class Gate = NoGate>
NPH_D void warm_manifold(const DevSolver &S, uint32_t g, const Gate &gate = Gate())
{
    uint4 hdr = S.hdr[g];
    const V3 n = v3(S.nrm[g]);
    const uint32_t bits = hdr.z;
    const uint32_t pc = bits & kHdrPointsMask;
    if (pc == 0u) {
        return;
    }
    // Every load of the manifold at once: the rows, the bodies, their inertia.
    V3 ra[4], rb[4];
    float4 im[4];
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            const uint32_t row = k * S.mcap + g;
            ra[k] = v3(__ldcs(&S.pa[row]));
            rb[k] = v3(__ldcs(&S.pb[row]));
            im[k] = __ldcs(&S.pi[row]);
        }
    }
    const Sides sd = load_sides(S.prm, hdr.x, hdr.y, bits);
    gate(hdr);
    BodyState a = load_state(S.vel, hdr.x);
    BodyState b = load_state(S.vel, hdr.y);
    const V3 t1 = perpendicular(n);
    const V3 t2 = cross(n, t1);
    if ((bits & kHdrImpacted) != 0u) {
        // The normal speeds now and after the whole warm start, and the share of it that
        // pushes no point apart faster than it already moves apart.
        BodyState a1 = a;
        BodyState b1 = b;
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < pc) {
                apply2(sd, a1, b1, im[k].x, n, ra[k], rb[k]);
                apply2(sd, a1, b1, im[k].z, t1, ra[k], rb[k]);
                apply2(sd, a1, b1, im[k].w, t2, ra[k], rb[k]);
            }
        }
        float share = 1.0f;
        const uint32_t gp = (bits >> kHdrGroupShift) & kHdrPointsMask;
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < gp) {
                // Points of the group this lane lacks have zero anchors.
                const V3 za = k < pc ? ra[k] : v3(0.0f, 0.0f, 0.0f);
                const V3 zb = k < pc ? rb[k] : v3(0.0f, 0.0f, 0.0f);
                const float before = dot(rel_vel(a, b, za, zb), n);
                const float after = dot(rel_vel(a1, b1, za, zb), n);
                const float allowed = fmax_ref(before, 0.0f);
                const bool pushed = after > allowed;
                const float part = (allowed - before) / (pushed ? after - before : 1.0f);
                share = fmin_ref(share, pushed ? part : 1.0f);
            }
        }
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < pc) {
                im[k].x = im[k].x * share;
                im[k].z = im[k].z * share;
                im[k].w = im[k].w * share;
                __stcs(&S.pi[k * S.mcap + g], im[k]);
            }
        }
        hdr.z = bits & ~kHdrImpacted;
        S.hdr[g] = hdr;
    }
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            apply2(sd, a, b, im[k].x, n, ra[k], rb[k]);
            apply2(sd, a, b, im[k].z, t1, ra[k], rb[k]);
            apply2(sd, a, b, im[k].w, t2, ra[k], rb[k]);
        }
    }
    if (sd.wa) {
        store_state(S.vel, hdr.x, a);
    }
    if (sd.wb) {
        store_state(S.vel, hdr.y, b);
    }
}

// ---------------------------------------------------------------------------------------
// Solve and relax (solver_impl.h:400-602)
// ---------------------------------------------------------------------------------------

// solver_impl.h:446-464: the current separation from the bodies' motion this step.
NPH_D float separation(const BodyPose &a, const BodyPose &b, V3 ra, V3 rb, float adjusted, V3 n)
{
    const V3 pa = rotate(a.dq, ra);
    const V3 pb = rotate(b.dq, rb);
    const V3 d = v3((b.dp.x - a.dp.x) + (pb.x - pa.x), (b.dp.y - a.dp.y) + (pb.y - pa.y),
                    (b.dp.z - a.dp.z) + (pb.z - pa.z));
    return dot(d, n) + adjusted;
}

// solver_impl.h:471-482 (`slop`: TGS's; the soft step's is zero).
NPH_D void normal_row(float s, float inv_h, float slop, float soft_bias, float min_bias, float soft_mass,
                      float soft_impulse, float &bias, float &mass_scale, float &impulse_scale)
{
    const bool apart = s > 0.0f;
    const float overlap = fmin_ref(s + slop, 0.0f);
    bias = apart ? s * inv_h : fmax_ref(soft_bias * overlap, min_bias);
    mass_scale = apart ? 1.0f : soft_mass;
    impulse_scale = apart ? 0.0f : soft_impulse;
}

// solver_impl.h:400-421. The reference computes every branch of every lane and selects;
// here only the selected branch is computed, with the same operations, so the results are the
// same bits: inside the circle the impulse stands, past it without slip it is scaled to the
// circle, and sliding it blends towards opposing the slip.
NPH_D void friction_circle(float vt1, float vt2, float limit, float &new1, float &new2)
{
    const float len = sqrtf(new1 * new1 + new2 * new2);
    if (!(len > limit)) {
        return;
    }
    const float slip = sqrtf(vt1 * vt1 + vt2 * vt2);
    const float r = limit / len;
    if (!(slip > 0.0f)) {
        new1 = new1 * r;
        new2 = new2 * r;
        return;
    }
    const float stop_share = r / len;
    const float slip_share = (1.0f - r) / slip;
    const float d1 = stop_share * new1 - slip_share * vt1;
    const float d2 = stop_share * new2 - slip_share * vt2;
    const float dlen = sqrtf(d1 * d1 + d2 * d2);
    const float to_edge = limit / dlen;
    new1 = d1 * to_edge;
    new2 = d2 * to_edge;
}

template <bool kUseBias>
NPH_D void solve_manifold(const DevSolver &S, uint32_t g, const StepConsts &K)
{
    const uint4 hdr = S.hdr[g];
    const float4 nf = S.nrm[g];
    const uint32_t bits = hdr.z;
    const uint32_t pc = bits & kHdrPointsMask;
    if (pc == 0u) {
        return;
    }
    const Sides sd = load_sides(S.prm, hdr.x, hdr.y, bits);
    BodyState a = load_state(S.vel, hdr.x);
    BodyState b = load_state(S.vel, hdr.y);
    const BodyPose pa_ = load_pose(S.pos, hdr.x);
    const BodyPose pb_ = load_pose(S.pos, hdr.y);
    const V3 n = v3(nf);
    const float friction = nf.w;
    const Soft soft = (bits & kHdrStaticSoft) != 0u ? K.static_soft : K.contact_soft;
    const float soft_bias = kUseBias ? soft.bias_rate : 0.0f;
    const float soft_mass = kUseBias ? soft.mass_scale : 1.0f;
    const float soft_impulse = kUseBias ? soft.impulse_scale : 0.0f;
    const float min_bias = -K.push_max;

    V3 ra[4], rb[4];
    float adj[4], nm[4];
    float4 im[4], tm[4];
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            const uint32_t row = k * S.mcap + g;
            const float4 A = __ldcs(&S.pa[row]);
            const float4 B = __ldcs(&S.pb[row]);
            ra[k] = v3(A);
            adj[k] = A.w;
            rb[k] = v3(B);
            nm[k] = B.w;
            im[k] = __ldcs(&S.pi[row]);
            tm[k] = __ldcs(&S.pt[row]);
        }
    }
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            float bias, mass_scale, impulse_scale;
            normal_row(separation(pa_, pb_, ra[k], rb[k], adj[k], n), K.inv_h, K.slop, soft_bias,
                       min_bias, soft_mass, soft_impulse, bias, mass_scale, impulse_scale);
            const float vn = dot(rel_vel(a, b, ra[k], rb[k]), n);
            const float row = nm[k] * mass_scale;
            const float acc = im[k].x;
            const float impulse = -(row * (vn + bias)) - impulse_scale * acc;
            const float total = fmax_ref(acc + impulse, 0.0f);
            const float delta = total - acc;
            im[k].x = total;
            im[k].y = fmax_ref(im[k].y, total);
            apply2(sd, a, b, delta, n, ra[k], rb[k]);
        }
    }
    // Under TGS a hit scales the next warm start (solver_impl.h:528-532).
    if (K.scale_hits != 0u && (bits & kHdrImpact) != 0u) {
        S.hdr[g].z = bits | kHdrImpacted;
    }
    const uint32_t gp = (bits >> kHdrGroupShift) & kHdrPointsMask;
    if (gp > 1u && (bits & kHdrImpact) != 0u) {
        // The rows as the pass made them (the bodies have not moved), swept seven more times
        // (PHYS_IMPACT_SWEEPS, world_internal.h:383).
        float row_bias[4], row_mass[4], row_soft[4];
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < pc) {
                float mass_scale;
                normal_row(separation(pa_, pb_, ra[k], rb[k], adj[k], n), K.inv_h, K.slop, soft_bias,
                           min_bias, soft_mass, soft_impulse, row_bias[k], mass_scale, row_soft[k]);
                row_mass[k] = nm[k] * mass_scale;
            }
        }
        for (uint32_t sweep = 0; sweep < 7u; ++sweep) {
#pragma unroll
            for (uint32_t k = 0; k < 4u; ++k) {
                if (k < pc) {
                    const float vn = dot(rel_vel(a, b, ra[k], rb[k]), n);
                    const float acc = im[k].x;
                    const float impulse = -(row_mass[k] * (vn + row_bias[k])) - row_soft[k] * acc;
                    const float total = fmax_ref(acc + impulse, 0.0f);
                    const float delta = total - acc;
                    im[k].x = total;
                    im[k].y = fmax_ref(im[k].y, total);
                    apply2(sd, a, b, delta, n, ra[k], rb[k]);
                }
            }
        }
    }
    const V3 t1 = perpendicular(n);
    const V3 t2 = cross(n, t1);
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            const V3 dv = rel_vel(a, b, ra[k], rb[k]);
            const float vt1 = dot(dv, t1);
            const float vt2 = dot(dv, t2);
            const float old1 = im[k].z;
            const float old2 = im[k].w;
            float new1 = old1 - (tm[k].x * vt1 + tm[k].y * vt2);
            float new2 = old2 - (tm[k].y * vt1 + tm[k].z * vt2);
            friction_circle(vt1, vt2, friction * im[k].x, new1, new2);
            im[k].z = new1;
            im[k].w = new2;
            apply2(sd, a, b, new1 - old1, t1, ra[k], rb[k]);
            apply2(sd, a, b, new2 - old2, t2, ra[k], rb[k]);
        }
    }
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            __stcs(&S.pi[k * S.mcap + g], im[k]);
        }
    }
    if (sd.wa) {
        store_state(S.vel, hdr.x, a);
    }
    if (sd.wb) {
        store_state(S.vel, hdr.y, b);
    }
}

// ---------------------------------------------------------------------------------------
// Restitution (solver_impl.h:611-668)
// ---------------------------------------------------------------------------------------

NPH_D void restitution_manifold(const DevSolver &S, uint32_t g, const StepConsts &K)
{
    const uint4 hdr = S.hdr[g];
    const uint32_t bits = hdr.z;
    const uint32_t pc = bits & kHdrPointsMask;
    if (pc == 0u) {
        return;
    }
    bool loaded[4];
    float4 tmv[4];
    float4 im[4];
    bool bounced = false;
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        loaded[k] = false;
        if (k < pc) {
            tmv[k] = __ldcs(&S.pt[k * S.mcap + g]);
            im[k] = __ldcs(&S.pi[k * S.mcap + g]);
            loaded[k] = tmv[k].w < -K.restitution_threshold && im[k].y > 0.0f;
            bounced = bounced || loaded[k];
        }
    }
    if (!bounced) {
        return;
    }
    // Under TGS a bounce is the step's alone, not the next step's warm start
    // (solver_impl.h:662-665).
    if (K.scale_hits != 0u) {
        S.hdr[g].z = bits | kHdrImpacted;
    }
    const Sides sd = load_sides(S.prm, hdr.x, hdr.y, bits);
    BodyState a = load_state(S.vel, hdr.x);
    BodyState b = load_state(S.vel, hdr.y);
    const V3 n = v3(S.nrm[g]);
    const float e = S.rest[g];
    V3 ra[4], rb[4];
    float nm[4];
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            ra[k] = v3(__ldcs(&S.pa[k * S.mcap + g]));
            const float4 B = __ldcs(&S.pb[k * S.mcap + g]);
            rb[k] = v3(B);
            nm[k] = B.w;
        }
    }
    const uint32_t gp = (bits >> kHdrGroupShift) & kHdrPointsMask;
    const uint32_t sweeps = gp > 1u ? 8u : 1u; // 1 + PHYS_IMPACT_SWEEPS
    for (uint32_t sweep = 0; sweep < sweeps; ++sweep) {
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < pc && loaded[k]) {
                const float vn = dot(rel_vel(a, b, ra[k], rb[k]), n);
                const float acc = im[k].x;
                const float impulse = -(nm[k] * (vn + e * tmv[k].w));
                const float total = fmax_ref(acc + impulse, 0.0f);
                const float delta = total - acc;
                im[k].x = acc + delta;
                im[k].y = fmax_ref(im[k].y, acc + delta);
                apply2(sd, a, b, delta, n, ra[k], rb[k]);
            }
        }
    }
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc && loaded[k]) {
            __stcs(&S.pi[k * S.mcap + g], im[k]);
        }
    }
    if (sd.wa) {
        store_state(S.vel, hdr.x, a);
    }
    if (sd.wb) {
        store_state(S.vel, hdr.y, b);
    }
}

// ---------------------------------------------------------------------------------------
// Store (solver.c:475-499)
// ---------------------------------------------------------------------------------------

NPH_D void store_manifold(const DevSolver &S, uint32_t g, NphGpuContact &c)
{
    const uint4 hdr = S.hdr[g];
    const uint32_t bits = hdr.z;
    const uint32_t pc = bits & kHdrPointsMask;
    if (pc == 0u) {
        return;
    }
    c.flags = (bits & kHdrImpacted) != 0u ? (c.flags | NPH_GPU_CONTACT_HIT)
                                          : (c.flags & ~NPH_GPU_CONTACT_HIT);
    const V3 n = v3(S.nrm[g]);
    const V3 t1 = perpendicular(n);
    const V3 t2 = cross(n, t1);
    for (uint32_t k = 0; k < pc; ++k) {
        const uint32_t row = k * S.mcap + g;
        const float4 im = S.pi[row];
        NphGpuContactPoint &cp = c.points[k];
        cp.normal_impulse = im.x;
        cp.max_normal_impulse = im.y;
        cp.relative_velocity = S.pt[row].w;
        cp.tangent_impulse[0] = t1.x * im.z + t2.x * im.w;
        cp.tangent_impulse[1] = t1.y * im.z + t2.y * im.w;
        cp.tangent_impulse[2] = t1.z * im.z + t2.z * im.w;
    }
}

} // namespace nph

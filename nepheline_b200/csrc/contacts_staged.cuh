// SPDX-License-Identifier: Apache-2.0
//
// The warm start, solve and relax rows of contacts.cuh with their loads staged through shared
// memory: after the manifold's header, each lane issues every load it needs (its point rows
// and its two bodies' velocities, displacements and inertia) as asynchronous 16-byte copies
// into its own column of the block's tile, waits for them once, and computes from the tile.
// The copies hold no registers while in flight, so a lane keeps all of its loads in flight at
// once whatever its register budget. The tile is [slot][lane]: a warp's 32 lanes read 512
// contiguous bytes per slot, free of bank conflicts. The arithmetic is contacts.cuh's, in
// its order: the staged and unstaged passes give the same bits.
//
// The lean form (kBodies = false) stages only the point rows, which the arithmetic reads
// again and again, and loads the body rows straight into registers, where they stay for the
// whole manifold anyway: its tile is 16 slots instead of 30, so an SM holds more warps.
#pragma once

#include <cuda_pipeline_primitives.h>

#include "contacts.cuh"

namespace nph {

// Tile slots: per point k, 4k + {0 pa, 1 pb, 2 pi, 3 pt}; then the bodies.
constexpr uint32_t kSlotVa = 16, kSlotWa = 17, kSlotVb = 18, kSlotWb = 19;
constexpr uint32_t kSlotDpa = 20, kSlotDqa = 21, kSlotDpb = 22, kSlotDqb = 23;
constexpr uint32_t kSlotIa = 24, kSlotIb = 27; // three columns each
constexpr uint32_t kSlots = 30;
constexpr uint32_t kPointSlots = 16; // the lean form's tile: the point rows only

template <uint32_t kLanes> struct Tile {
    float4 *base;
    uint32_t lane;
    NPH_D float4 *at(uint32_t slot) const { return base + slot * kLanes + lane; }
    NPH_D float4 get(uint32_t slot) const { return *at(slot); }
};

NPH_D void copy16(float4 *dst, const float4 *src) { __pipeline_memcpy_async(dst, src, 16); }

// An asynchronous 16-byte copy with an L2 eviction policy: the manifold rows stream through
// (read once a pass, evicted first), the body rows (read by every manifold of the body, about
// the size of L2 for the 1M-body graph) are kept; measured 1.4 % off the step.
NPH_D void copy16_policy(float4 *dst, const float4 *src, uint64_t policy)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "l"(policy)
                 : "memory");
}
NPH_D uint64_t policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}
NPH_D uint64_t policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}

// A 16-byte load into registers with an L2 eviction policy (the lean form's body rows).
NPH_D float4 ld_policy(const float4 *src, uint64_t policy)
{
    float4 v;
    asm volatile("ld.global.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;\n"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(src), "l"(policy));
    return v;
}


// Issues the manifold's loads into the lane's column: the rows of its own points (pt only
// when `tangents`), and when `bodies` the velocities of both bodies, their displacements and
// rotations when `poses`, and the inertia of the sides that take results. The copies are not
// committed.
template <uint32_t kLanes>
NPH_D void issue_manifold(const DevSolver &S, uint32_t g, uint4 hdr, const Tile<kLanes> &T,
                          bool tangents, bool poses, bool bodies = true)
{
    const uint32_t bits = hdr.z;
    const uint32_t pc = bits & kHdrPointsMask;
    const uint64_t stream = policy_evict_first(), keep = policy_evict_last();
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            const uint32_t row = k * S.mcap + g;
            copy16_policy(T.at(4u * k + 0u), &S.pa[row], stream);
            copy16_policy(T.at(4u * k + 1u), &S.pb[row], stream);
            copy16_policy(T.at(4u * k + 2u), &S.pi[row], stream);
            if (tangents) {
                copy16_policy(T.at(4u * k + 3u), &S.pt[row], stream);
            }
        }
    }
    if (!bodies) {
        return;
    }
    copy16_policy(T.at(kSlotVa), &S.vel[2u * hdr.x], keep);
    copy16_policy(T.at(kSlotWa), &S.vel[2u * hdr.x + 1u], keep);
    copy16_policy(T.at(kSlotVb), &S.vel[2u * hdr.y], keep);
    copy16_policy(T.at(kSlotWb), &S.vel[2u * hdr.y + 1u], keep);
    if (poses) {
        copy16_policy(T.at(kSlotDpa), &S.pos[2u * hdr.x], keep);
        copy16_policy(T.at(kSlotDqa), &S.pos[2u * hdr.x + 1u], keep);
        copy16_policy(T.at(kSlotDpb), &S.pos[2u * hdr.y], keep);
        copy16_policy(T.at(kSlotDqb), &S.pos[2u * hdr.y + 1u], keep);
    }
    if ((bits & kHdrWriteA) != 0u) {
        copy16_policy(T.at(kSlotIa + 0u), &S.prm[3u * hdr.x + 0u], keep);
        copy16_policy(T.at(kSlotIa + 1u), &S.prm[3u * hdr.x + 1u], keep);
        copy16_policy(T.at(kSlotIa + 2u), &S.prm[3u * hdr.x + 2u], keep);
    }
    if ((bits & kHdrWriteB) != 0u) {
        copy16_policy(T.at(kSlotIb + 0u), &S.prm[3u * hdr.y + 0u], keep);
        copy16_policy(T.at(kSlotIb + 1u), &S.prm[3u * hdr.y + 1u], keep);
        copy16_policy(T.at(kSlotIb + 2u), &S.prm[3u * hdr.y + 2u], keep);
    }
}

// The same, committed and waited for.
template <uint32_t kLanes>
NPH_D void stage_manifold(const DevSolver &S, uint32_t g, uint4 hdr, const Tile<kLanes> &T,
                          bool tangents, bool poses)
{
    issue_manifold(S, g, hdr, T, tangents, poses);
    __pipeline_commit();
    __pipeline_wait_prior(0);
}

// The two bodies of a manifold as the passes use them.
struct ManifoldBodies {
    Sides sd;
    BodyState a, b;
    BodyPose pa, pb;
};

// The lean form's body rows, loaded into registers (the poses only when `poses`). The
// velocities come last, after `gate(hdr)`: a dependency-driven pass waits there for the
// constraints of earlier colours on the bodies (the poses and inertias do not change during a
// pass).
template <class Gate = NoGate>
NPH_D ManifoldBodies load_bodies(const DevSolver &S, uint4 hdr, bool poses, const Gate &gate = Gate())
{
    const uint64_t keep = policy_evict_last();
    const uint32_t bits = hdr.z;
    ManifoldBodies m;
    m.sd.wa = (bits & kHdrWriteA) != 0u;
    m.sd.wb = (bits & kHdrWriteB) != 0u;
    if (poses) {
        const float4 pa = ld_policy(&S.pos[2u * hdr.x], keep);
        const float4 qa = ld_policy(&S.pos[2u * hdr.x + 1u], keep);
        const float4 pb = ld_policy(&S.pos[2u * hdr.y], keep);
        const float4 qb = ld_policy(&S.pos[2u * hdr.y + 1u], keep);
        m.pa = BodyPose{v3(pa), q4(qa)};
        m.pb = BodyPose{v3(pb), q4(qb)};
    }
    m.sd.ma = 0.0f;
    m.sd.mb = 0.0f;
    m.sd.ia = m_zero();
    m.sd.ib = m_zero();
    if (m.sd.wa) {
        const float4 c0 = ld_policy(&S.prm[3u * hdr.x], keep);
        const float4 c1 = ld_policy(&S.prm[3u * hdr.x + 1u], keep);
        const float4 c2 = ld_policy(&S.prm[3u * hdr.x + 2u], keep);
        m.sd.ma = c0.w;
        m.sd.ia = M3{v3(c0), v3(c1), v3(c2)};
    }
    if (m.sd.wb) {
        const float4 c0 = ld_policy(&S.prm[3u * hdr.y], keep);
        const float4 c1 = ld_policy(&S.prm[3u * hdr.y + 1u], keep);
        const float4 c2 = ld_policy(&S.prm[3u * hdr.y + 2u], keep);
        m.sd.mb = c0.w;
        m.sd.ib = M3{v3(c0), v3(c1), v3(c2)};
    }
    gate(hdr);
    const float4 va = ld_policy(&S.vel[2u * hdr.x], keep);
    const float4 wa = ld_policy(&S.vel[2u * hdr.x + 1u], keep);
    const float4 vb = ld_policy(&S.vel[2u * hdr.y], keep);
    const float4 wb = ld_policy(&S.vel[2u * hdr.y + 1u], keep);
    m.a = BodyState{v3(va), v3(wa)};
    m.b = BodyState{v3(vb), v3(wb)};
    return m;
}

template <uint32_t kLanes> NPH_D Sides staged_sides(const Tile<kLanes> &T, uint32_t bits)
{
    Sides s;
    s.wa = (bits & kHdrWriteA) != 0u;
    s.wb = (bits & kHdrWriteB) != 0u;
    s.ma = 0.0f;
    s.mb = 0.0f;
    s.ia = m_zero();
    s.ib = m_zero();
    if (s.wa) {
        const float4 c0 = T.get(kSlotIa), c1 = T.get(kSlotIa + 1u), c2 = T.get(kSlotIa + 2u);
        s.ma = c0.w;
        s.ia = M3{v3(c0), v3(c1), v3(c2)};
    }
    if (s.wb) {
        const float4 c0 = T.get(kSlotIb), c1 = T.get(kSlotIb + 1u), c2 = T.get(kSlotIb + 2u);
        s.mb = c0.w;
        s.ib = M3{v3(c0), v3(c1), v3(c2)};
    }
    return s;
}

// warm_manifold (solver_impl.h:181-258) on the staged loads.
// kIssued: the lane's column already holds the manifold's loads (a pipelined pass issued and
// waited for them). kBodies: the tile holds the body rows (else they are loaded into registers).
template <uint32_t kLanes, bool kIssued = false, bool kBodies = true>
NPH_D void warm_manifold_staged(const DevSolver &S, uint32_t g, const Tile<kLanes> &T)
{
    uint4 hdr = S.hdr[g];
    const V3 n = v3(S.nrm[g]);
    const uint32_t bits = hdr.z;
    const uint32_t pc = bits & kHdrPointsMask;
    if (pc == 0u) {
        return;
    }
    Sides sd;
    BodyState a, b;
    if (kBodies) {
        if (!kIssued) {
            stage_manifold(S, g, hdr, T, false, false);
        }
        sd = staged_sides(T, bits);
        a = BodyState{v3(T.get(kSlotVa)), v3(T.get(kSlotWa))};
        b = BodyState{v3(T.get(kSlotVb)), v3(T.get(kSlotWb))};
    } else {
        issue_manifold(S, g, hdr, T, false, false, false);
        __pipeline_commit();
        const ManifoldBodies m = load_bodies(S, hdr, false);
        __pipeline_wait_prior(0);
        sd = m.sd;
        a = m.a;
        b = m.b;
    }
    const V3 t1 = perpendicular(n);
    const V3 t2 = cross(n, t1);
    if ((bits & kHdrImpacted) != 0u) {
        BodyState a1 = a;
        BodyState b1 = b;
        for (uint32_t k = 0; k < pc; ++k) {
            const V3 ra = v3(T.get(4u * k)), rb = v3(T.get(4u * k + 1u));
            const float4 im = T.get(4u * k + 2u);
            apply2(sd, a1, b1, im.x, n, ra, rb);
            apply2(sd, a1, b1, im.z, t1, ra, rb);
            apply2(sd, a1, b1, im.w, t2, ra, rb);
        }
        float share = 1.0f;
        const uint32_t gp = (bits >> kHdrGroupShift) & kHdrPointsMask;
        for (uint32_t k = 0; k < gp; ++k) {
            const V3 ra = k < pc ? v3(T.get(4u * k)) : v3(0.0f, 0.0f, 0.0f);
            const V3 rb = k < pc ? v3(T.get(4u * k + 1u)) : v3(0.0f, 0.0f, 0.0f);
            const float before = dot(rel_vel(a, b, ra, rb), n);
            const float after = dot(rel_vel(a1, b1, ra, rb), n);
            const float allowed = fmax_ref(before, 0.0f);
            const bool pushed = after > allowed;
            const float part = (allowed - before) / (pushed ? after - before : 1.0f);
            share = fmin_ref(share, pushed ? part : 1.0f);
        }
        for (uint32_t k = 0; k < pc; ++k) {
            float4 im = T.get(4u * k + 2u);
            im.x = im.x * share;
            im.z = im.z * share;
            im.w = im.w * share;
            *T.at(4u * k + 2u) = im;
            __stcs(&S.pi[k * S.mcap + g], im);
        }
        hdr.z = bits & ~kHdrImpacted;
        S.hdr[g] = hdr;
    }
    for (uint32_t k = 0; k < pc; ++k) {
        const V3 ra = v3(T.get(4u * k)), rb = v3(T.get(4u * k + 1u));
        const float4 im = T.get(4u * k + 2u);
        apply2(sd, a, b, im.x, n, ra, rb);
        apply2(sd, a, b, im.z, t1, ra, rb);
        apply2(sd, a, b, im.w, t2, ra, rb);
    }
    if (sd.wa) {
        store_state(S.vel, hdr.x, a);
    }
    if (sd.wb) {
        store_state(S.vel, hdr.y, b);
    }
}

// solve_manifold (solver_impl.h:484-602) on the staged loads; the lean form waits at `gate`
// before it reads the velocities (load_bodies).
template <bool kUseBias, uint32_t kLanes, bool kIssued = false, bool kBodies = true, class Gate = NoGate>
NPH_D void solve_manifold_staged(const DevSolver &S, uint32_t g, const StepConsts &K,
                                 const Tile<kLanes> &T, const Gate &gate = Gate())
{
    const uint4 hdr = S.hdr[g];
    const float4 nf = S.nrm[g];
    const uint32_t bits = hdr.z;
    const uint32_t pc = bits & kHdrPointsMask;
    if (pc == 0u) {
        return;
    }
    Sides sd;
    BodyState a, b;
    BodyPose pa_, pb_;
    if (kBodies) {
        if (!kIssued) {
            stage_manifold(S, g, hdr, T, true, true);
        }
        sd = staged_sides(T, bits);
        a = BodyState{v3(T.get(kSlotVa)), v3(T.get(kSlotWa))};
        b = BodyState{v3(T.get(kSlotVb)), v3(T.get(kSlotWb))};
        pa_ = BodyPose{v3(T.get(kSlotDpa)), q4(T.get(kSlotDqa))};
        pb_ = BodyPose{v3(T.get(kSlotDpb)), q4(T.get(kSlotDqb))};
    } else {
        issue_manifold(S, g, hdr, T, true, true, false);
        __pipeline_commit();
        const ManifoldBodies m = load_bodies(S, hdr, true, gate);
        __pipeline_wait_prior(0);
        sd = m.sd;
        a = m.a;
        b = m.b;
        pa_ = m.pa;
        pb_ = m.pb;
    }
    const V3 n = v3(nf);
    const float friction = nf.w;
    const Soft soft = (bits & kHdrStaticSoft) != 0u ? K.static_soft : K.contact_soft;
    const float soft_bias = kUseBias ? soft.bias_rate : 0.0f;
    const float soft_mass = kUseBias ? soft.mass_scale : 1.0f;
    const float soft_impulse = kUseBias ? soft.impulse_scale : 0.0f;
    const float min_bias = -K.push_max;
    for (uint32_t k = 0; k < pc; ++k) {
        const float4 A = T.get(4u * k), B = T.get(4u * k + 1u);
        float4 im = T.get(4u * k + 2u);
        const V3 ra = v3(A), rb = v3(B);
        float bias, mass_scale, impulse_scale;
        normal_row(separation(pa_, pb_, ra, rb, A.w, n), K.inv_h, K.slop, soft_bias, min_bias,
                   soft_mass, soft_impulse, bias, mass_scale, impulse_scale);
        const float vn = dot(rel_vel(a, b, ra, rb), n);
        const float row = B.w * mass_scale;
        const float acc = im.x;
        const float impulse = -(row * (vn + bias)) - impulse_scale * acc;
        const float total = fmax_ref(acc + impulse, 0.0f);
        const float delta = total - acc;
        im.x = total;
        im.y = fmax_ref(im.y, total);
        *T.at(4u * k + 2u) = im;
        apply2(sd, a, b, delta, n, ra, rb);
    }
    if (K.scale_hits != 0u && (bits & kHdrImpact) != 0u) {
        S.hdr[g].z = bits | kHdrImpacted;
    }
    const uint32_t gp = (bits >> kHdrGroupShift) & kHdrPointsMask;
    if (gp > 1u && (bits & kHdrImpact) != 0u) {
        float row_bias[4], row_mass[4], row_soft[4];
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < pc) {
                const float4 A = T.get(4u * k), B = T.get(4u * k + 1u);
                float mass_scale;
                normal_row(separation(pa_, pb_, v3(A), v3(B), A.w, n), K.inv_h, K.slop, soft_bias,
                           min_bias, soft_mass, soft_impulse, row_bias[k], mass_scale, row_soft[k]);
                row_mass[k] = B.w * mass_scale;
            }
        }
        for (uint32_t sweep = 0; sweep < 7u; ++sweep) {
#pragma unroll
            for (uint32_t k = 0; k < 4u; ++k) {
                if (k < pc) {
                    const V3 ra = v3(T.get(4u * k)), rb = v3(T.get(4u * k + 1u));
                    float4 im = T.get(4u * k + 2u);
                    const float vn = dot(rel_vel(a, b, ra, rb), n);
                    const float acc = im.x;
                    const float impulse = -(row_mass[k] * (vn + row_bias[k])) - row_soft[k] * acc;
                    const float total = fmax_ref(acc + impulse, 0.0f);
                    const float delta = total - acc;
                    im.x = total;
                    im.y = fmax_ref(im.y, total);
                    *T.at(4u * k + 2u) = im;
                    apply2(sd, a, b, delta, n, ra, rb);
                }
            }
        }
    }
    const V3 t1 = perpendicular(n);
    const V3 t2 = cross(n, t1);
    for (uint32_t k = 0; k < pc; ++k) {
        const V3 ra = v3(T.get(4u * k)), rb = v3(T.get(4u * k + 1u));
        const float4 tm = T.get(4u * k + 3u);
        float4 im = T.get(4u * k + 2u);
        const V3 dv = rel_vel(a, b, ra, rb);
        const float vt1 = dot(dv, t1);
        const float vt2 = dot(dv, t2);
        const float old1 = im.z;
        const float old2 = im.w;
        float new1 = old1 - (tm.x * vt1 + tm.y * vt2);
        float new2 = old2 - (tm.y * vt1 + tm.z * vt2);
        friction_circle(vt1, vt2, friction * im.x, new1, new2);
        im.z = new1;
        im.w = new2;
        __stcs(&S.pi[k * S.mcap + g], im);
        apply2(sd, a, b, new1 - old1, t1, ra, rb);
        apply2(sd, a, b, new2 - old2, t2, ra, rb);
    }
    if (sd.wa) {
        store_state(S.vel, hdr.x, a);
    }
    if (sd.wb) {
        store_state(S.vel, hdr.y, b);
    }
}

} // namespace nph

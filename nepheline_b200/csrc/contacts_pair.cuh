// SPDX-License-Identifier: Apache-2.0
//
// The warm start of contacts.cuh (solver_impl.h:181-258) with two lanes a manifold: the even
// lane of a pair holds body A's side (its velocity, inverse inertia and mass, the points'
// anchors on A), the odd lane body B's. Each lane applies the stored impulses of every point to
// its own body (A loses them, B gains them), the angular term I^-1 (r x axis) of its own side
// only, so the two sides run in parallel. Only the hit share of an impacted manifold needs both
// sides: the relative velocity (v_B + w_B x r_B) - (v_A + w_A x r_A) is made from each lane's
// term and its partner's, traded with one shuffle within the pair, by both lanes in the
// reference's order, so both hold the same bits. The results equal contacts.cuh's bit for bit.
// The two lanes of a pair always take the same branches, so the shuffles use a mask of the
// pair alone.
//
// The same split of the solve and relax passes was measured slower than one lane a manifold
// (both lanes repeat every row's scalar arithmetic and trade three values a row), so those
// passes keep one lane.
#pragma once

#include "contacts_staged.cuh"

namespace nph {

struct Pair {
    uint32_t mask; // this lane and its partner
    bool b;        // this lane holds body B's side
};

NPH_D float partner(const Pair &p, float x) { return __shfl_xor_sync(p.mask, x, 1); }
NPH_D V3 partner(const Pair &p, V3 v) { return v3(partner(p, v.x), partner(p, v.y), partner(p, v.z)); }

// One side's part of a constraint row.
struct Side {
    bool write;  // the side is dynamic: it takes the results
    float mass;  // inverse mass (zero unless dynamic)
    M3 inertia;  // world inverse inertia (zero unless dynamic)
    BodyState s; // velocities
};

// v + w x r, this side's term of the relative velocity (rel_vel, solver_impl.h:121-142).
NPH_D V3 side_velocity(const Side &d, V3 r) { return add(d.s.v, cross(d.s.w, r)); }

// The relative velocity from this lane's term and its partner's, in the reference's order.
NPH_D V3 pair_rel_vel(const Pair &p, const Side &d, V3 r)
{
    const V3 mine = side_velocity(d, r);
    const V3 theirs = partner(p, mine);
    return p.b ? sub(mine, theirs) : sub(theirs, mine);
}

// apply2's half for this lane's body (solver_impl.h:147-168).
NPH_D void pair_apply(const Pair &p, Side &d, float lambda, V3 axis, V3 r)
{
    if (!d.write) {
        return;
    }
    const V3 ang = m_mul_v(d.inertia, cross(r, axis));
    if (p.b) {
        apply_b(d.s, d.mass, lambda, axis, ang);
    } else {
        apply_a(d.s, d.mass, lambda, axis, ang);
    }
}

// warm_manifold (contacts.cuh; solver_impl.h:181-258) with the pair's lanes: each lane applies
// the stored impulses of every point to its own body. Only the hit share of an impacted
// manifold needs both sides (the normal speeds before and after the whole warm start).
NPH_D void warm_manifold_pair(const DevSolver &S, uint32_t g, const Pair &p)
{
    uint4 hdr = S.hdr[g];
    const V3 n = v3(S.nrm[g]);
    const uint32_t bits = hdr.z;
    const uint32_t pc = bits & kHdrPointsMask;
    if (pc == 0u) {
        return;
    }
    const uint64_t keep = policy_evict_last();
    const uint32_t body = p.b ? hdr.y : hdr.x;
    Side d;
    d.write = (bits & (p.b ? kHdrWriteB : kHdrWriteA)) != 0u;
    d.s = BodyState{v3(ld_policy(&S.vel[2u * body], keep)), v3(ld_policy(&S.vel[2u * body + 1u], keep))};
    d.mass = 0.0f;
    d.inertia = m_zero();
    if (d.write) {
        const float4 c0 = ld_policy(&S.prm[3u * body], keep), c1 = ld_policy(&S.prm[3u * body + 1u], keep),
                     c2 = ld_policy(&S.prm[3u * body + 2u], keep);
        d.mass = c0.w;
        d.inertia = M3{v3(c0), v3(c1), v3(c2)};
    }
    V3 r[4];
    float4 im[4];
    const float4 *own = p.b ? S.pb : S.pa;
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            const uint32_t row = k * S.mcap + g;
            r[k] = v3(__ldcs(&own[row]));
            im[k] = __ldcs(&S.pi[row]);
        }
    }
    const V3 t1 = perpendicular(n);
    const V3 t2 = cross(n, t1);
    if ((bits & kHdrImpacted) != 0u) {
        Side d1 = d;
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < pc) {
                pair_apply(p, d1, im[k].x, n, r[k]);
                pair_apply(p, d1, im[k].z, t1, r[k]);
                pair_apply(p, d1, im[k].w, t2, r[k]);
            }
        }
        float share = 1.0f;
        const uint32_t gp = (bits >> kHdrGroupShift) & kHdrPointsMask;
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < gp) {
                // Points of the group this lane lacks have zero anchors.
                const V3 z = k < pc ? r[k] : v3(0.0f, 0.0f, 0.0f);
                const float before = dot(pair_rel_vel(p, d, z), n);
                const float after = dot(pair_rel_vel(p, d1, z), n);
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
                if (!p.b) {
                    __stcs(&S.pi[k * S.mcap + g], im[k]);
                }
            }
        }
        if (!p.b) {
            hdr.z = bits & ~kHdrImpacted;
            S.hdr[g] = hdr;
        }
    }
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            pair_apply(p, d, im[k].x, n, r[k]);
            pair_apply(p, d, im[k].z, t1, r[k]);
            pair_apply(p, d, im[k].w, t2, r[k]);
        }
    }
    if (d.write) {
        store_state(S.vel, body, d.s);
    }
}

} // namespace nph

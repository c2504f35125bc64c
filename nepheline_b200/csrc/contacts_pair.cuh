// SPDX-License-Identifier: Apache-2.0
//
// The solve and relax rows of contacts.cuh (solver_impl.h:484-602) with two lanes a manifold:
// the even lane of a pair holds body A's side (its velocity, displacement, rotation, inverse
// inertia and mass, the points' anchors on A), the odd lane body B's. The rows' scalars (the
// separation, the approach speed, the impulses) are computed by both lanes from the same
// operands in the same order, so both hold the same bits; the only exchanges are the per-side
// partial sums the reference adds across the sides, traded with one shuffle within the pair:
//
//   separation   (dp_B - dp_A) + (q_B r_B - q_A r_A), each lane rotating its own anchor;
//   rel_vel      (v_B + w_B x r_B) - (v_A + w_A x r_A), each lane adding its own side;
//   apply        each lane applies the impulse to its own body (A loses it, B gains it), the
//                angular term I^-1 (r x axis) of its own side only.
//
// Each lane's chain of dependent operations is about half the one-lane manifold's, and it holds
// one body's state instead of two. The results equal contacts.cuh's bit for bit. The two lanes of
// a pair always take the same branches (their decisions come from the shared scalars), so the
// pair's shuffles use a mask of the pair alone and pairs of one warp may diverge.
//
// In the staged form the pair's point rows go through shared memory: each lane copies its own
// anchor rows and half of the shared ones (A the impulses, B the tangent masses) with
// asynchronous copies, and both read every row from the tile, so a lane keeps only the
// impulses and one body in registers. Two lanes share a manifold's rows: the tile is 4 KB a
// warp.
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
    BodyPose pose;
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

// separation (solver_impl.h:446-464) from this lane's rotated anchor and its partner's.
NPH_D float pair_separation(const Pair &p, const Side &d, V3 dp_a, V3 dp_b, V3 r, float adjusted, V3 n)
{
    const V3 mine = rotate(d.pose.dq, r);
    const V3 theirs = partner(p, mine);
    const V3 pa = p.b ? theirs : mine;
    const V3 pb = p.b ? mine : theirs;
    const V3 dd = v3((dp_b.x - dp_a.x) + (pb.x - pa.x), (dp_b.y - dp_a.y) + (pb.y - pa.y),
                     (dp_b.z - dp_a.z) + (pb.z - pa.z));
    return dot(dd, n) + adjusted;
}

// The staged form's tile: per point k the rows pa, pb, pi, pt at slots 4k..4k+3, a slot holding
// the block's manifolds in a row ([slot][manifold]).
struct PairTile {
    float4 *base;
    uint32_t stride; // manifolds of the block
    uint32_t m;      // this lane's manifold within the block
    NPH_D float4 *at(uint32_t slot) const { return base + slot * stride + m; }
    NPH_D float4 get(uint32_t slot) const { return *at(slot); }
};

// solve_manifold<kUseBias> (contacts.cuh) with the pair's lanes: manifold g, this lane's side.
template <bool kUseBias, bool kStaged = false>
NPH_D void solve_manifold_pair(const DevSolver &S, uint32_t g, const Pair &p, const StepConsts &K,
                               const PairTile &T = PairTile{nullptr, 0u, 0u})
{
    const uint4 hdr = S.hdr[g];
    const float4 nf = S.nrm[g];
    const uint32_t bits = hdr.z;
    const uint32_t pc = bits & kHdrPointsMask;
    if (pc == 0u) {
        return;
    }
    const uint64_t keep = policy_evict_last();
    const uint32_t body = p.b ? hdr.y : hdr.x;
    Side d;
    d.write = (bits & (p.b ? kHdrWriteB : kHdrWriteA)) != 0u;
    {
        const float4 v = ld_policy(&S.vel[2u * body], keep), w = ld_policy(&S.vel[2u * body + 1u], keep);
        const float4 dp = ld_policy(&S.pos[2u * body], keep), dq = ld_policy(&S.pos[2u * body + 1u], keep);
        d.s = BodyState{v3(v), v3(w)};
        d.pose = BodyPose{v3(dp), q4(dq)};
    }
    d.mass = 0.0f;
    d.inertia = m_zero();
    if (d.write) {
        const float4 c0 = ld_policy(&S.prm[3u * body], keep), c1 = ld_policy(&S.prm[3u * body + 1u], keep),
                     c2 = ld_policy(&S.prm[3u * body + 2u], keep);
        d.mass = c0.w;
        d.inertia = M3{v3(c0), v3(c1), v3(c2)};
    }
    // The points: this side's anchors; the adjusted separation (A's row) and the normal mass
    // (B's row); the impulses and tangent masses, which both lanes read.
    V3 r_reg[4];
    float adj_reg[4], nm_reg[4];
    float4 im[4], tm_reg[4];
    if (kStaged) {
        const uint64_t stream = policy_evict_first();
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < pc) {
                const uint32_t row = k * S.mcap + g;
                copy16_policy(T.at(4u * k + (p.b ? 1u : 0u)), &(p.b ? S.pb : S.pa)[row], stream);
                copy16_policy(T.at(4u * k + (p.b ? 3u : 2u)), &(p.b ? S.pt : S.pi)[row], stream);
            }
        }
        __pipeline_commit();
        __pipeline_wait_prior(0);
        __syncwarp(p.mask);
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < pc) {
                im[k] = T.get(4u * k + 2u);
            }
        }
    } else {
        const float4 *own = p.b ? S.pb : S.pa;
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < pc) {
                const uint32_t row = k * S.mcap + g;
                const float4 R = __ldcs(&own[row]);
                r_reg[k] = v3(R);
                const float other = partner(p, R.w);
                adj_reg[k] = p.b ? other : R.w;
                nm_reg[k] = p.b ? R.w : other;
                im[k] = __ldcs(&S.pi[row]);
                tm_reg[k] = __ldcs(&S.pt[row]);
            }
        }
    }
    auto anchor = [&](uint32_t k) -> V3 { return kStaged ? v3(T.get(4u * k + (p.b ? 1u : 0u))) : r_reg[k]; };
    auto adjusted = [&](uint32_t k) -> float { return kStaged ? T.get(4u * k).w : adj_reg[k]; };
    auto normal_mass = [&](uint32_t k) -> float { return kStaged ? T.get(4u * k + 1u).w : nm_reg[k]; };
    auto tangent_mass = [&](uint32_t k) -> float4 { return kStaged ? T.get(4u * k + 3u) : tm_reg[k]; };
    const V3 my_dp = d.pose.dp;
    const V3 their_dp = partner(p, my_dp);
    const V3 dp_a = p.b ? their_dp : my_dp;
    const V3 dp_b = p.b ? my_dp : their_dp;
    const V3 n = v3(nf);
    const float friction = nf.w;
    const Soft soft = (bits & kHdrStaticSoft) != 0u ? K.static_soft : K.contact_soft;
    const float soft_bias = kUseBias ? soft.bias_rate : 0.0f;
    const float soft_mass = kUseBias ? soft.mass_scale : 1.0f;
    const float soft_impulse = kUseBias ? soft.impulse_scale : 0.0f;
    const float min_bias = -K.push_max;
    // One normal row of point k: the row made from the current poses (which do not move during
    // the pass, so a row remade later has the same bits) and its impulse.
    auto normal_step = [&](uint32_t k) {
        const V3 r = anchor(k);
        float bias, mass_scale, impulse_scale;
        normal_row(pair_separation(p, d, dp_a, dp_b, r, adjusted(k), n), K.inv_h, K.slop, soft_bias, min_bias,
                   soft_mass, soft_impulse, bias, mass_scale, impulse_scale);
        const float row = normal_mass(k) * mass_scale;
        const float vn = dot(pair_rel_vel(p, d, r), n);
        const float acc = im[k].x;
        const float impulse = -(row * (vn + bias)) - impulse_scale * acc;
        const float total = fmax_ref(acc + impulse, 0.0f);
        const float delta = total - acc;
        im[k].x = total;
        im[k].y = fmax_ref(im[k].y, total);
        pair_apply(p, d, delta, n, r);
    };
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            normal_step(k);
        }
    }
    if (K.scale_hits != 0u && (bits & kHdrImpact) != 0u && !p.b) {
        S.hdr[g].z = bits | kHdrImpacted;
    }
    const uint32_t gp = (bits >> kHdrGroupShift) & kHdrPointsMask;
    if (gp > 1u && (bits & kHdrImpact) != 0u) {
        // Seven more sweeps over the rows as the pass made them (PHYS_IMPACT_SWEEPS,
        // world_internal.h:383), each row remade from the unchanged poses.
        for (uint32_t sweep = 0; sweep < 7u; ++sweep) {
#pragma unroll
            for (uint32_t k = 0; k < 4u; ++k) {
                if (k < pc) {
                    normal_step(k);
                }
            }
        }
    }
    const V3 t1 = perpendicular(n);
    const V3 t2 = cross(n, t1);
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (k < pc) {
            const V3 r = anchor(k);
            const float4 tm = tangent_mass(k);
            const V3 dv = pair_rel_vel(p, d, r);
            const float vt1 = dot(dv, t1);
            const float vt2 = dot(dv, t2);
            const float old1 = im[k].z;
            const float old2 = im[k].w;
            float new1 = old1 - (tm.x * vt1 + tm.y * vt2);
            float new2 = old2 - (tm.y * vt1 + tm.z * vt2);
            friction_circle(vt1, vt2, friction * im[k].x, new1, new2);
            im[k].z = new1;
            im[k].w = new2;
            pair_apply(p, d, new1 - old1, t1, r);
            pair_apply(p, d, new2 - old2, t2, r);
        }
    }
    if (!p.b) {
#pragma unroll
        for (uint32_t k = 0; k < 4u; ++k) {
            if (k < pc) {
                __stcs(&S.pi[k * S.mcap + g], im[k]);
            }
        }
    }
    if (d.write) {
        store_state(S.vel, body, d.s);
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

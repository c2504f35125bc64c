// SPDX-License-Identifier: Apache-2.0
//
// The narrow phase's closed-form pairs on the device (collide.c:281-458, dispatch
// collide.c:474-535): sphere-sphere, capsule-sphere, capsule-capsule (with the segment
// distance of Ericson, "Real-Time Collision Detection" 5.1.9, collide.c:16-59) and
// box-sphere (the clamp, Ericson 5.1.3), and box-box and box-capsule (collide_box.cuh). Each
// keeps the reference's operations in its order, so a pair's manifold is the same bits as
// nph_physics_collide's. Hulls, meshes and heightfields are not here.
#pragma once

#include "nepheline_b200.h"

namespace nph_nc {

#define NPH_NC __host__ __device__ inline

struct V {
    float x, y, z;
};
struct Q {
    float x, y, z, w;
};

NPH_NC V v(float x, float y, float z) { return V{x, y, z}; }
NPH_NC V add(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }
NPH_NC V sub(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }
NPH_NC V scale(V a, float s) { return V{a.x * s, a.y * s, a.z * s}; }
NPH_NC V mul_add(V a, V b, float s) { return V{a.x + b.x * s, a.y + b.y * s, a.z + b.z * s}; }
NPH_NC V neg(V a) { return V{-a.x, -a.y, -a.z}; }
NPH_NC float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
NPH_NC V cross(V a, V b) { return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
NPH_NC float fmin_(float a, float b) { return a < b ? a : b; }
NPH_NC float fmax_(float a, float b) { return a > b ? a : b; }
NPH_NC float clamp01(float t) { return t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t); }
NPH_NC float at(V a, uint32_t i) { return i == 0u ? a.x : (i == 1u ? a.y : a.z); }
NPH_NC V absv(V a) { return V{fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }

// v + 2w (u x v) + u x (2 (u x v)), u the vector part (quat.h:157-164).
NPH_NC V rotate(Q q, V p)
{
    const V u{q.x, q.y, q.z};
    const V t = scale(cross(u, p), 2.0f);
    return add(add(p, scale(t, q.w)), cross(u, t));
}
NPH_NC V rotate_inverse(Q q, V p) { return rotate(Q{-q.x, -q.y, -q.z, q.w}, p); }
NPH_NC V axis_x(Q q)
{
    return V{1.0f - 2.0f * (q.y * q.y + q.z * q.z), 2.0f * (q.x * q.y + q.w * q.z), 2.0f * (q.x * q.z - q.w * q.y)};
}
NPH_NC V axis_y(Q q)
{
    return V{2.0f * (q.x * q.y - q.w * q.z), 1.0f - 2.0f * (q.x * q.x + q.z * q.z), 2.0f * (q.y * q.z + q.w * q.x)};
}

// The unit vector along a (a not zero): a / |a| as a times 1 / sqrt(|a|^2).
NPH_NC V normalize(V a) { return scale(a, 1.0f / sqrtf(dot(a, a))); }

// a's normalised direction, or `fallback` for a zero, underflowing or non-finite vector; a
// finite vector whose squared length overflows is rescaled by its largest component first.
NPH_NC V normalize_or(V a, V fallback)
{
    const float len_sq = dot(a, a);
    const float big = 3.402823466e+38f;
    if (len_sq > 0.0f && len_sq <= big) {
        return scale(a, 1.0f / sqrtf(len_sq));
    }
    if (!(len_sq > big) || !isfinite(a.x) || !isfinite(a.y) || !isfinite(a.z)) {
        return fallback;
    }
    const float m = fmax_(fabsf(a.x), fmax_(fabsf(a.y), fabsf(a.z)));
    const V u = scale(a, 1.0f / m);
    return scale(u, 1.0f / sqrtf(dot(u, u)));
}

// n x (the axis n leans on least), normalised (vec.h:460-469).
NPH_NC V perpendicular(V n)
{
    const V a = absv(n);
    const V axis = (a.x <= a.y && a.x <= a.z) ? V{1.0f, 0.0f, 0.0f} : (a.y <= a.z) ? V{0.0f, 1.0f, 0.0f} : V{0.0f, 0.0f, 1.0f};
    return normalize(cross(n, axis));
}

// The point of segment ab nearest to p and its fraction.
NPH_NC V closest_on_segment(V a, V b, V p, float *t_out)
{
    const V ab = sub(b, a);
    const float len_sq = dot(ab, ab);
    float t = 0.0f;
    if (len_sq > 0.0f) {
        t = clamp01(dot(sub(p, a), ab) / len_sq);
    }
    *t_out = t;
    return mul_add(a, ab, t);
}

struct SegmentDistance {
    V c1, c2;
    float dist_sq;
};

// The closest points of segments p1q1 and p2q2.
NPH_NC SegmentDistance segment_distance(V p1, V q1, V p2, V q2)
{
    const V d1 = sub(q1, p1), d2 = sub(q2, p2), r = sub(p1, p2);
    const float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    const float eps = 1e-12f;
    float s = 0.0f, t = 0.0f;
    if (a <= eps && e <= eps) {
        s = 0.0f;
        t = 0.0f;
    } else if (a <= eps) {
        t = clamp01(f / e);
    } else {
        const float c = dot(d1, r);
        if (e <= eps) {
            s = clamp01(-c / a);
        } else {
            const float b = dot(d1, d2);
            const float denom = a * e - b * b;
            s = denom > 0.0f ? clamp01((b * f - c * e) / denom) : 0.0f;
            t = (b * s + f) / e;
            if (t < 0.0f) {
                t = 0.0f;
                s = clamp01(-c / a);
            } else if (t > 1.0f) {
                t = 1.0f;
                s = clamp01((b - c) / a);
            }
        }
    }
    SegmentDistance out;
    out.c1 = mul_add(p1, d1, s);
    out.c2 = mul_add(p2, d2, t);
    const V d = sub(out.c1, out.c2);
    out.dist_sq = dot(d, d);
    return out;
}

NPH_NC void push(NphGpuManifold &m, V p, float sep, uint32_t id)
{
    if (m.point_count < NPH_GPU_MAX_POINTS) {
        NphGpuManifoldPoint &q = m.points[m.point_count++];
        q.point[0] = p.x;
        q.point[1] = p.y;
        q.point[2] = p.z;
        q.separation = sep;
        q.id = id;
    }
}

NPH_NC void set_normal(NphGpuManifold &m, V n)
{
    m.normal[0] = n.x;
    m.normal[1] = n.y;
    m.normal[2] = n.z;
}

// Two balls (collide.c:281-296).
NPH_NC void balls(V ca, float ra, V cb, float rb, float spec, uint32_t id, V fallback, NphGpuManifold &out)
{
    const V d = sub(cb, ca);
    const float dist_sq = dot(d, d);
    const float limit = ra + rb + spec;
    if (dist_sq > limit * limit) {
        return;
    }
    const float dist = sqrtf(dist_sq);
    const V n = dist > 1e-9f ? scale(d, 1.0f / dist) : fallback;
    const V sa = mul_add(ca, n, ra);
    const V sb = mul_add(cb, n, -rb);
    set_normal(out, n);
    push(out, scale(add(sa, sb), 0.5f), dist - ra - rb, id);
}

NPH_NC void capsule_core(float half_height, V pos, Q rot, V &p, V &q)
{
    const V axis = scale(axis_y(rot), half_height);
    p = sub(pos, axis);
    q = add(pos, axis);
}

// Capsule A and sphere B (collide.c:311-322).
NPH_NC void capsule_sphere(float hh, float ra, V pa, Q qa, float rb, V pb, float spec, NphGpuManifold &out)
{
    V p, q;
    capsule_core(hh, pa, qa, p, q);
    float t;
    const V c = closest_on_segment(p, q, pb, &t);
    balls(c, ra, pb, rb, spec, 0u, axis_x(qa), out);
}

// Two capsules (collide.c:324-396).
NPH_NC void capsules(float ha, float ra, V pa, Q qa, float hb, float rb, V pb, Q qb, float spec, NphGpuManifold &out)
{
    V a0, a1, b0, b1;
    capsule_core(ha, pa, qa, a0, a1);
    capsule_core(hb, pb, qb, b0, b1);
    const SegmentDistance sd = segment_distance(a0, a1, b0, b1);
    const float limit = ra + rb + spec;
    if (sd.dist_sq > limit * limit) {
        return;
    }
    const V da = sub(a1, a0), db = sub(b1, b0);
    const float la_sq = dot(da, da), lb_sq = dot(db, db);
    const float dist = sqrtf(sd.dist_sq);
    V n;
    if (dist > 1e-6f) {
        n = scale(sub(sd.c2, sd.c1), 1.0f / dist);
    } else {
        V c = cross(da, db);
        if (dot(c, c) <= 1e-12f * fmax_(la_sq * lb_sq, 1e-12f)) {
            c = la_sq > 0.0f ? perpendicular(normalize(da)) : V{0.0f, 1.0f, 0.0f};
        }
        n = normalize_or(c, V{0.0f, 1.0f, 0.0f});
        if (dot(n, sub(pb, pa)) < 0.0f) {
            n = neg(n);
        }
    }
    const V cr = cross(da, db);
    const float cross_sq = dot(cr, cr);
    if (la_sq > 1e-12f && lb_sq > 1e-12f && cross_sq <= 1e-4f * la_sq * lb_sq) {
        const float la = sqrtf(la_sq);
        const V ua = scale(da, 1.0f / la);
        const float t0 = dot(sub(b0, a0), ua);
        const float t1 = dot(sub(b1, a0), ua);
        const float lo = fmax_(0.0f, fmin_(t0, t1));
        const float hi = fmin_(la, fmax_(t0, t1));
        if (hi - lo > 0.005f) { // NPH_PHYSICS_LINEAR_SLOP, types.h:38
            const float ts[2] = {lo, hi};
            set_normal(out, n);
            for (uint32_t k = 0; k < 2u; ++k) {
                const V pa_core = mul_add(a0, ua, ts[k]);
                float tb;
                const V pb_core = closest_on_segment(b0, b1, pa_core, &tb);
                const float sep = dot(sub(pb_core, pa_core), n) - ra - rb;
                if (sep <= spec) {
                    const V sa = mul_add(pa_core, n, ra);
                    const V sb = mul_add(pb_core, n, -rb);
                    push(out, scale(add(sa, sb), 0.5f), sep, k);
                }
            }
            if (out.point_count > 0u) {
                return;
            }
        }
    }
    const V sa = mul_add(sd.c1, n, ra);
    const V sb = mul_add(sd.c2, n, -rb);
    set_normal(out, n);
    push(out, scale(add(sa, sb), 0.5f), dist - ra - rb, 2u);
}

// Box A and sphere B (collide.c:402-458).
NPH_NC void box_sphere(V h, V pa, Q qa, float rb, V pb, float spec, NphGpuManifold &out)
{
    const V c = rotate_inverse(qa, sub(pb, pa));
    const V q = V{fmin_(fmax_(c.x, -h.x), h.x), fmin_(fmax_(c.y, -h.y), h.y), fmin_(fmax_(c.z, -h.z), h.z)};
    const V d = sub(c, q);
    const float dist_sq = dot(d, d);
    V n_local, surface_a;
    float sep;
    uint32_t id;
    if (dist_sq > 0.0f) {
        const float limit = rb + spec;
        if (dist_sq > limit * limit) {
            return;
        }
        const float dist = sqrtf(dist_sq);
        n_local = scale(d, 1.0f / dist);
        surface_a = q;
        sep = dist - rb;
        id = 0u;
    } else {
        const V depth = sub(h, absv(c));
        uint32_t axis = 0u;
        if (depth.y < depth.x && depth.y <= depth.z) {
            axis = 1u;
        } else if (depth.z < depth.x && depth.z < depth.y) {
            axis = 2u;
        }
        const float s = at(c, axis) < 0.0f ? -1.0f : 1.0f;
        n_local = V{0.0f, 0.0f, 0.0f};
        surface_a = c;
        if (axis == 0u) {
            n_local.x = s;
            surface_a.x = s * h.x;
        } else if (axis == 1u) {
            n_local.y = s;
            surface_a.y = s * h.y;
        } else {
            n_local.z = s;
            surface_a.z = s * h.z;
        }
        sep = -at(depth, axis) - rb;
        id = 1u + axis;
    }
    const V surface_b = mul_add(c, n_local, -rb);
    const V mid = scale(add(surface_a, surface_b), 0.5f);
    set_normal(out, rotate(qa, n_local));
    push(out, add(rotate(qa, mid), pa), sep, id);
}

#include "collide_box.cuh"

NPH_NC V pos_of(const NphGpuPose &p) { return V{p.position[0], p.position[1], p.position[2]}; }
NPH_NC Q rot_of(const NphGpuPose &p) { return Q{p.rotation[0], p.rotation[1], p.rotation[2], p.rotation[3]}; }

// Pairs with a's type >= b's type (collide.c:474-519).
NPH_NC void collide_ordered(const NphGpuShape &a, const NphGpuPose &pa, const NphGpuShape &b, const NphGpuPose &pb,
                            float spec, NphGpuManifold &out)
{
    const V xa = pos_of(pa), xb = pos_of(pb);
    const Q ra = rot_of(pa), rb = rot_of(pb);
    if (a.type == NPH_GPU_SHAPE_SPHERE) {
        balls(xa, a.dims[0], xb, b.dims[0], spec, 0u, V{0.0f, 1.0f, 0.0f}, out);
    } else if (a.type == NPH_GPU_SHAPE_CAPSULE) {
        if (b.type == NPH_GPU_SHAPE_SPHERE) {
            capsule_sphere(a.dims[0], a.dims[1], xa, ra, b.dims[0], xb, spec, out);
        } else {
            capsules(a.dims[0], a.dims[1], xa, ra, b.dims[0], b.dims[1], xb, rb, spec, out);
        }
    } else if (a.type == NPH_GPU_SHAPE_BOX && b.type == NPH_GPU_SHAPE_SPHERE) {
        box_sphere(V{a.dims[0], a.dims[1], a.dims[2]}, xa, ra, b.dims[0], xb, spec, out);
    } else if (a.type == NPH_GPU_SHAPE_BOX && b.type == NPH_GPU_SHAPE_BOX) {
        boxes(V{a.dims[0], a.dims[1], a.dims[2]}, xa, ra, V{b.dims[0], b.dims[1], b.dims[2]}, xb, rb, spec, out);
    } else if (a.type == NPH_GPU_SHAPE_BOX && b.type == NPH_GPU_SHAPE_CAPSULE) {
        box_capsule(V{a.dims[0], a.dims[1], a.dims[2]}, xa, ra, b.dims[0], b.dims[1], xb, rb, spec, out);
    }
}

// nph_physics_collide (collide.c:524-535) for the closed-form pairs: the manifold of a and b,
// given in either order (the other order gives the same points and the normal reversed).
NPH_NC void collide(const NphGpuShape &a, const NphGpuPose &pa, const NphGpuShape &b, const NphGpuPose &pb,
                    float speculative, NphGpuManifold &out)
{
    // Cleared as nph_physics_manifold_clear does (physics_internal.h:294-298): +y, no points.
    out.normal[0] = 0.0f;
    out.normal[1] = 1.0f;
    out.normal[2] = 0.0f;
    out.point_count = 0u;
    const float spec = fmax_(speculative, 0.0f);
    if (a.type >= b.type) {
        collide_ordered(a, pa, b, pb, spec, out);
        return;
    }
    collide_ordered(b, pb, a, pa, spec, out);
    out.normal[0] = -out.normal[0];
    out.normal[1] = -out.normal[1];
    out.normal[2] = -out.normal[2];
}

#undef NPH_NC

} // namespace nph_nc

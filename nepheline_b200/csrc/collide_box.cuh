// SPDX-License-Identifier: Apache-2.0
//
// Box against box on the device (nph_physics_collide_boxes, collide_hull.c:1030-1266): the
// fifteen axes of the oriented-box test with closed-form projection radii; then the contact
// as the reference makes any hull pair's: the incident face of one box clipped against the
// reference face's side planes (face_contact, collide_hull.c:780-877) and reduced to four
// points by catch angle (nph_physics_manifold_reduce, collide.c:62-277); the closest points of
// the two supporting edges for an edge pair; and, for boxes apart by more than the linear
// slop, GJK's closest points with the signed-volumes subalgorithm (gjk.c:26-420). Every step
// keeps the reference's operations in its order, so a pair's manifold is the same bits as
// nph_physics_collide's. Included by collide.cuh inside its namespace.

// The box's topology as the reference's box view has it (collide_hull.c:48-100): corners by
// bit (x, y, z); faces -x +x -y +y -z +z, each with its first half-edge; half-edges as
// {next, twin, origin, face}. The polygon order and the feature ids of a face contact come
// from this table.
struct HalfEdge {
    uint16_t next, twin, origin, face;
};

NPH_NC uint32_t box_face_first(uint32_t f)
{
    constexpr uint16_t kFirst[6] = {0u, 8u, 16u, 5u, 7u, 19u};
    return kFirst[f];
}

NPH_NC HalfEdge box_edge_of(uint32_t e)
{
    constexpr uint16_t kEdges[24][4] = {
        {2u, 1u, 0u, 0u},   {16u, 0u, 4u, 2u},  {4u, 3u, 4u, 0u},   {19u, 2u, 6u, 5u},
        {6u, 5u, 6u, 0u},   {20u, 4u, 2u, 3u},  {0u, 7u, 2u, 0u},   {23u, 6u, 0u, 4u},
        {10u, 9u, 1u, 1u},  {17u, 8u, 3u, 4u},  {12u, 11u, 3u, 1u}, {22u, 10u, 7u, 3u},
        {14u, 13u, 7u, 1u}, {21u, 12u, 5u, 5u}, {8u, 15u, 5u, 1u},  {18u, 14u, 1u, 2u},
        {15u, 17u, 0u, 2u}, {7u, 16u, 1u, 4u},  {1u, 19u, 5u, 2u},  {13u, 18u, 4u, 5u},
        {11u, 21u, 6u, 3u}, {3u, 20u, 7u, 5u},  {5u, 23u, 3u, 3u},  {9u, 22u, 2u, 4u},
    };
    return HalfEdge{kEdges[e][0], kEdges[e][1], kEdges[e][2], kEdges[e][3]};
}

NPH_NC V box_vertex(V h, uint32_t i)
{
    return V{(i & 1u) != 0u ? h.x : -h.x, (i & 2u) != 0u ? h.y : -h.y, (i & 4u) != 0u ? h.z : -h.z};
}

struct Plane {
    V n;
    float d;
};

// The box's face planes (collide_hull.c:77-82): outward unit normal, d = -half extent.
NPH_NC Plane box_plane(V h, uint32_t f)
{
    const float s = (f & 1u) != 0u ? 1.0f : -1.0f;
    const uint32_t a = f >> 1;
    return Plane{V{a == 0u ? s : 0.0f, a == 1u ? s : 0.0f, a == 2u ? s : 0.0f}, -at(h, a)};
}

NPH_NC V axis_z(Q q)
{
    return V{2.0f * (q.x * q.z + q.w * q.y), 2.0f * (q.y * q.z - q.w * q.x),
             1.0f - 2.0f * (q.x * q.x + q.y * q.y)};
}

// quat.h:70-76.
NPH_NC Q q_mul(Q a, Q b)
{
    return Q{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
             a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}

NPH_NC float length_sq(V a) { return dot(a, a); }
NPH_NC float length(V a) { return sqrtf(dot(a, a)); }
// vec.h:427-430.
NPH_NC V reject(V v, V n) { return sub(v, scale(n, dot(v, n))); }
// scalar.h:108-111 per component.
NPH_NC V lerp(V a, V b, float t)
{
    return V{(1.0f - t) * a.x + t * b.x, (1.0f - t) * a.y + t * b.y, (1.0f - t) * a.z + t * b.z};
}
// vec.h:412-420.
NPH_NC uint32_t max_abs_index(V v)
{
    const V a = absv(v);
    return a.x >= a.y ? (a.x >= a.z ? 0u : 2u) : (a.y >= a.z ? 1u : 2u);
}

// physics_internal.h:286-291.
NPH_NC uint32_t mix_id(uint32_t a, uint32_t b)
{
    uint32_t h = a * 0x9E3779B1u;
    h ^= b + 0x7F4A7C15u + (h << 6u) + (h >> 2u);
    return h;
}

struct CPoint {
    V p;
    float sep;
    uint32_t id;
};

// A point of a polygon being clipped: its separation is not known until the clip ends, so the
// point is its place and feature id only, 16 bytes that move in one vector access.
struct __align__(16) ClipPoint {
    V p;
    uint32_t id;
};

// ---------------------------------------------------------------------------------------
// Manifold reduction by catch angle (collide.c:62-277)
// ---------------------------------------------------------------------------------------

struct ReduceAxis {
    V origin, across, normal;
    bool about_point;
    float side, min_arm;
};

NPH_NC float reduce_arm(const ReduceAxis &ax, V p)
{
    const V d = sub(p, ax.origin);
    float arm;
    if (ax.about_point) {
        arm = length_sq(reject(d, ax.normal));
    } else {
        const float a = dot(d, ax.across);
        arm = ax.side == 0.0f ? fabsf(a) : ax.side * a;
    }
    return arm > ax.min_arm ? arm : 0.0f;
}

NPH_NC uint32_t catches_first(const CPoint *pts, uint32_t from, uint32_t end, float level, const ReduceAxis &ax)
{
    uint32_t level_best = end;
    float level_arm = 0.0f;
    uint32_t least = end;
    float least_height = 0.0f, least_arm = 0.0f;
    for (uint32_t i = from; i < end; ++i) {
        const float arm = reduce_arm(ax, pts[i].p);
        if (!(arm > 0.0f)) {
            continue;
        }
        float height = pts[i].sep - level;
        if (!(height > 0.0f)) {
            if (arm > level_arm) {
                level_arm = arm;
                level_best = i;
            }
            continue;
        }
        height = ax.about_point ? height * height : height;
        if (least == end || height * least_arm < least_height * arm) {
            least = i;
            least_height = height;
            least_arm = arm;
        }
    }
    if (level_best != end || least == end) {
        return level_best;
    }
    const float tie = ax.about_point ? (1.0f + 0.1f) * (1.0f + 0.1f) : 1.0f + 0.1f;
    uint32_t best = least;
    float best_arm = least_arm;
    for (uint32_t i = from; i < end; ++i) {
        const float arm = reduce_arm(ax, pts[i].p);
        if (arm > best_arm) {
            float height = pts[i].sep - level;
            height = ax.about_point ? height * height : height;
            if (height * least_arm <= tie * least_height * arm) {
                best_arm = arm;
                best = i;
            }
        }
    }
    return best;
}

NPH_NC void swap_points(CPoint *pts, uint32_t i, uint32_t j)
{
    const CPoint t = pts[i];
    pts[i] = pts[j];
    pts[j] = t;
}

NPH_NC float signed_area(V a, V b, V c, V n) { return dot(cross(sub(b, a), sub(c, a)), n); }

NPH_NC uint32_t manifold_reduce(CPoint *pts, uint32_t count, V normal)
{
    if (count <= 4u) {
        return count;
    }
    constexpr float kLevel = 0.002f * 0.005f; // REDUCE_LEVEL: 0.002 x the linear slop
    float deepest = pts[0].sep;
    V centre = pts[0].p;
    for (uint32_t i = 1u; i < count; ++i) {
        deepest = fmin_(deepest, pts[i].sep);
        centre = add(centre, pts[i].p);
    }
    centre = scale(centre, 1.0f / (float)count);
    {
        uint32_t best = 0u;
        float far = -1.0f;
        for (uint32_t i = 0u; i < count; ++i) {
            const float dd = length_sq(reject(sub(pts[i].p, centre), normal));
            if (pts[i].sep <= deepest + kLevel && dd > far) {
                far = dd;
                best = i;
            }
        }
        swap_points(pts, 0u, best);
    }
    const float level = fmax_(deepest, 0.0f) + kLevel;
    const V p0 = pts[0].p;
    ReduceAxis ax{p0, V{0.0f, 0.0f, 0.0f}, normal, true, 0.0f, 1e-6f * 1e-6f};
    const uint32_t second = catches_first(pts, 1u, count, level, ax);
    if (second == count) {
        return 1u;
    }
    swap_points(pts, 1u, second);
    const V p1 = pts[1].p;
    const V line = reject(sub(p1, p0), normal);
    const float line_length = length(line);
    ax.about_point = false;
    ax.across = scale(cross(normal, line), 1.0f / line_length);
    ax.min_arm = 1e-3f * line_length;
    const uint32_t third = catches_first(pts, 2u, count, level, ax);
    if (third == count) {
        return 2u;
    }
    swap_points(pts, 2u, third);
    const V p2 = pts[2].p;
    ax.side = dot(sub(p2, p0), ax.across) < 0.0f ? 1.0f : -1.0f;
    uint32_t fourth = catches_first(pts, 3u, count, level, ax);
    if (fourth == count) {
        const float sign = signed_area(p0, p1, p2, normal) < 0.0f ? -1.0f : 1.0f;
        float best_out = -3.40282347e38f;
        fourth = 3u;
        for (uint32_t i = 3u; i < count; ++i) {
            const V p = pts[i].p;
            const float a0 = sign * signed_area(p0, p1, p, normal);
            const float a1 = sign * signed_area(p1, p2, p, normal);
            const float a2 = sign * signed_area(p2, p0, p, normal);
            const float out = -fmin_(a0, fmin_(a1, a2));
            if (out > best_out) {
                best_out = out;
                fourth = i;
            }
        }
    }
    swap_points(pts, 3u, fourth);
    return 4u;
}

// ---------------------------------------------------------------------------------------
// GJK distance between two vertex sets in one frame (gjk.c:26-420)
// ---------------------------------------------------------------------------------------

struct GjkVertex {
    V a, b, w;
    uint32_t ia, ib;
};

struct GjkSimplex {
    GjkVertex v[4];
    float lambda[4];
    uint32_t count;
};

// The identity pose's transforms, kept as operations (gjk.c:40-48).
NPH_NC V identity_point(V p) { return add(rotate(Q{0.0f, 0.0f, 0.0f, 1.0f}, p), V{0.0f, 0.0f, 0.0f}); }

// nph_physics_proxy_support (geometry.c:495-508) along a direction given in the common frame.
NPH_NC uint32_t support(const V *pts, uint32_t count, V direction)
{
    const V d = rotate_inverse(Q{0.0f, 0.0f, 0.0f, 1.0f}, direction);
    uint32_t best = 0u;
    float best_dot = dot(pts[0], d);
    for (uint32_t i = 1u; i < count; ++i) {
        const float x = dot(pts[i], d);
        if (x > best_dot) {
            best_dot = x;
            best = i;
        }
    }
    return best;
}

NPH_NC GjkVertex make_vertex(const V *pa, uint32_t ia, const V *pb, uint32_t ib)
{
    GjkVertex v;
    v.a = identity_point(pa[ia]);
    v.b = identity_point(pb[ib]);
    v.w = sub(v.a, v.b);
    v.ia = ia;
    v.ib = ib;
    return v;
}

NPH_NC bool same_sign(float a, float b) { return (a > 0.0f && b > 0.0f) || (a < 0.0f && b < 0.0f); }

// gjk.c:79-103.
NPH_NC void s1d(V s1, V s2, float *lambda)
{
    const V t = sub(s2, s1);
    const float tt = dot(t, t);
    if (!(tt > 0.0f)) {
        lambda[0] = 1.0f;
        lambda[1] = 0.0f;
        return;
    }
    const V p0 = mul_add(s1, t, -dot(s1, t) / tt);
    const uint32_t axis = max_abs_index(t);
    const float mu = at(s1, axis) - at(s2, axis);
    const float c1 = at(p0, axis) - at(s2, axis);
    const float c2 = at(s1, axis) - at(p0, axis);
    if (same_sign(mu, c1) && same_sign(mu, c2)) {
        lambda[0] = c1 / mu;
        lambda[1] = c2 / mu;
    } else if (same_sign(mu, c1)) {
        lambda[0] = 1.0f;
        lambda[1] = 0.0f;
    } else {
        lambda[0] = 0.0f;
        lambda[1] = 1.0f;
    }
}

NPH_NC V weighted2(V s1, V s2, const float *l) { return add(scale(s1, l[0]), scale(s2, l[1])); }
NPH_NC V weighted3(V s1, V s2, V s3, const float *l)
{
    return add(add(scale(s1, l[0]), scale(s2, l[1])), scale(s3, l[2]));
}

// gjk.c:116-142.
NPH_NC void s2d_edges(const V *s, const bool *test, float *lambda)
{
    float best = 3.40282347e38f;
    lambda[0] = 1.0f;
    lambda[1] = 0.0f;
    lambda[2] = 0.0f;
    for (uint32_t j = 0u; j < 3u; ++j) {
        if (!test[j]) {
            continue;
        }
        const uint32_t i0 = (j + 1u) % 3u;
        const uint32_t i1 = (j + 2u) % 3u;
        float l[2];
        s1d(s[i0], s[i1], l);
        const float d = length_sq(weighted2(s[i0], s[i1], l));
        if (d < best) {
            best = d;
            lambda[j] = 0.0f;
            lambda[i0] = l[0];
            lambda[i1] = l[1];
        }
    }
}

NPH_NC float area2(V p, V q, V r, uint32_t i, uint32_t j)
{
    return (at(q, i) - at(p, i)) * (at(r, j) - at(p, j)) - (at(q, j) - at(p, j)) * (at(r, i) - at(p, i));
}

// gjk.c:150-176.
NPH_NC void s2d(const V *s, float *lambda)
{
    const V n = cross(sub(s[1], s[0]), sub(s[2], s[0]));
    const float nn = dot(n, n);
    if (!(nn > 0.0f)) {
        const bool all[3] = {true, true, true};
        s2d_edges(s, all, lambda);
        return;
    }
    const V p0 = scale(n, dot(s[0], n) / nn);
    const uint32_t k = max_abs_index(n);
    const uint32_t i = (k + 1u) % 3u;
    const uint32_t j = (k + 2u) % 3u;
    const float mu = at(n, k);
    const float c[3] = {area2(p0, s[1], s[2], i, j), area2(s[0], p0, s[2], i, j), area2(s[0], s[1], p0, i, j)};
    const bool wrong[3] = {!same_sign(mu, c[0]), !same_sign(mu, c[1]), !same_sign(mu, c[2])};
    if (!wrong[0] && !wrong[1] && !wrong[2]) {
        lambda[0] = c[0] / mu;
        lambda[1] = c[1] / mu;
        lambda[2] = c[2] / mu;
        return;
    }
    s2d_edges(s, wrong, lambda);
}

NPH_NC float det3(V a, V b, V c) { return dot(a, cross(b, c)); }

// gjk.c:184-240: true when the origin is inside the tetrahedron.
NPH_NC bool s3d(const V *s, float *lambda)
{
    const V e1 = sub(s[1], s[0]);
    const V e2 = sub(s[2], s[0]);
    const V e3 = sub(s[3], s[0]);
    const float det = det3(e1, e2, e3);
    const V o0 = neg(s[0]);
    const float c[4] = {det3(s[1], s[2], s[3]), det3(o0, e2, e3), det3(e1, o0, e3), det3(e1, e2, o0)};
    bool wrong[4];
    bool inside = det != 0.0f;
    for (uint32_t i = 0u; i < 4u; ++i) {
        wrong[i] = !same_sign(det, c[i]);
        inside = inside && !wrong[i];
    }
    if (inside) {
        for (uint32_t i = 0u; i < 4u; ++i) {
            lambda[i] = c[i] / det;
        }
        return true;
    }
    float best = 3.40282347e38f;
    for (uint32_t i = 0u; i < 4u; ++i) {
        lambda[i] = i == 0u ? 1.0f : 0.0f;
    }
    for (uint32_t f = 0u; f < 4u; ++f) {
        if (!wrong[f] && det != 0.0f) {
            continue;
        }
        V tri[3];
        uint32_t map[3];
        uint32_t n = 0u;
        for (uint32_t i = 0u; i < 4u; ++i) {
            if (i != f) {
                tri[n] = s[i];
                map[n] = i;
                n += 1u;
            }
        }
        float l[3];
        s2d(tri, l);
        const float d = length_sq(weighted3(tri[0], tri[1], tri[2], l));
        if (d < best) {
            best = d;
            for (uint32_t i = 0u; i < 4u; ++i) {
                lambda[i] = 0.0f;
            }
            lambda[map[0]] = l[0];
            lambda[map[1]] = l[1];
            lambda[map[2]] = l[2];
        }
    }
    return false;
}

// gjk.c:243-284.
NPH_NC V simplex_solve(GjkSimplex &s, bool &inside)
{
    inside = false;
    float lambda[4] = {1.0f, 0.0f, 0.0f, 0.0f};
    if (s.count == 2u) {
        s1d(s.v[0].w, s.v[1].w, lambda);
    } else if (s.count == 3u) {
        const V tri[3] = {s.v[0].w, s.v[1].w, s.v[2].w};
        s2d(tri, lambda);
    } else if (s.count == 4u) {
        const V tet[4] = {s.v[0].w, s.v[1].w, s.v[2].w, s.v[3].w};
        inside = s3d(tet, lambda);
    }
    V v = V{0.0f, 0.0f, 0.0f};
    uint32_t kept = 0u;
    for (uint32_t i = 0u; i < s.count; ++i) {
        if (lambda[i] > 0.0f || s.count == 1u) {
            s.v[kept] = s.v[i];
            s.lambda[kept] = lambda[i];
            v = mul_add(v, s.v[i].w, lambda[i]);
            kept += 1u;
        }
    }
    if (kept == 0u) {
        s.lambda[0] = 1.0f;
        v = s.v[0].w;
        kept = 1u;
    }
    s.count = kept;
    return v;
}

struct GjkDistance {
    V point_a, point_b, normal;
    float distance;
};

// nph_physics_distance (gjk.c:306-420) of two point sets at the identity pose, without radii
// or a simplex cache.
NPH_NC GjkDistance gjk_distance(const V *pa, uint32_t na, const V *pb, uint32_t nb)
{
    GjkSimplex s;
    s.v[0] = make_vertex(pa, 0u, pb, 0u);
    s.count = 1u;
    const float scl = fmax_(length_sq(s.v[0].a), length_sq(s.v[0].b)) + length_sq(s.v[0].w) + 1e-12f;
    bool inside = false;
    V v = simplex_solve(s, inside);
    float v_sq = length_sq(v);
    uint32_t iterations = 0u;
    while (!inside && iterations < 40u) {
        if (v_sq <= 1e-12f * scl) {
            inside = true;
            break;
        }
        iterations += 1u;
        const uint32_t ia = support(pa, na, neg(v));
        const uint32_t ib = support(pb, nb, v);
        bool duplicate = false;
        for (uint32_t i = 0u; i < s.count; ++i) {
            duplicate = duplicate || (s.v[i].ia == ia && s.v[i].ib == ib);
        }
        if (duplicate) {
            break;
        }
        const GjkVertex w = make_vertex(pa, ia, pb, ib);
        if (v_sq - dot(v, w.w) <= 1e-6f * v_sq) {
            break;
        }
        s.v[s.count++] = w;
        bool in2 = false;
        const V v_new = simplex_solve(s, in2);
        inside = in2;
        const float v_new_sq = length_sq(v_new);
        if (!inside && v_new_sq >= v_sq) {
            break;
        }
        v = v_new;
        v_sq = v_new_sq;
    }
    // simplex_points (gjk.c:286-304).
    V a = V{0.0f, 0.0f, 0.0f}, b = V{0.0f, 0.0f, 0.0f};
    float total = 0.0f;
    for (uint32_t i = 0u; i < s.count; ++i) {
        a = mul_add(a, s.v[i].a, s.lambda[i]);
        b = mul_add(b, s.v[i].b, s.lambda[i]);
        total += s.lambda[i];
    }
    if (total > 0.0f && total != 1.0f) {
        a = scale(a, 1.0f / total);
        b = scale(b, 1.0f / total);
    }
    GjkDistance out;
    const float distance = inside ? 0.0f : length(sub(a, b));
    out.normal = V{0.0f, 1.0f, 0.0f};
    if (distance > 0.0f) {
        out.normal = scale(sub(b, a), 1.0f / distance);
    }
    out.point_a = a;
    out.point_b = b;
    out.distance = distance;
    return out;
}

// ---------------------------------------------------------------------------------------
// The pair
// ---------------------------------------------------------------------------------------

// More clipped points than a quadrilateral clipped by four planes can have (each plane at
// most doubles a polygon's points: 4 x 2^4), so the bound never cuts a polygon short, as the
// reference's larger bound never does for boxes.
constexpr uint32_t kClipCapacity = 65u;

struct BoxPair {
    V ha, hb;
    V rel_p;
    Q rel_q;
    V av[8], bv[8]; // A's corners, and B's in A's frame
};

// plane_b_in_a (collide_hull.c:418-423).
NPH_NC Plane plane_b_in_a(const BoxPair &bp, uint32_t f)
{
    const Plane pl = box_plane(bp.hb, f);
    const V n = rotate(bp.rel_q, pl.n);
    return Plane{n, pl.d - dot(n, bp.rel_p)};
}

// face_contact (collide_hull.c:780-877): reference face `ref` of A (of B when `flip`), the
// other box's incident face clipped against its sides; A-frame points; the normal from A to B.
NPH_NC V face_contact(const BoxPair &bp, bool flip, uint32_t ref, float speculative, CPoint *points,
                      uint32_t &count)
{
    const V *rv = flip ? bp.bv : bp.av;
    const V *iv = flip ? bp.av : bp.bv;
    const Plane ref_plane = flip ? plane_b_in_a(bp, ref) : box_plane(bp.ha, ref);
    const V n = ref_plane.n;
    uint32_t inc = 0u;
    float best = 3.40282347e38f;
    for (uint32_t f = 0u; f < 6u; ++f) {
        const V fn = flip ? box_plane(bp.ha, f).n : plane_b_in_a(bp, f).n;
        const float d = dot(fn, n);
        if (d < best) {
            best = d;
            inc = f;
        }
    }
    ClipPoint buf[2][kClipCapacity];
    uint32_t len = 0u;
    {
        const uint32_t first = box_face_first(inc);
        uint32_t e = first;
        do {
            const HalfEdge he = box_edge_of(e);
            buf[0][len] = ClipPoint{iv[he.origin], he.origin};
            len += 1u;
            e = he.next;
        } while (e != first && len < kClipCapacity && len < 24u);
    }
    uint32_t cur = 0u;
    const uint32_t first = box_face_first(ref);
    uint32_t e = first;
    uint32_t side = 0u;
    do {
        const HalfEdge he = box_edge_of(e);
        const V a = rv[he.origin];
        const V b = rv[box_edge_of(he.next).origin];
        const V sn = cross(sub(b, a), n);
        const float so = dot(sn, a);
        const ClipPoint *in = buf[cur];
        ClipPoint *outp = buf[cur ^ 1u];
        uint32_t out_len = 0u;
        for (uint32_t i = 0u; i < len && out_len + 1u < kClipCapacity; ++i) {
            const ClipPoint p = in[i];
            const ClipPoint q = in[(i + 1u) % len];
            const float dp = dot(sn, p.p) - so;
            const float dq = dot(sn, q.p) - so;
            if (dp <= 0.0f) {
                outp[out_len++] = p;
            }
            if ((dp <= 0.0f) != (dq <= 0.0f)) {
                const float t = dp / (dp - dq);
                outp[out_len] = ClipPoint{lerp(p.p, q.p, t), mix_id(mix_id(p.id, q.id), 0x100u + side)};
                out_len += 1u;
            }
        }
        len = out_len;
        cur ^= 1u;
        e = he.next;
        side += 1u;
    } while (e != first && len > 0u && side < 24u);
    const uint32_t tag = mix_id((flip ? 0x80000000u : 0u) | (ref << 16u), inc);
    const ClipPoint *clipped = buf[cur];
    CPoint cand[kClipCapacity];
    uint32_t n_out = 0u;
    for (uint32_t i = 0u; i < len; ++i) {
        const float sep = dot(ref_plane.n, clipped[i].p) + ref_plane.d;
        if (sep <= speculative) {
            cand[n_out].p = mul_add(clipped[i].p, n, -0.5f * sep);
            cand[n_out].sep = sep;
            cand[n_out].id = mix_id(tag, clipped[i].id);
            n_out += 1u;
        }
    }
    if (n_out > 4u) {
        n_out = manifold_reduce(cand, n_out, n);
    }
    for (uint32_t i = 0u; i < n_out; ++i) {
        points[i] = cand[i];
    }
    count = n_out;
    return flip ? neg(n) : n;
}

struct BoxAxes {
    float r[3][3];  // A_i . B_j
    float ar[3][3]; // |r| + 1e-6
    float t[3];     // B's centre in A's frame
    float ha[3], hb[3];
};

// collide_hull.c:1045-1050.
NPH_NC float box_face_a(const BoxAxes &x, uint32_t i, float &sign)
{
    const float rb = x.hb[0] * x.ar[i][0] + x.hb[1] * x.ar[i][1] + x.hb[2] * x.ar[i][2];
    sign = x.t[i] >= 0.0f ? 1.0f : -1.0f;
    return fabsf(x.t[i]) - (x.ha[i] + rb);
}

// collide_hull.c:1052-1058.
NPH_NC float box_face_b(const BoxAxes &x, uint32_t j, float &sign)
{
    const float tb = x.t[0] * x.r[0][j] + x.t[1] * x.r[1][j] + x.t[2] * x.r[2][j];
    const float ra = x.ha[0] * x.ar[0][j] + x.ha[1] * x.ar[1][j] + x.ha[2] * x.ar[2][j];
    sign = tb >= 0.0f ? 1.0f : -1.0f;
    return fabsf(tb) - (ra + x.hb[j]);
}

// collide_hull.c:1061-1083: along A_i x B_j normalised; -FLT_MAX for parallel axes.
NPH_NC float box_edge(const BoxAxes &x, uint32_t i, uint32_t j, V &axis)
{
    const uint32_t i1 = (i + 1u) % 3u, i2 = (i + 2u) % 3u;
    const uint32_t j1 = (j + 1u) % 3u, j2 = (j + 2u) % 3u;
    const float len_sq = 1.0f - x.r[i][j] * x.r[i][j];
    if (len_sq < 1e-6f) {
        return -3.40282347e38f;
    }
    const float ra = x.ha[i1] * x.ar[i2][j] + x.ha[i2] * x.ar[i1][j];
    const float rb = x.hb[j1] * x.ar[i][j2] + x.hb[j2] * x.ar[i][j1];
    const float tl = x.t[i2] * x.r[i1][j] - x.t[i1] * x.r[i2][j];
    const float inv_len = 1.0f / sqrtf(len_sq);
    float l[3];
    l[i] = 0.0f;
    l[i1] = -x.r[i2][j];
    l[i2] = x.r[i1][j];
    const float s = tl >= 0.0f ? inv_len : -inv_len;
    axis = V{l[0] * s, l[1] * s, l[2] * s};
    return (fabsf(tl) - (ra + rb)) * inv_len;
}

// nph_physics_collide_boxes (collide_hull.c:1085-1266) without the temporal-coherence cache,
// which only returns early for pairs the full test also finds apart.
NPH_NC void boxes(V half_a, V pa_p, Q pa_q, V half_b, V pb_p, Q pb_q, float speculative, NphGpuManifold &out)
{
    // nph_physics_pose_inv_mul (types.h:106-110).
    const V rel_p = rotate_inverse(pa_q, sub(pb_p, pa_p));
    const Q rel_q = q_mul(Q{-pa_q.x, -pa_q.y, -pa_q.z, pa_q.w}, pb_q);
    const V rc[3] = {axis_x(rel_q), axis_y(rel_q), axis_z(rel_q)};
    BoxAxes x;
    for (uint32_t i = 0u; i < 3u; ++i) {
        for (uint32_t j = 0u; j < 3u; ++j) {
            x.r[i][j] = at(rc[j], i);
            x.ar[i][j] = fabsf(x.r[i][j]) + 1e-6f;
        }
    }
    x.t[0] = rel_p.x;
    x.t[1] = rel_p.y;
    x.t[2] = rel_p.z;
    x.ha[0] = half_a.x;
    x.ha[1] = half_a.y;
    x.ha[2] = half_a.z;
    x.hb[0] = half_b.x;
    x.hb[1] = half_b.y;
    x.hb[2] = half_b.z;
    float face_a_sep = -3.40282347e38f;
    uint32_t face_a = 0u;
    for (uint32_t i = 0u; i < 3u; ++i) {
        float sign;
        const float s = box_face_a(x, i, sign);
        if (s > face_a_sep) {
            face_a_sep = s;
            face_a = 2u * i + (sign > 0.0f ? 1u : 0u);
        }
    }
    float face_b_sep = -3.40282347e38f;
    uint32_t face_b = 0u;
    for (uint32_t j = 0u; j < 3u; ++j) {
        float sign;
        const float s = box_face_b(x, j, sign);
        if (s > face_b_sep) {
            face_b_sep = s;
            face_b = 2u * j + (sign > 0.0f ? 0u : 1u);
        }
    }
    float edge_sep = -3.40282347e38f;
    uint32_t edge_i = 0u, edge_j = 0u;
    V edge_axis = V{0.0f, 1.0f, 0.0f};
    for (uint32_t i = 0u; i < 3u; ++i) {
        for (uint32_t j = 0u; j < 3u; ++j) {
            V axis;
            const float s = box_edge(x, i, j, axis);
            if (s > edge_sep) {
                edge_sep = s;
                edge_i = i;
                edge_j = j;
                edge_axis = axis;
            }
        }
    }
    constexpr float kSlop = 0.005f; // NPH_PHYSICS_LINEAR_SLOP
    constexpr float kEdgeBias = 0.5f * kSlop;
    constexpr float kFaceBias = 0.1f * kSlop;
    const float face_sep = fmax_(face_a_sep, face_b_sep);
    const bool use_edge = edge_sep > face_sep + kEdgeBias;
    const bool flip = !use_edge && face_b_sep > face_a_sep + kFaceBias;
    const float best = use_edge ? edge_sep : (flip ? face_b_sep : face_a_sep);
    if (fmax_(face_sep, edge_sep) > speculative) {
        return;
    }
    BoxPair bp;
    bp.ha = half_a;
    bp.hb = half_b;
    bp.rel_p = rel_p;
    bp.rel_q = rel_q;
    for (uint32_t i = 0u; i < 8u; ++i) {
        bp.av[i] = box_vertex(half_a, i);
        bp.bv[i] = add(rotate(rel_q, box_vertex(half_b, i)), rel_p);
    }
    if (best > kSlop) {
        const GjkDistance gd = gjk_distance(bp.av, 8u, bp.bv, 8u);
        if (gd.distance > speculative) {
            return;
        }
        const V sat_axis = use_edge ? edge_axis : (flip ? neg(plane_b_in_a(bp, face_b).n) : box_plane(half_a, face_a).n);
        if (gd.distance > 0.0f && (use_edge || dot(gd.normal, sat_axis) < 0.995f)) {
            const V mid = scale(add(gd.point_a, gd.point_b), 0.5f);
            set_normal(out, rotate(pa_q, gd.normal));
            push(out, add(rotate(pa_q, mid), pa_p), gd.distance, 0x40000000u);
            return;
        }
    }
    if (use_edge) {
        V ca = V{0.0f, 0.0f, 0.0f};
        for (uint32_t k = 0u; k < 3u; ++k) {
            if (k != edge_i) {
                const float s = at(edge_axis, k) >= 0.0f ? x.ha[k] : -x.ha[k];
                if (k == 0u) {
                    ca.x = s;
                } else if (k == 1u) {
                    ca.y = s;
                } else {
                    ca.z = s;
                }
            }
        }
        V ea = V{0.0f, 0.0f, 0.0f};
        if (edge_i == 0u) {
            ea.x = x.ha[0];
        } else if (edge_i == 1u) {
            ea.y = x.ha[1];
        } else {
            ea.z = x.ha[2];
        }
        V cb = rel_p;
        for (uint32_t m = 0u; m < 3u; ++m) {
            if (m != edge_j) {
                const float d = dot(rc[m], edge_axis);
                cb = mul_add(cb, rc[m], d >= 0.0f ? -x.hb[m] : x.hb[m]);
            }
        }
        const V eb = scale(rc[edge_j], x.hb[edge_j]);
        const SegmentDistance sd = segment_distance(sub(ca, ea), add(ca, ea), sub(cb, eb), add(cb, eb));
        const float sep = dot(sub(sd.c2, sd.c1), edge_axis);
        if (sep > speculative) {
            return;
        }
        const V mid = scale(add(sd.c1, sd.c2), 0.5f);
        set_normal(out, rotate(pa_q, edge_axis));
        push(out, add(rotate(pa_q, mid), pa_p), sep, mix_id(0x20000000u | edge_i, edge_j));
        return;
    }
    CPoint pts[4];
    uint32_t count = 0u;
    const V n = face_contact(bp, flip, flip ? face_b : face_a, speculative, pts, count);
    set_normal(out, rotate(pa_q, n));
    for (uint32_t i = 0u; i < count; ++i) {
        push(out, add(rotate(pa_q, pts[i].p), pa_p), pts[i].sep, pts[i].id);
    }
}

// ---------------------------------------------------------------------------------------
// Box and capsule (nph_physics_collide_hull_capsule, collide_hull.c:207-378, the box's view)
// ---------------------------------------------------------------------------------------

// clip_segment_to_face (collide_hull.c:207-249): the segment [p, q] clipped to the prism over
// face `face`; false when nothing is left.
NPH_NC bool clip_segment_to_face(V h, uint32_t face, V &p, V &q)
{
    const V n = box_plane(h, face).n;
    float t0 = 0.0f, t1 = 1.0f;
    const V p0 = p;
    const V d = sub(q, p);
    const uint32_t first = box_face_first(face);
    uint32_t e = first;
    uint32_t guard = 0u;
    do {
        const HalfEdge he = box_edge_of(e);
        const V a = box_vertex(h, he.origin);
        const V b = box_vertex(h, box_edge_of(he.next).origin);
        const V side = cross(sub(b, a), n);
        const float s0 = dot(side, sub(p0, a));
        const float sd = dot(side, d);
        if (sd == 0.0f) {
            if (s0 > 0.0f) {
                return false;
            }
        } else {
            const float t = -s0 / sd;
            if (sd > 0.0f) {
                t1 = fmin_(t1, t);
            } else {
                t0 = fmax_(t0, t);
            }
            if (t0 > t1) {
                return false;
            }
        }
        e = he.next;
        guard += 1u;
    } while (e != first && guard < 24u);
    p = mul_add(p0, d, t0);
    q = mul_add(p0, d, t1);
    return true;
}

NPH_NC void box_capsule(V h, V pa_p, Q pa_q, float half_height, float radius, V pb_p, Q pb_q, float speculative,
                        NphGpuManifold &out)
{
    const V rel_p = rotate_inverse(pa_q, sub(pb_p, pa_p));
    const Q rel_q = q_mul(Q{-pa_q.x, -pa_q.y, -pa_q.z, pa_q.w}, pb_q);
    const V axis = scale(axis_y(rel_q), half_height);
    const V s0 = sub(rel_p, axis);
    const V s1 = add(rel_p, axis);
    const float limit = radius + speculative;
    float face_sep = -3.40282347e38f;
    uint32_t face = 0u;
    for (uint32_t f = 0u; f < 6u; ++f) {
        const Plane pl = box_plane(h, f);
        const float s = fmin_(dot(pl.n, s0) + pl.d, dot(pl.n, s1) + pl.d);
        if (s > face_sep) {
            face_sep = s;
            face = f;
        }
    }
    if (face_sep > limit) {
        return;
    }
    const V d = sub(s1, s0);
    const float d_len_sq = length_sq(d);
    float edge_sep = -3.40282347e38f;
    uint32_t edge = 0u;
    V edge_axis = V{0.0f, 1.0f, 0.0f};
    if (d_len_sq > 1e-12f) {
        for (uint32_t e = 0u; e < 24u; e += 2u) {
            const HalfEdge he = box_edge_of(e);
            const V n1 = box_plane(h, he.face).n;
            const V n2 = box_plane(h, box_edge_of(e + 1u).face).n;
            if (dot(n1, d) * dot(n2, d) >= 0.0f) {
                continue;
            }
            const V p = box_vertex(h, he.origin);
            const V u = sub(box_vertex(h, box_edge_of(he.next).origin), p);
            V x = cross(u, d);
            const float len = length(x);
            if (len < 0.005f * sqrtf(length_sq(u) * d_len_sq)) {
                continue;
            }
            x = scale(x, 1.0f / len);
            if (dot(x, sub(p, V{0.0f, 0.0f, 0.0f})) < 0.0f) { // the box view's centroid is zero
                x = neg(x);
            }
            const float s = dot(x, sub(s0, p));
            if (s > edge_sep) {
                edge_sep = s;
                edge = e;
                edge_axis = x;
            }
        }
    }
    if (edge_sep > limit) {
        return;
    }
    constexpr float kSlop = 0.005f;
    const bool use_face = face_sep >= edge_sep - 0.5f * kSlop;
    const float best = use_face ? face_sep : edge_sep;
    if (best > kSlop) {
        V av[8];
        for (uint32_t i = 0u; i < 8u; ++i) {
            av[i] = box_vertex(h, i);
        }
        const V seg[2] = {s0, s1};
        const GjkDistance gd = gjk_distance(av, 8u, seg, d_len_sq > 0.0f ? 2u : 1u);
        if (gd.distance > limit) {
            return;
        }
        const V sat_axis = use_face ? box_plane(h, face).n : edge_axis;
        if (gd.distance > 0.0f && (!use_face || dot(gd.normal, sat_axis) < 0.995f)) {
            const V surface_b = mul_add(gd.point_b, gd.normal, -radius);
            const V mid = scale(add(gd.point_a, surface_b), 0.5f);
            set_normal(out, rotate(pa_q, gd.normal));
            push(out, add(rotate(pa_q, mid), pa_p), gd.distance - radius, 0x20000u);
            return;
        }
    }
    if (use_face) {
        const Plane pl = box_plane(h, face);
        V p = s0, q = s1;
        if (!clip_segment_to_face(h, face, p, q)) {
            p = (dot(pl.n, s0) + pl.d) <= (dot(pl.n, s1) + pl.d) ? s0 : s1;
            q = p;
        }
        set_normal(out, rotate(pa_q, pl.n));
        const V pts[2] = {p, q};
        const uint32_t count = length_sq(sub(p, q)) > 1e-12f ? 2u : 1u;
        for (uint32_t k = 0u; k < count; ++k) {
            const float dist = dot(pl.n, pts[k]) + pl.d;
            const float sep = dist - radius;
            if (sep <= speculative) {
                const V mid = mul_add(pts[k], pl.n, -0.5f * (dist + radius));
                push(out, add(rotate(pa_q, mid), pa_p), sep, (face << 8u) | k);
            }
        }
        return;
    }
    const HalfEdge he = box_edge_of(edge);
    const V ep = box_vertex(h, he.origin);
    const V eq = box_vertex(h, box_edge_of(he.next).origin);
    const SegmentDistance sd = segment_distance(ep, eq, s0, s1);
    const float sep = dot(sub(sd.c2, sd.c1), edge_axis) - radius;
    if (sep > speculative) {
        return;
    }
    const V surface_b = mul_add(sd.c2, edge_axis, -radius);
    const V mid = scale(add(sd.c1, surface_b), 0.5f);
    set_normal(out, rotate(pa_q, edge_axis));
    push(out, add(rotate(pa_q, mid), pa_p), sep, 0x10000u | edge);
}

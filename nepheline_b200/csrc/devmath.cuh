// SPDX-License-Identifier: Apache-2.0
//
// Vector, quaternion and matrix arithmetic of the reference's math library
// (engine/math/include/nepheline/math/{vec,quat,mat,scalar}.h), on the device. Each function
// keeps the reference's operation order: this translation unit is compiled with
// -fmad=false -prec-div=true -prec-sqrt=true -ftz=false, so every add, multiply, divide and
// square root rounds once to nearest as the reference's SSE/AVX code does (the reference
// forbids FMA contraction and keeps denormals, cmake/NphArch.cmake:23-31). Min and max are
// the reference's comparisons (a < b ? a : b, a > b ? a : b: scalar.h:67-74 and
// _mm_min_ps/_mm_max_ps), not fminf/fmaxf, whose signed-zero and NaN rules differ.
#pragma once

#include <cstdint>

#define NPH_D __device__ __forceinline__

namespace nph {

struct V3 {
    float x, y, z;
};
struct Q4 {
    float x, y, z, w;
};
// Column-major 3x3 (NphMat3): c0, c1, c2.
struct M3 {
    V3 c0, c1, c2;
};

NPH_D V3 v3(float x, float y, float z) { return V3{x, y, z}; }
NPH_D V3 v3(float4 a) { return V3{a.x, a.y, a.z}; }
NPH_D float4 f4(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
NPH_D Q4 q4(float4 a) { return Q4{a.x, a.y, a.z, a.w}; }
NPH_D float4 f4(Q4 q) { return make_float4(q.x, q.y, q.z, q.w); }

NPH_D float fmin_ref(float a, float b) { return a < b ? a : b; }
NPH_D float fmax_ref(float a, float b) { return a > b ? a : b; }

NPH_D V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
NPH_D V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
NPH_D V3 scale(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
NPH_D V3 neg(V3 a) { return V3{-a.x, -a.y, -a.z}; }
// vec.h:292-295: a + b s.
NPH_D V3 mul_add(V3 a, V3 b, float s) { return V3{a.x + b.x * s, a.y + b.y * s, a.z + b.z * s}; }
// vec.h:300-303: (ax bx + ay by) + az bz.
NPH_D float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// vec.h:305-308.
NPH_D V3 cross(V3 a, V3 b)
{
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
NPH_D float length(V3 a) { return sqrtf(dot(a, a)); }
// vec.h:326-331 with scalar.h:181-184: v * (1 / sqrt(|v|^2)), two rounded operations.
NPH_D V3 normalize(V3 a) { return scale(a, 1.0f / sqrtf(dot(a, a))); }

NPH_D Q4 q_identity() { return Q4{0.0f, 0.0f, 0.0f, 1.0f}; }
// quat.h:70-76.
NPH_D Q4 q_mul(Q4 a, Q4 b)
{
    return Q4{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
              a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
              a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
              a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
NPH_D Q4 q_conj(Q4 q) { return Q4{-q.x, -q.y, -q.z, q.w}; }
NPH_D Q4 q_scale(Q4 q, float s) { return Q4{q.x * s, q.y * s, q.z * s, q.w * s}; }
NPH_D float q_dot(Q4 a, Q4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
// quat.h:102-107.
NPH_D Q4 q_normalize(Q4 q) { return q_scale(q, 1.0f / sqrtf(q_dot(q, q))); }
// quat.h:109-113.
NPH_D Q4 q_normalize_or_identity(Q4 q)
{
    const float len_sq = q_dot(q, q);
    return len_sq > 0.0f ? q_scale(q, 1.0f / sqrtf(len_sq)) : q_identity();
}
// quat.h:156-163: v + 2 w (u x v) + 2 u x (u x v).
NPH_D V3 rotate(Q4 q, V3 v)
{
    const V3 u = V3{q.x, q.y, q.z};
    const V3 t = scale(cross(u, v), 2.0f);
    return add(add(v, scale(t, q.w)), cross(u, t));
}
// quat.h:234-239: normalize(q + (omega, 0) q * dt / 2), or the identity.
NPH_D Q4 q_integrate(Q4 q, V3 omega, float dt)
{
    const Q4 w = Q4{omega.x, omega.y, omega.z, 0.0f};
    const Q4 d = q_scale(q_mul(w, q), 0.5f * dt);
    return q_normalize_or_identity(Q4{q.x + d.x, q.y + d.y, q.z + d.z, q.w + d.w});
}
// quat.h:171-185: the rotated basis vectors.
NPH_D V3 axis_x(Q4 q)
{
    return V3{1.0f - 2.0f * (q.y * q.y + q.z * q.z), 2.0f * (q.x * q.y + q.w * q.z),
              2.0f * (q.x * q.z - q.w * q.y)};
}
NPH_D V3 axis_y(Q4 q)
{
    return V3{2.0f * (q.x * q.y - q.w * q.z), 1.0f - 2.0f * (q.x * q.x + q.z * q.z),
              2.0f * (q.y * q.z + q.w * q.x)};
}
NPH_D V3 axis_z(Q4 q)
{
    return V3{2.0f * (q.x * q.z + q.w * q.y), 2.0f * (q.y * q.z - q.w * q.x),
              1.0f - 2.0f * (q.x * q.x + q.y * q.y)};
}
// mat.h:103-107: (c0 v.x + c1 v.y) + c2 v.z.
NPH_D V3 m_mul_v(const M3 &m, V3 v) { return add(add(scale(m.c0, v.x), scale(m.c1, v.y)), scale(m.c2, v.z)); }
NPH_D M3 m_mul(const M3 &a, const M3 &b) { return M3{m_mul_v(a, b.c0), m_mul_v(a, b.c1), m_mul_v(a, b.c2)}; }
NPH_D M3 m_transpose(const M3 &m)
{
    return M3{V3{m.c0.x, m.c1.x, m.c2.x}, V3{m.c0.y, m.c1.y, m.c2.y}, V3{m.c0.z, m.c1.z, m.c2.z}};
}
NPH_D M3 m_zero() { return M3{V3{0.f, 0.f, 0.f}, V3{0.f, 0.f, 0.f}, V3{0.f, 0.f, 0.f}}; }

// vec.h:460-469 (Hughes and Moller): cross with the axis n is least aligned with.
NPH_D V3 perpendicular(V3 n)
{
    const float ax = fabsf(n.x);
    const float ay = fabsf(n.y);
    const float az = fabsf(n.z);
    const V3 axis = (ax <= ay && ax <= az) ? V3{1.0f, 0.0f, 0.0f}
                    : (ay <= az)           ? V3{0.0f, 1.0f, 0.0f}
                                           : V3{0.0f, 0.0f, 1.0f};
    return normalize(cross(n, axis));
}

// A soft constraint's coefficients (PhysSoftness, world_internal.h:258-262).
struct Soft {
    float bias_rate, mass_scale, impulse_scale;
};

// solver.c:48-65.
NPH_D Soft make_soft(float hertz, float zeta, float h)
{
    if (hertz <= 0.0f) {
        return Soft{0.0f, 1.0f, 0.0f};
    }
    const float omega = 2.0f * 3.14159265f * hertz;
    const float a1 = 2.0f * zeta + h * omega;
    const float a2 = h * omega * a1;
    const float a3 = 1.0f / (1.0f + a2);
    return Soft{omega / a1, a2 * a3, a3};
}

} // namespace nph

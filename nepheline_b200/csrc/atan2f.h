// SPDX-License-Identifier: Apache-2.0
//
// The single-precision arctangent the reference's joint rows get from its C library: glibc
// 2.39's atan2f (joint_solver.c:77-84, 303-394 through nph_f32_atan2, scalar.h:239-242),
// restated so the device's joint angles round to the same bits as the reference's.
//
// glibc 2.39 computes atan2f in single precision by fdlibm's method. fdlibm's notice, kept as
// it asks for the method and coefficients restated here:
//
//   Copyright (C) 1993 by Sun Microsystems, Inc. All rights reserved.
//   Developed at SunPro, a Sun Microsystems, Inc. business.
//   Permission to use, copy, modify, and distribute this software is freely granted, provided
//   that this notice is preserved.
//
// The method:
//
//   atan(t), t >= 0: reduce to |u| < 7/16 around a breakpoint b in {0, 1/2, 1, 3/2, inf},
//     atan(t) = atan(b) + atan(u) with u = (t - b) / (1 + b t)  (u = -1/t for b = inf),
//   and evaluate atan(u) = u - u (s1 + s2), the odd series sum_{i=0..10} c_i u^(2i+3) split
//   into even and odd powers of w = u^4; atan(b) is carried as a float head plus a float
//   tail. The head is atan(b) truncated to float and the tail the remainder truncated to
//   float; the c_i are fdlibm's series coefficients rounded to float.
//   atan2(y, x): atan(|y / x|) placed in x and y's quadrant with pi as a head plus a tail.
//
// Every operation is a plain IEEE single-precision one (no contraction, correctly rounded
// division), so the same source gives the same bits compiled by nvcc for the device (with
// -fmad=false -prec-div=true) and by gcc for the host (-ffp-contract=off). Checked against
// the host library on every float through atan (x = 1) and on random pairs.
#pragma once

#if !defined(__cplusplus)
#include <stdbool.h>
#endif
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define NPH_ATAN_FN __host__ __device__ __forceinline__
#else
#define NPH_ATAN_FN static inline
#endif

NPH_ATAN_FN uint32_t nph_atan_bits(float f)
{
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
#endif
}

NPH_ATAN_FN float nph_atan_float(uint32_t u)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

// atan(t) for finite or infinite t of either sign (the sign is carried through).
NPH_ATAN_FN float nph_atanf(float t)
{
    // Breakpoints 1/2, 1, 3/2, inf: atan(b) head (truncated to float) and tail (the rest,
    // truncated to float), as bit patterns.
    const uint32_t head[4] = {0x3eed6338u, 0x3f490fdau, 0x3f7b985eu, 0x3fc90fdau};
    const uint32_t tail[4] = {0x31ac3769u, 0x33222168u, 0x33140fb4u, 0x33a22168u};
    // fdlibm's eleven series coefficients, rounded to float.
    const float c0 = nph_atan_float(0x3eaaaaabu), c1 = nph_atan_float(0xbe4ccccdu);
    const float c2 = nph_atan_float(0x3e124925u), c3 = nph_atan_float(0xbde38e38u);
    const float c4 = nph_atan_float(0x3dba2e6eu), c5 = nph_atan_float(0xbd9d8795u);
    const float c6 = nph_atan_float(0x3d886b35u), c7 = nph_atan_float(0xbd6ef16bu);
    const float c8 = nph_atan_float(0x3d4bda59u), c9 = nph_atan_float(0xbd15a221u);
    const float c10 = nph_atan_float(0x3c8569d7u);

    const uint32_t bits = nph_atan_bits(t);
    const uint32_t mag = bits & 0x7fffffffu;
    const bool negative = (bits >> 31) != 0u;
    if (mag >= 0x4c000000u) { // |t| >= 2^25 (or NaN): atan is pi/2 to float precision
        if (mag > 0x7f800000u) {
            return t + t;
        }
        const float h = nph_atan_float(head[3]) + nph_atan_float(tail[3]);
        return negative ? -h : h;
    }
    int id = -1;
    float u = t;
    if (mag < 0x3ee00000u) { // |t| < 7/16: no reduction
        if (mag < 0x39800000u) { // |t| < 2^-12: atan(t) rounds to t
            return t;
        }
    } else {
        const float a = negative ? -t : t;
        if (mag < 0x3f300000u) { // 7/16 <= |t| < 11/16: b = 1/2
            id = 0;
            u = (2.0f * a - 1.0f) / (2.0f + a);
        } else if (mag < 0x3f980000u) { // 11/16 <= |t| < 19/16: b = 1
            id = 1;
            u = (a - 1.0f) / (a + 1.0f);
        } else if (mag < 0x401c0000u) { // 19/16 <= |t| < 39/16: b = 3/2
            id = 2;
            u = (a - 1.5f) / (1.0f + 1.5f * a);
        } else { // b = inf
            id = 3;
            u = -1.0f / a;
        }
    }
    const float z = u * u;
    const float w = z * z;
    const float s1 = z * (c0 + w * (c2 + w * (c4 + w * (c6 + w * (c8 + w * c10)))));
    const float s2 = w * (c1 + w * (c3 + w * (c5 + w * (c7 + w * c9))));
    if (id < 0) {
        return u - u * (s1 + s2);
    }
    const float r = nph_atan_float(head[id]) - ((u * (s1 + s2) - nph_atan_float(tail[id])) - u);
    return negative ? -r : r;
}

// atan2(y, x) in [-pi, pi], with the special values of C's atan2f.
NPH_ATAN_FN float nph_atan2f(float y, float x)
{
    const float pi = nph_atan_float(0x40490fdbu);      // pi rounded to float
    const float pi_tail = nph_atan_float(0xb3bbbd2eu); // pi minus that, rounded to float
    const float half_pi = nph_atan_float(0x3fc90fdbu);
    const float quarter_pi = nph_atan_float(0x3f490fdbu);
    const uint32_t bx = nph_atan_bits(x), by = nph_atan_bits(y);
    const uint32_t ax = bx & 0x7fffffffu, ay = by & 0x7fffffffu;
    if (ax > 0x7f800000u || ay > 0x7f800000u) {
        return x + y; // NaN
    }
    const bool y_neg = (by >> 31) != 0u;
    const bool x_neg = (bx >> 31) != 0u;
    if (ay == 0u) {
        return x_neg ? (y_neg ? -pi : pi) : y;
    }
    if (ax == 0u) {
        return y_neg ? -half_pi : half_pi;
    }
    if (ax == 0x7f800000u) {
        if (ay == 0x7f800000u) {
            const float q = x_neg ? 3.0f * quarter_pi : quarter_pi;
            return y_neg ? -q : q;
        }
        return x_neg ? (y_neg ? -pi : pi) : (y_neg ? -0.0f : 0.0f);
    }
    if (ay == 0x7f800000u) {
        return y_neg ? -half_pi : half_pi;
    }
    // |y/x| beyond 2^26 is pi/2 to float precision; below 2^-26 with x < 0 the angle is pi.
    const int k = ((int)ay - (int)ax) >> 23;
    float z;
    if (k > 26) {
        z = half_pi + 0.5f * pi_tail;
    } else if (x_neg && k < -26) {
        z = 0.0f;
    } else {
        z = nph_atanf(nph_atan_float(nph_atan_bits(y / x) & 0x7fffffffu)); // |y/x|, -0 to +0
    }
    if (!x_neg) {
        return y_neg ? -z : z;
    }
    return y_neg ? (z - pi_tail) - pi : pi - (z - pi_tail);
}

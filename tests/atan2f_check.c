/* Compares the library's single-precision arctangent (nepheline_b200/csrc/atan2f.h) with the
   host C library's atan2f, the function the reference's joint rows call: every float through
   atan (x = 1) at a stride, special values, and random pairs of several distributions.
   Prints the mismatch count and the first few mismatches. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "atan2f.h"

static uint64_t state = 0x9E3779B97F4A7C15ull;
static uint32_t next_u32(void)
{
    state ^= state << 13;
    state ^= state >> 7;
    state ^= state << 17;
    return (uint32_t)(state >> 16);
}

static long bad = 0;
static void check(float y, float x)
{
    const float want = atan2f(y, x), got = nph_atan2f(y, x);
    if (nph_atan_bits(want) != nph_atan_bits(got) && !(isnan(want) && isnan(got))) {
        if (bad < 8) {
            printf("mismatch y=%a x=%a libm=%a ours=%a\n", y, x, want, got);
        }
        ++bad;
    }
}

int main(int argc, char **argv)
{
    const uint32_t stride = argc > 1 ? (uint32_t)atoi(argv[1]) : 61u;
    const long pairs = argc > 2 ? atol(argv[2]) : 20000000L;
    for (uint64_t u = 0; u <= 0xffffffffull; u += stride) {
        check(nph_atan_float((uint32_t)u), 1.0f);
    }
    const float special[] = {0.0f, -0.0f, 1.0f, -1.0f, INFINITY, -INFINITY, NAN, 1e-45f, -1e-45f,
                             3.4e38f, -3.4e38f, 0.4375f, 0.6875f, 1.1875f, 2.4375f, 33554432.0f,
                             67108864.0f, 2.44140625e-4f};
    const int ns = (int)(sizeof(special) / sizeof(special[0]));
    for (int i = 0; i < ns; ++i) {
        for (int j = 0; j < ns; ++j) {
            check(special[i], special[j]);
        }
    }
    for (long t = 0; t < pairs; ++t) {
        float y, x;
        switch (t % 4) {
        case 0: /* any bit patterns */
            y = nph_atan_float(next_u32());
            x = nph_atan_float(next_u32());
            break;
        case 1: /* the unit square, as the joint rows' sines and cosines */
            y = (float)((int)(next_u32() % 2000001u) - 1000000) * 1e-6f;
            x = (float)((int)(next_u32() % 2000001u) - 1000000) * 1e-6f;
            break;
        case 2: /* magnitudes below 2, either sign */
            y = nph_atan_float(next_u32() & 0xbfffffffu);
            x = nph_atan_float(next_u32() & 0xbfffffffu);
            break;
        default: /* small twists: y tiny against x near 1 */
            x = (float)(next_u32() % 1000001u) * 1e-6f;
            y = ((float)(next_u32() % 2000001u) * 1e-6f - 1.0f) *
                nph_atan_float(0x3a000000u + next_u32() % 0x06000000u);
            break;
        }
        check(y, x);
    }
    printf("mismatches %ld\n", bad);
    return bad != 0;
}

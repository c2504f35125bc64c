// SPDX-License-Identifier: Apache-2.0
//
// The learned warm start's kernels and the residual-driven mode that judges a warm start.
// Neither has a counterpart in the reference: its new contact points start at zero impulse
// (contact.c:547-565). All of them read the rows prepare_manifold wrote for the step:
//   pa (rA, adjusted separation), pb (rB, normal mass), pt (tangent effective-mass inverse,
//   the normal approach speed at the step's start), pi (normal impulse, its maximum, t1 and
//   t2 impulses: the warm start), and the bodies' velocity rows at the step's start.
#pragma once

#include "contacts.cuh"

namespace nph {

struct FeatureConsts {
    float inv_gh;     // 1 / (g h)
    float gh;         // g h
    float gdir[3];    // gravity / |gravity|
};

// A live point slot's kind: a point with a persisted impulse, or a cold point.
NPH_D uint32_t point_kind(const float4 &im)
{
    return (im.x == 0.0f && im.z == 0.0f && im.w == 0.0f) ? NPH_GPU_POINT_COLD : NPH_GPU_POINT_WARM;
}

// The 16 features of manifold g's point k (layout in nepheline_b200.h) and the impulse scale
// g h / kn a network output of 1 stands for.
NPH_D void point_features(const DevSolver &S, uint32_t g, uint32_t k, uint4 hdr, const FeatureConsts &F,
                          float f[NPH_GPU_MLP_INPUTS], float &scale)
{
    const uint32_t bits = hdr.z;
    const uint32_t row = k * S.mcap + g;
    const float4 A = S.pa[row];
    const float4 B = S.pb[row];
    const float4 T = S.pt[row];
    const float4 nf = S.nrm[g];
    const V3 n = v3(nf);
    const V3 t1 = perpendicular(n);
    const V3 t2 = cross(n, t1);
    const V3 ra = v3(A), rb = v3(B);
    const bool dyn_a = (bits & kHdrWriteA) != 0u;
    const bool dyn_b = (bits & kHdrWriteB) != 0u;
    float ma = 0.0f, mb = 0.0f;
    const M3 ia = dyn_a ? load_inv_inertia(S.prm, hdr.x, &ma) : m_zero();
    const M3 ib = dyn_b ? load_inv_inertia(S.prm, hdr.y, &mb) : m_zero();
    ma = dyn_a ? ma : 0.0f;
    mb = dyn_b ? mb : 0.0f;
    const V3 rxa = cross(ra, n), rxb = cross(rb, n);
    const float ang_a = dot(rxa, m_mul_v(ia, rxa));
    const float ang_b = dot(rxb, m_mul_v(ib, rxb));
    const float kn = B.w > 0.0f ? 1.0f / B.w : 0.0f;
    const float inv_kn = B.w; // the normal mass
    const BodyState a = load_state(S.vel, hdr.x);
    const BodyState b = load_state(S.vel, hdr.y);
    const V3 dv = rel_vel(a, b, ra, rb);
    const float sep = A.w + dot(sub(rb, ra), n);
    f[0] = T.w * F.inv_gh;
    f[1] = dot(dv, t1) * F.inv_gh;
    f[2] = dot(dv, t2) * F.inv_gh;
    f[3] = n.x;
    f[4] = n.y;
    f[5] = n.z;
    f[6] = sep * 50.0f;
    f[7] = ma * inv_kn;
    f[8] = mb * inv_kn;
    f[9] = ang_a * inv_kn;
    f[10] = ang_b * inv_kn;
    f[11] = (float)(bits & kHdrPointsMask) * 0.25f;
    f[12] = nf.w;
    f[13] = -(n.x * F.gdir[0] + n.y * F.gdir[1] + n.z * F.gdir[2]);
    f[14] = (dyn_a && dyn_b) ? 0.0f : 1.0f;
    f[15] = T.x * kn;
    scale = F.gh * inv_kn;
}

// Every point slot's features, scale and kind (the training-data path).
__global__ void __launch_bounds__(256) k_all_features(DevSolver S, uint32_t m, FeatureConsts F, float *feat,
                                                      float *scale, uint32_t *kind)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= m) {
        return;
    }
    const uint4 hdr = S.hdr[g];
    const uint32_t pc = hdr.z & kHdrPointsMask;
    for (uint32_t k = 0; k < 4u; ++k) {
        const size_t slot = 4ull * g + k;
        float f[NPH_GPU_MLP_INPUTS];
        float sc = 0.0f;
        uint32_t kd = NPH_GPU_POINT_NONE;
        if (k < pc) {
            point_features(S, g, k, hdr, F, f, sc);
            kd = point_kind(S.pi[k * S.mcap + g]);
        } else {
#pragma unroll
            for (int i = 0; i < NPH_GPU_MLP_INPUTS; ++i) {
                f[i] = 0.0f;
            }
        }
        float4 *dst = reinterpret_cast<float4 *>(feat + slot * NPH_GPU_MLP_INPUTS);
#pragma unroll
        for (int i = 0; i < NPH_GPU_MLP_INPUTS / 4; ++i) {
            dst[i] = make_float4(f[4 * i], f[4 * i + 1], f[4 * i + 2], f[4 * i + 3]);
        }
        scale[slot] = sc;
        kind[slot] = kd;
    }
}

// The cold points' features, compacted (in any order: each prediction depends on its own row
// only); counts[0] the cold points, counts[1] those given a row (at most `cap`).
__global__ void __launch_bounds__(256) k_cold_features(DevSolver S, uint32_t m, FeatureConsts F, float *feat,
                                                       float *scale, uint32_t *slot, uint32_t *counts,
                                                       uint32_t cap, uint32_t write)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= m) {
        return;
    }
    const uint4 hdr = S.hdr[g];
    const uint32_t pc = hdr.z & kHdrPointsMask;
    for (uint32_t k = 0; k < pc; ++k) {
        if (point_kind(S.pi[k * S.mcap + g]) != NPH_GPU_POINT_COLD) {
            continue;
        }
        atomicAdd(&counts[0], 1u);
        if (write == 0u) {
            continue;
        }
        const uint32_t i = atomicAdd(&counts[1], 1u);
        if (i >= cap) {
            continue;
        }
        float f[NPH_GPU_MLP_INPUTS];
        float sc;
        point_features(S, g, k, hdr, F, f, sc);
        float4 *dst = reinterpret_cast<float4 *>(feat + (size_t)i * NPH_GPU_MLP_INPUTS);
#pragma unroll
        for (int q = 0; q < NPH_GPU_MLP_INPUTS / 4; ++q) {
            dst[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
        }
        scale[i] = sc;
        slot[i] = 4u * g + k;
    }
}

// The predictions as warm-start impulses of their cold points: normal max(y0, 0) x scale,
// friction (y1, y2) x scale along t1, t2, scaled back onto the friction cone when outside it.
__global__ void __launch_bounds__(256) k_apply_predictions(DevSolver S, const float *pred, const float *scale,
                                                           const uint32_t *slot, const uint32_t *counts,
                                                           uint32_t cap)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t count = min(counts[1], cap);
    if (i >= count) {
        return;
    }
    const uint32_t g = slot[i] >> 2, k = slot[i] & 3u;
    const float sc = scale[i];
    const float ln = fmaxf(pred[3 * i], 0.0f) * sc;
    float l1 = pred[3 * i + 1] * sc;
    float l2 = pred[3 * i + 2] * sc;
    const float limit = S.nrm[g].w * ln;
    const float len = sqrtf(l1 * l1 + l2 * l2);
    if (len > limit) {
        const float r = len > 0.0f ? limit / len : 0.0f;
        l1 *= r;
        l2 *= r;
    }
    S.pi[k * S.mcap + g] = make_float4(ln, 0.0f, l1, l2);
}

// ---- the residual-driven mode -----------------------------------------------------

// A rigid pass (the relax pass) over one colour, skipped once the residual reached the
// tolerance.
template <int kThreads>
__global__ void __launch_bounds__(kThreads) k_converge_pass(DevSolver S, uint32_t cfirst, uint32_t ccount,
                                                            StepConsts K, const uint32_t *done)
{
    if (*done != 0u) {
        return;
    }
    const uint32_t g = blockIdx.x * kThreads + threadIdx.x;
    if (g < ccount) {
        solve_manifold<false>(S, cfirst + g, K);
    }
}

__global__ void __launch_bounds__(256) k_converge_joint_pass(DevSolver S, uint32_t jfirst, uint32_t jcount,
                                                             StepConsts K, const uint32_t *done)
{
    if (*done != 0u) {
        return;
    }
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < jcount) {
        solve_joint<false>(S, jfirst + j, K);
    }
}

__global__ void k_converge_overflow(DevSolver S, uint32_t cfirst, uint32_t ccount, uint32_t jfirst,
                                    uint32_t jcount, StepConsts K, const uint32_t *done)
{
    if (*done != 0u || threadIdx.x != 0 || blockIdx.x != 0) {
        return;
    }
    for (uint32_t j = 0; j < jcount; ++j) {
        solve_joint<false>(S, jfirst + j, K);
    }
    for (uint32_t g = 0; g < ccount; ++g) {
        solve_manifold<false>(S, cfirst + g, K);
    }
}

// The squared residual of manifold g's points (the rigid rows the relax pass solves).
NPH_D float manifold_residual_sq(const DevSolver &S, uint32_t g, float inv_h)
{
    const uint4 hdr = S.hdr[g];
    const uint32_t pc = hdr.z & kHdrPointsMask;
    if (pc == 0u) {
        return 0.0f;
    }
    const float4 nf = S.nrm[g];
    const V3 n = v3(nf);
    const V3 t1 = perpendicular(n);
    const V3 t2 = cross(n, t1);
    const BodyState a = load_state(S.vel, hdr.x);
    const BodyState b = load_state(S.vel, hdr.y);
    const BodyPose pa_ = load_pose(S.pos, hdr.x);
    const BodyPose pb_ = load_pose(S.pos, hdr.y);
    float sum = 0.0f;
    for (uint32_t k = 0; k < pc; ++k) {
        const uint32_t row = k * S.mcap + g;
        const float4 A = S.pa[row];
        const float4 B = S.pb[row];
        const float4 im = S.pi[row];
        const V3 ra = v3(A), rb = v3(B);
        const float s = separation(pa_, pb_, ra, rb, A.w, n);
        const V3 dv = rel_vel(a, b, ra, rb);
        const float vn = dot(dv, n) + (s > 0.0f ? s * inv_h : 0.0f);
        const float rn = im.x > 0.0f ? fabsf(vn) : fmaxf(-vn, 0.0f);
        float rt = 0.0f;
        const float lim = nf.w * im.x;
        if (sqrtf(im.z * im.z + im.w * im.w) < lim * 0.999f) {
            const float v1 = dot(dv, t1), v2 = dot(dv, t2);
            rt = v1 * v1 + v2 * v2;
        }
        sum += rn * rn + rt;
    }
    return sum;
}

// The residual's square: each block's sum over its manifolds into partials[blockIdx.x].
constexpr uint32_t kResidualBlocks = 148u * 8u; // the most blocks a residual launch has
__global__ void __launch_bounds__(256) k_residual(DevSolver S, uint32_t m, float inv_h, float *partials,
                                                  const uint32_t *done)
{
    if (*done != 0u) {
        return;
    }
    __shared__ float part[8];
    float sum = 0.0f;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < m; g += gridDim.x * blockDim.x) {
        sum += manifold_residual_sq(S, g, inv_h);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
    }
    if ((threadIdx.x & 31u) == 0u) {
        part[threadIdx.x >> 5] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (uint32_t w = 0; w < blockDim.x / 32u; ++w) {
            t += part[w];
        }
        partials[blockIdx.x] = t;
    }
}

// After pass p (0: the warm start), one block of 256 threads: the blocks' partial sums added
// in a fixed order (so a run's residuals are the same bits every time), the residual, the
// reference residual at p = 0, and the stop test. state[0] done, state[1] the passes run.
__global__ void __launch_bounds__(256) k_residual_check(const float *partials, uint32_t nparts, float *res_sq,
                                                        float *residuals, float *ref, uint32_t p,
                                                        float tolerance, float ref_in, uint32_t *state)
{
    if (state[0] != 0u) { // read by every thread before any thread writes it
        return;
    }
    __shared__ float sh[256];
    float v = 0.0f;
    for (uint32_t i = threadIdx.x; i < nparts; i += 256u) {
        v += partials[i];
    }
    sh[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t half = 128u; half > 0u; half >>= 1) {
        if (threadIdx.x < half) {
            sh[threadIdx.x] += sh[threadIdx.x + half];
        }
        __syncthreads();
    }
    if (threadIdx.x != 0u) {
        return;
    }
    res_sq[p] = sh[0];
    const float r = sqrtf(sh[0]);
    residuals[p] = r;
    if (p == 0u) {
        ref[0] = ref_in > 0.0f ? ref_in : r;
    }
    state[1] = p;
    if (r <= tolerance * ref[0]) {
        state[0] = 1u;
    }
}

// Every point slot's impulses in the contact frame (normal, t1, t2).
__global__ void __launch_bounds__(256) k_slot_impulses(DevSolver S, uint32_t m, float *out)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= m) {
        return;
    }
    const uint32_t pc = S.hdr[g].z & kHdrPointsMask;
    for (uint32_t k = 0; k < 4u; ++k) {
        float4 im = make_float4(0.f, 0.f, 0.f, 0.f);
        if (k < pc) {
            im = S.pi[k * S.mcap + g];
        }
        float *o = out + 12ull * g + 3ull * k;
        o[0] = im.x;
        o[1] = im.z;
        o[2] = im.w;
    }
}

} // namespace nph

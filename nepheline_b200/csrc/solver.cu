// SPDX-License-Identifier: Apache-2.0
//
// The solver stage on the device for one world of any size: the reference's stage list
// (phys_solve, engine/physics/src/solver.c:961-1105) as kernels, one launch per stage and
// colour, replayed as one CUDA graph per step:
//
//   prepare bodies; prepare joints and contacts;
//   per substep: integrate velocities, warm start, solve, integrate positions, relax
//     (each constraint pass: the overflow serially in list order, then colours 0..23, each
//      colour's joints and contacts in one launch: push_contact_pass, solver.c:774-789);
//   restitution (contacts only); store; finalize; the driven joints' sleep reset.
//
// The reference's lockstep thread claiming (solver.c:628-713) becomes kernel boundaries:
// every stage's writes are visible to the next launch on the stream.

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <vector>

#include "nepheline_b200.h"
#include "solver_link.h"

#include "bodies.cuh"
#include "contacts.cuh"
#include "contacts_pair.cuh"
#include "contacts_staged.cuh"
#include "joints.cuh"
#include "learned.cuh"
#include "warm_match.h"

// The network's inference (mlp.cu): `count` rows, or the first *count_dev of at most
// max_count rows.
void nph_mlp_forward_device(const NphGpuMlp *n, const float *x, uint32_t count, float *y, cudaStream_t st);
void nph_mlp_forward_device_count(const NphGpuMlp *n, const float *x, const uint32_t *count_dev,
                                  uint32_t max_count, float *y, cudaStream_t st);
int nph_mlp_device(const NphGpuMlp *n);

namespace nph {

constexpr uint32_t kBlock = 256;

struct ColorTable {
    uint32_t cfirst[NPH_GPU_COLOR_SLOTS];
    uint32_t ccount[NPH_GPU_COLOR_SLOTS];
};

enum Pass : int { kWarm = 0, kSolve = 1, kRelax = 2, kRestitution = 3 };

// ------------------------------------------------------------------------------------
// Kernels
// ------------------------------------------------------------------------------------

// Record staging: a block copies its records between global and shared memory with 16- or
// 8-byte accesses covering whole cache lines, and the threads work on the shared copies.
constexpr uint32_t kStage = 128;

template <typename V, typename Rec>
__device__ __forceinline__ void stage_in(const Rec *src, uint32_t count, Rec *dst)
{
    const V *s = reinterpret_cast<const V *>(src);
    V *d = reinterpret_cast<V *>(dst);
    const uint32_t words = (uint32_t)(count * sizeof(Rec) / sizeof(V));
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
        d[i] = s[i];
    }
}

template <typename V, typename Rec>
__device__ __forceinline__ void stage_out(const Rec *src, uint32_t count, Rec *dst)
{
    const V *s = reinterpret_cast<const V *>(src);
    V *d = reinterpret_cast<V *>(dst);
    const uint32_t words = (uint32_t)(count * sizeof(Rec) / sizeof(V));
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
        d[i] = s[i];
    }
}

static_assert(sizeof(NphGpuBody) % 16 == 0, "body records stage in 16-byte words");
static_assert(sizeof(NphGpuContact) % 16 == 0, "contact records stage in 16-byte words");

// Whether every value of a body record that the stage reads is finite: the centre, the rotation,
// the velocities, force and torque, the mass properties and the integration settings.
__device__ bool body_finite(const NphGpuBody &b)
{
    bool ok = isfinite(b.center[0]) && isfinite(b.center[1]) && isfinite(b.center[2]);
    const float *f = b.rotation; // rotation .. max_extent: 44 consecutive floats
    static_assert(offsetof(NphGpuBody, type) - offsetof(NphGpuBody, rotation) == 44 * sizeof(float),
                  "the record's float block");
#pragma unroll 4
    for (uint32_t k = 0; k < 44u; ++k) {
        ok = ok && isfinite(f[k]);
    }
    return ok;
}

__global__ void __launch_bounds__(kStage) k_prepare_bodies(BodyArrays B, const NphGpuBody *bodies,
                                                           uint32_t n, StepConsts K, uint32_t *err)
{
    __shared__ NphGpuBody rec[kStage];
    const uint32_t first = blockIdx.x * kStage;
    if (first < n) {
        const uint32_t count = min(kStage, n - first);
        stage_in<uint4>(bodies + first, count, rec);
        __syncthreads();
        if (threadIdx.x < count) {
            if (body_finite(rec[threadIdx.x])) {
                prepare_body(B, first + threadIdx.x, rec[threadIdx.x], K);
            } else {
                // Refused: the call returns before anything is written back. Meanwhile the body
                // is inert (a static body at rest), so nothing it touches takes a non-finite value.
                atomicOr(err, kErrBadBody);
                NphGpuBody inert = rec[threadIdx.x];
                inert.type = NPH_GPU_BODY_STATIC;
                for (uint32_t k = 0; k < 3u; ++k) {
                    inert.linear_velocity[k] = 0.0f;
                    inert.angular_velocity[k] = 0.0f;
                }
                inert.rotation[0] = inert.rotation[1] = inert.rotation[2] = 0.0f;
                inert.rotation[3] = 1.0f;
                prepare_body(B, first + threadIdx.x, inert, K);
            }
        }
    }
    if (first + threadIdx.x == n) {
        prepare_dummy(B, n);
    }
}

// The largest point count of the eight-lane group holding manifold g (build_groups,
// solver.c:810-843: a colour's list in eights, the overflow one per group), and g's colour.
__device__ uint32_t group_points(const NphGpuContact *contacts, const NphGpuContact *staged,
                                 uint32_t first, uint32_t count, uint32_t g, const ColorTable &T,
                                 uint32_t &color)
{
    uint32_t c = 0;
    while (c + 1u < NPH_GPU_COLOR_SLOTS && g >= T.cfirst[c] + T.ccount[c]) {
        ++c;
    }
    const uint32_t per = c == NPH_GPU_OVERFLOW ? 1u : 8u;
    const uint32_t start = T.cfirst[c] + ((g - T.cfirst[c]) / per) * per;
    const uint32_t end = min(start + per, T.cfirst[c] + T.ccount[c]);
    uint32_t gp = 0;
    for (uint32_t q = start; q < end; ++q) {
        const uint32_t pc = q >= first && q < first + count ? staged[q - first].point_count
                                                            : contacts[q].point_count;
        gp = pc <= NPH_GPU_MAX_POINTS && pc > gp ? pc : gp;
    }
    color = c;
    return gp;
}

// Whether a view index is a dynamic body, and its inverse mass (zero unless dynamic).
__device__ __forceinline__ void body_kind(const float4 *prm, const NphGpuBody *fixed, uint32_t n,
                                          uint32_t index, bool &dyn, float &inv_mass)
{
    if (index < n) {
        dyn = prm[3u * index + 1u].w != 0.0f;
        inv_mass = prm[3u * index].w;
    } else {
        const NphGpuBody &f = fixed[index - n];
        dyn = f.type == NPH_GPU_BODY_DYNAMIC;
        inv_mass = dyn ? f.inv_mass : 0.0f;
    }
}

__global__ void __launch_bounds__(kStage)
k_prepare_contacts(DevSolver S, const NphGpuContact *contacts, const NphGpuBody *fixed, uint32_t n,
                   uint32_t nf, uint32_t m, ColorTable T, uint32_t *err, uint32_t *color_points)
{
    __shared__ NphGpuContact rec[kStage];
    __shared__ uint32_t points[NPH_GPU_COLOR_SLOTS];
    const uint32_t first = blockIdx.x * kStage;
    const uint32_t count = min(kStage, m - first);
    if (threadIdx.x < NPH_GPU_COLOR_SLOTS) {
        points[threadIdx.x] = 0u;
    }
    stage_in<uint4>(contacts + first, count, rec);
    __syncthreads();
    const uint32_t g = first + threadIdx.x;
    const uint32_t total = n + nf;
    if (threadIdx.x < count) {
        const NphGpuContact &c = rec[threadIdx.x];
        if (c.body_a >= total || c.body_b >= total) {
            atomicOr(err, kErrBadIndex);
            S.hdr[g] = make_uint4(n, n, 0u, 0u);
        } else if (c.point_count < 1u || c.point_count > NPH_GPU_MAX_POINTS) {
            atomicOr(err, kErrBadPoints);
            S.hdr[g] = make_uint4(n, n, 0u, 0u);
        } else {
            bool dyn_a, dyn_b;
            float ma, mb;
            body_kind(S.prm, fixed, n, c.body_a, dyn_a, ma);
            body_kind(S.prm, fixed, n, c.body_b, dyn_b, mb);
            S.nrm[g] = make_float4(c.normal[0], c.normal[1], c.normal[2], c.friction);
            S.rest[g] = c.restitution;
            uint32_t color = 0;
            const uint32_t gp = group_points(contacts, rec, first, count, g, T, color);
            prepare_manifold(S, g, c, c.body_a < n ? c.body_a : n, c.body_b < n ? c.body_b : n,
                             dyn_a, dyn_b, ma, mb, gp);
            atomicAdd(&points[color], c.point_count);
        }
    }
    // The points per colour (the byte counts of a profiled step): one global add per block.
    __syncthreads();
    if (threadIdx.x < NPH_GPU_COLOR_SLOTS && points[threadIdx.x] != 0u) {
        atomicAdd(&color_points[threadIdx.x], points[threadIdx.x]);
    }
}

__global__ void __launch_bounds__(kBlock)
k_prepare_joints(DevSolver S, const NphGpuJoint *joints, const NphGpuBody *bodies,
                 const NphGpuBody *fixed, uint32_t n, uint32_t nf, uint32_t nj, float h, uint32_t *err)
{
    // Each joint reads only what its type uses of its record (a ball or hinge joint about
    // half of it), straight from global memory: the sectors it touches are its own.
    const uint32_t j = blockIdx.x * kBlock + threadIdx.x;
    if (j >= nj) {
        return;
    }
    const uint32_t total = n + nf;
    const NphGpuJoint &jr = joints[j];
    if (jr.body_a >= total || jr.body_b >= total || nph_joint_check(&jr) != NPH_GPU_OK) {
        atomicOr(err, kErrBadJoint);
        // Inert: both ends the dummy, no impulse, nothing written.
        for (uint32_t r = 0; r < kJointRows; ++r) {
            S.jw[r * S.jcap + j] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        S.jw[kJrFrameA * S.jcap + j] = make_float4(0.f, 0.f, 0.f, 1.f);
        S.jw[kJrFrameB * S.jcap + j] = make_float4(0.f, 0.f, 0.f, 1.f);
        S.jw[kJrHead * S.jcap + j] = make_float4(__uint_as_float(n), __uint_as_float(n), 0.f, 0.f);
        return;
    }
    const NphGpuBody &a = jr.body_a < n ? bodies[jr.body_a] : fixed[jr.body_a - n];
    const NphGpuBody &b = jr.body_b < n ? bodies[jr.body_b] : fixed[jr.body_b - n];
    prepare_joint(S, j, jr, a, b, jr.body_a < n ? jr.body_a : n, jr.body_b < n ? jr.body_b : n, h);
}

template <int P, int kSet>
__device__ __forceinline__ void joint_set_op(const DevSolver &S, uint32_t j, const StepConsts &K)
{
    if (P == kWarm) {
        warm_joint<kSet>(S, j);
    } else if (P == kSolve) {
        solve_joint<true, kSet>(S, j, K);
    } else if (P == kRelax) {
        solve_joint<false, kSet>(S, j, K);
    }
}

template <int P>
__device__ __forceinline__ void joint_op(const DevSolver &S, uint32_t j, const StepConsts &K)
{
    joint_set_op<P, kJointsAll>(S, j, K);
}

template <int P>
__device__ __forceinline__ void contact_op(const DevSolver &S, uint32_t g, const StepConsts &K)
{
    if (P == kWarm) {
        warm_manifold(S, g);
    } else if (P == kSolve) {
        solve_manifold<true>(S, g, K);
    } else if (P == kRelax) {
        solve_manifold<false>(S, g, K);
    } else {
        restitution_manifold(S, g, K);
    }
}

// One colour of one constraint pass: its joints' blocks, then its contacts'. Instantiated
// for several block sizes and register budgets (the pass configurations the autotuner picks
// from).
template <int P, int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
k_pass(DevSolver S, uint32_t cfirst, uint32_t ccount, StepConsts K)
{
    const uint32_t g = blockIdx.x * kThreads + threadIdx.x;
    if (g < ccount) {
        contact_op<P>(S, cfirst + g, K);
    }
}

// One colour's joints in one constraint pass. A colour's joints share no dynamic body with its
// contacts, so the two kernels run side by side.
template <int P, int kSet>
__global__ void __launch_bounds__(kBlock) k_joint_pass(DevSolver S, uint32_t jfirst, uint32_t jcount,
                                                       StepConsts K)
{
    const uint32_t j = blockIdx.x * kBlock + threadIdx.x;
    if (j < jcount) {
        joint_set_op<P, kSet>(S, jfirst + j, K);
    }
}

// The same pass with the manifold's loads staged through shared memory (contacts_staged.cuh);
// kBodies false: the lean form, only the point rows staged.
template <int P, uint32_t kLanes, int kMinBlocks, bool kBodies = true>
__global__ void __launch_bounds__(kLanes, kMinBlocks)
k_pass_staged(DevSolver S, uint32_t cfirst, uint32_t ccount, StepConsts K)
{
    extern __shared__ float4 tile[];
    const uint32_t g = blockIdx.x * kLanes + threadIdx.x;
    if (g >= ccount) {
        return;
    }
    const Tile<kLanes> T{tile, threadIdx.x};
    if (P == kWarm) {
        warm_manifold_staged<kLanes, false, kBodies>(S, cfirst + g, T);
    } else if (P == kSolve) {
        solve_manifold_staged<true, kLanes, false, kBodies>(S, cfirst + g, K, T);
    } else if (P == kRelax) {
        solve_manifold_staged<false, kLanes, false, kBodies>(S, cfirst + g, K, T);
    } else {
        restitution_manifold(S, cfirst + g, K);
    }
}

// The warm start with two lanes a manifold (contacts_pair.cuh): lanes 2i and 2i + 1 of the
// grid take manifold i, bodies A and B.
template <int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_warm_pair(DevSolver S, uint32_t cfirst, uint32_t ccount)
{
    const uint32_t g = (blockIdx.x * kThreads + threadIdx.x) >> 1;
    if (g >= ccount) {
        return;
    }
    const uint32_t lane = threadIdx.x & 31u;
    warm_manifold_pair(S, cfirst + g, Pair{3u << (lane & ~1u), (lane & 1u) != 0u});
}

// The contact update for the next step (contact.c:516-565): each contact's record becomes the
// narrow phase's manifold with its pair, flags and warm-started impulses from the record the
// last step stored.
__global__ void __launch_bounds__(128) k_warm_update(NphGpuContact *contacts, const NphGpuContact *fresh,
                                                     uint32_t m)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= m) {
        return;
    }
    NphGpuContact out;
    nph_warm_update(&contacts[g], &fresh[g], &out);
    contacts[g] = out;
}

// The staged pass, pipelined: a persistent grid whose blocks walk the colour's manifolds in
// chunks of one per lane, issuing the next chunk's loads into a second tile before computing
// the current one, so a warp's loads overlap its arithmetic. A colour's manifolds share no
// dynamic body, so loads issued ahead read what no other manifold of the colour writes, and
// each lane reads and writes only its own column of the tiles.
template <int P, uint32_t kLanes, int kMinBlocks>
__global__ void __launch_bounds__(kLanes, kMinBlocks)
k_pass_pipelined(DevSolver S, uint32_t cfirst, uint32_t ccount, StepConsts K)
{
    extern __shared__ float4 tiles[];
    const uint32_t lane = threadIdx.x;
    const uint32_t chunks = (ccount + kLanes - 1u) / kLanes;
    const Tile<kLanes> T[2] = {Tile<kLanes>{tiles, lane}, Tile<kLanes>{tiles + kSlots * kLanes, lane}};
    const bool tangents = P != kWarm;
    const bool poses = P != kWarm;
    auto header = [&](uint32_t chunk) -> uint4 {
        const uint32_t g = chunk * kLanes + lane;
        return chunk < chunks && g < ccount ? S.hdr[cfirst + g] : make_uint4(0u, 0u, 0u, 0u);
    };
    auto issue = [&](uint32_t chunk, uint4 hdr, uint32_t t) {
        if ((hdr.z & kHdrPointsMask) != 0u) {
            issue_manifold(S, cfirst + chunk * kLanes + lane, hdr, T[t], tangents, poses);
        }
        __pipeline_commit();
    };
    uint32_t c = blockIdx.x;
    issue(c, header(c), 0u);
    uint4 hdr_next = header(c + gridDim.x);
    for (uint32_t i = 0; c < chunks; ++i, c += gridDim.x) {
        const uint32_t next = c + gridDim.x;
        issue(next, hdr_next, (i + 1u) & 1u);
        hdr_next = header(next + gridDim.x);
        __pipeline_wait_prior(1); // this chunk's copies are in
        const uint32_t g = c * kLanes + lane;
        if (g < ccount) {
            if (P == kWarm) {
                warm_manifold_staged<kLanes, true>(S, cfirst + g, T[i & 1u]);
            } else {
                solve_manifold_staged<P == kSolve, kLanes, true>(S, cfirst + g, K, T[i & 1u]);
            }
        }
    }
    __pipeline_wait_prior(0);
}

// The pass configurations: threads per block and the blocks per SM the register budget
// allows (65,536 registers / (threads x blocks)); `staged`: 0 plain loads, 1 the loads staged
// through shared memory (kSlots x threads x 16 bytes per block), 2 staged and pipelined, 3 the
// lean staged form (kPointSlots x threads x 16 bytes per block), 4 two lanes a manifold for
// the warm start (contacts_pair.cuh; the other pass kinds run the plain kernel), 5 the whole
// pass in one dependency-driven launch of one-warp blocks (k_pass_flow: the warm start's
// contacts plain, the solve and relax passes' lean staged; restitution runs the plain kernel).
struct PassConfig {
    uint32_t threads, min_blocks, staged;
};
constexpr PassConfig kPassConfigs[] = {{256, 1, 0}, {256, 2, 0}, {128, 4, 0}, {256, 3, 0},
                                       {64, 6, 1},  {64, 7, 1},  {128, 3, 1}, {32, 14, 1},
                                       {32, 7, 2},  {64, 3, 2},  {32, 18, 3}, {32, 24, 3},
                                       {64, 9, 3},  {64, 12, 3}, {128, 6, 3}, {128, 6, 4},
                                       {128, 8, 4}, {64, 14, 4}, {256, 4, 4},  {32, 18, 5},
                                       {32, 16, 5}, {32, 20, 5}};
constexpr uint32_t kPassConfigCount = sizeof(kPassConfigs) / sizeof(kPassConfigs[0]);

template <int P>
void launch_pass(uint32_t config, uint32_t cc, cudaStream_t st, const DevSolver &S, uint32_t cfirst,
                 const StepConsts &K)
{
    const uint32_t t = kPassConfigs[config].threads;
    const uint32_t grid = (cc + t - 1) / t;
    if (kPassConfigs[config].staged == 5u) { // a colour at a time: the plain kernel
        k_pass<P, 128, 4><<<(cc + 127u) / 128u, 128, 0, st>>>(S, cfirst, cc, K);
        return;
    }
    if (kPassConfigs[config].staged == 4u) {
        if (P == kWarm) {
            const uint32_t pair_grid = (2u * cc + t - 1) / t;
            switch (config) {
            case 15: k_warm_pair<128, 6><<<pair_grid, 128, 0, st>>>(S, cfirst, cc); break;
            case 16: k_warm_pair<128, 8><<<pair_grid, 128, 0, st>>>(S, cfirst, cc); break;
            case 17: k_warm_pair<64, 14><<<pair_grid, 64, 0, st>>>(S, cfirst, cc); break;
            default: k_warm_pair<256, 4><<<pair_grid, 256, 0, st>>>(S, cfirst, cc); break;
            }
        } else {
            k_pass<P, 128, 4><<<(cc + 127u) / 128u, 128, 0, st>>>(S, cfirst, cc, K);
        }
        return;
    }
    const uint32_t slots = kPassConfigs[config].staged == 3u ? kPointSlots : kSlots;
    const size_t tile = kPassConfigs[config].staged ? (size_t)slots * t * sizeof(float4) : 0;
    if (kPassConfigs[config].staged == 2u) {
        if (P == kRestitution) { // no loads worth pipelining: the plain kernel
            k_pass<P, 128, 4><<<(cc + 127u) / 128u, 128, 0, st>>>(S, cfirst, cc, K);
            return;
        }
        // A persistent grid: the SMs times the blocks each holds.
        static const uint32_t sms = [] {
            int dev = 0, n = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
            return (uint32_t)n;
        }();
        const uint32_t blocks = std::max<uint32_t>(1u, std::min<uint32_t>(grid, sms * kPassConfigs[config].min_blocks));
        if (config == 8) {
            k_pass_pipelined<P, 32, 7><<<blocks, 32, 2 * tile, st>>>(S, cfirst, cc, K);
        } else {
            k_pass_pipelined<P, 64, 3><<<blocks, 64, 2 * tile, st>>>(S, cfirst, cc, K);
        }
        return;
    }
    switch (config) {
    case 0: k_pass<P, 256, 1><<<grid, 256, 0, st>>>(S, cfirst, cc, K); break;
    case 1: k_pass<P, 256, 2><<<grid, 256, 0, st>>>(S, cfirst, cc, K); break;
    case 2: k_pass<P, 128, 4><<<grid, 128, 0, st>>>(S, cfirst, cc, K); break;
    case 3: k_pass<P, 256, 3><<<grid, 256, 0, st>>>(S, cfirst, cc, K); break;
    case 4: k_pass_staged<P, 64, 6><<<grid, 64, tile, st>>>(S, cfirst, cc, K); break;
    case 5: k_pass_staged<P, 64, 7><<<grid, 64, tile, st>>>(S, cfirst, cc, K); break;
    case 6: k_pass_staged<P, 128, 3><<<grid, 128, tile, st>>>(S, cfirst, cc, K); break;
    case 7: k_pass_staged<P, 32, 14><<<grid, 32, tile, st>>>(S, cfirst, cc, K); break;
    case 10: k_pass_staged<P, 32, 18, false><<<grid, 32, tile, st>>>(S, cfirst, cc, K); break;
    case 11: k_pass_staged<P, 32, 24, false><<<grid, 32, tile, st>>>(S, cfirst, cc, K); break;
    case 12: k_pass_staged<P, 64, 9, false><<<grid, 64, tile, st>>>(S, cfirst, cc, K); break;
    case 13: k_pass_staged<P, 64, 12, false><<<grid, 64, tile, st>>>(S, cfirst, cc, K); break;
    default: k_pass_staged<P, 128, 6, false><<<grid, 128, tile, st>>>(S, cfirst, cc, K); break;
    }
}

// The staged kernels with tiles above the default 48 KiB of dynamic shared memory.
template <int P> void allow_tiles()
{
    cudaFuncSetAttribute(k_pass_staged<P, 128, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kSlots * 128 * sizeof(float4)));
    if (P != kRestitution) {
        cudaFuncSetAttribute(k_pass_pipelined<P, 64, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * kSlots * 64 * sizeof(float4)));
    }
}

// The overflow: its joints, then its contacts, one at a time in list order (they may share
// bodies; solver.c:778-782 runs them as one block each).
template <int P>
__global__ void k_overflow(DevSolver S, uint32_t cfirst, uint32_t ccount, uint32_t jfirst,
                           uint32_t jcount, StepConsts K)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) {
        return;
    }
    if (P != kRestitution) {
        for (uint32_t j = 0; j < jcount; ++j) {
            joint_op<P>(S, jfirst + j, K);
        }
    }
    for (uint32_t g = 0; g < ccount; ++g) {
        contact_op<P>(S, cfirst + g, K);
    }
}

// ---------------------------------------------------------------------------------------
// Dependency-driven passes
// ---------------------------------------------------------------------------------------
//
// One launch runs a whole warm start, solve or relax pass over every colour, in place of a
// launch per colour (whose start and tail leave SMs idle, and whose last colours hold a few
// constraints each). Warps take tickets in order; a ticket is 32 consecutive constraints of one
// kind (joints or contacts) of one colour, the ranges in colour order, a colour's joints before
// its contacts. A constraint of colour c waits until, on each body it writes, every constraint
// of an earlier colour that writes the body has finished this pass. A body has at most one
// constraint of each colour (the colouring's rule), so that count, the constraint's rank on the
// body, is the number of earlier colours in the body's colour mask; prepare stores the ranks
// (k_colour_ranks). Each finished constraint adds one to the counters of the bodies it wrote,
// with release semantics after its velocity stores; a waiting constraint reads them with
// acquire semantics, and only then reads the velocities, so by the PTX memory model it sees
// the released rows. Every body thus takes its constraints in colour order, as with a launch
// per colour, and every result has the same bits. A ticket waits only on lower tickets, held by
// warps that are running, so every wait ends; each is bounded all the same: a wait that gives
// up sets kErrWait (the call then fails) and the pass goes on without it, and once one has
// given up the others give up at once.

struct FlowTable {
    uint32_t ranges;                           // ranges in use
    uint32_t tickets;                          // tickets of all ranges
    uint32_t ticket[2 * NPH_GPU_COLORS];       // each range's first ticket
    uint32_t first[2 * NPH_GPU_COLORS];        // each range's first constraint
    uint32_t count[2 * NPH_GPU_COLORS];        // each range's constraints
    uint32_t colour_kind[2 * NPH_GPU_COLORS];  // the range's colour, | kFlowJoints for joints
};
constexpr uint32_t kFlowJoints = 0x100u;
constexpr uint32_t kFlowPolls = 1u << 20; // about a second of polls, 64 ns of sleep apart

NPH_D uint32_t ld_acquire_gpu(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

NPH_D void red_release_gpu_add(uint32_t *p, uint32_t v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// Waits until `need` constraints that write `body` have finished this pass.
NPH_D void flow_wait(uint32_t *done, uint32_t body, uint32_t need, uint32_t *err)
{
    if (need == 0u) {
        return;
    }
    for (uint32_t i = 0; i < kFlowPolls; ++i) {
        if (ld_acquire_gpu(&done[body]) >= need) {
            return;
        }
        if (i >= 8u) {
            if ((i & 1023u) == 0u && (*(const volatile uint32_t *)err & kErrWait) != 0u) {
                return;
            }
            __nanosleep(64);
        }
    }
    atomicOr(err, kErrWait);
}

// The wait of a manifold of a dependency-driven pass: its ranks are in hdr.w.
struct FlowGate {
    uint32_t *done;
    uint32_t *err;
    NPH_D void operator()(uint4 hdr) const
    {
        if ((hdr.z & kHdrWriteA) != 0u) {
            flow_wait(done, hdr.x, hdr.w & kRankMask, err);
        }
        if ((hdr.z & kHdrWriteB) != 0u) {
            flow_wait(done, hdr.y, (hdr.w >> kRankBits) & kRankMask, err);
        }
    }
};

// The bodies a constraint writes: contacts 0..m-1, then joints.
NPH_D void written_bodies(const DevSolver &S, bool joint, uint32_t k, uint32_t &a, uint32_t &b, bool &wa,
                          bool &wb)
{
    if (joint) {
        uint32_t flags;
        joint_head(S, k, a, b, flags);
        wa = (flags & kJWriteA) != 0u;
        wb = (flags & kJWriteB) != 0u;
    } else {
        const uint4 hdr = S.hdr[k];
        a = hdr.x;
        b = hdr.y;
        wa = (hdr.z & kHdrWriteA) != 0u && (hdr.z & kHdrPointsMask) != 0u;
        wb = (hdr.z & kHdrWriteB) != 0u && (hdr.z & kHdrPointsMask) != 0u;
    }
}

// A joint of a dependency-driven pass, out of line: the joints' registers stay out of the
// contacts' path.
template <int P> __device__ __noinline__ void flow_joint(const DevSolver &S, uint32_t j, const StepConsts &K)
{
    joint_op<P>(S, j, K);
}

template <int P, int kMinBlocks>
__global__ void __launch_bounds__(32, kMinBlocks)
k_pass_flow(DevSolver S, FlowTable F, StepConsts K, uint32_t *ticket, uint32_t *err)
{
    extern __shared__ float4 tile[];
    const uint32_t lane = threadIdx.x;
    const Tile<32> T{tile, lane};
    const FlowGate gate{S.done, err};
    // Tickets two deep: while ticket t runs, the next one is known (its constraint's header
    // fetched into L1 ahead of it) and the one after is being taken.
    uint32_t t = 0u, t1 = 0u;
    if (lane == 0u) {
        t = atomicAdd(ticket, 1u);
        t1 = atomicAdd(ticket, 1u);
    }
    t = __shfl_sync(0xFFFFFFFFu, t, 0);
    t1 = __shfl_sync(0xFFFFFFFFu, t1, 0);
    while (t < F.tickets) {
        uint32_t next = 0u;
        if (lane == 0u) {
            next = atomicAdd(ticket, 1u);
        }
        if (t1 < F.tickets) {
            uint32_t r1 = 0u;
            while (r1 + 1u < F.ranges && F.ticket[r1 + 1u] <= t1) {
                ++r1;
            }
            const uint32_t idx1 = (t1 - F.ticket[r1]) * 32u + lane;
            if (idx1 < F.count[r1]) {
                const uint32_t i1 = F.first[r1] + idx1;
                const void *row = (F.colour_kind[r1] & kFlowJoints) != 0u ? (const void *)&S.jw[kJrHead * S.jcap + i1]
                                                                          : (const void *)&S.hdr[i1];
                asm volatile("prefetch.global.L1 [%0];\n" ::"l"(row));
            }
        }
        uint32_t r = 0u;
        while (r + 1u < F.ranges && F.ticket[r + 1u] <= t) {
            ++r;
        }
        const uint32_t ck = F.colour_kind[r];
        const uint32_t idx = (t - F.ticket[r]) * 32u + lane;
        if (idx < F.count[r]) {
            const uint32_t i = F.first[r] + idx;
            const bool joint = (ck & kFlowJoints) != 0u;
            if (joint) {
                uint32_t a, b, flags;
                joint_head(S, i, a, b, flags);
                const uint32_t rank = S.jrank[i];
                if ((flags & kJWriteA) != 0u) {
                    flow_wait(S.done, a, rank & kRankMask, err);
                }
                if ((flags & kJWriteB) != 0u) {
                    flow_wait(S.done, b, (rank >> kRankBits) & kRankMask, err);
                }
                flow_joint<P>(S, i, K);
            } else if (P == kWarm) {
                warm_manifold(S, i, gate);
            } else {
                solve_manifold_staged<P == kSolve, 32, false, false>(S, i, K, T, gate);
            }
            // The header again (the pass kept none of it live): the bodies written, released
            // where a constraint of a later colour waits on them.
            uint32_t a, b;
            bool wa, wb;
            written_bodies(S, joint, i, a, b, wa, wb);
            const uint32_t rank = joint ? S.jrank[i] : S.hdr[i].w;
            if (wa && (rank & kRankLaterA) != 0u) {
                red_release_gpu_add(&S.done[a], 1u);
            }
            if (wb && (rank & kRankLaterB) != 0u) {
                red_release_gpu_add(&S.done[b], 1u);
            }
        }
        t = t1;
        t1 = __shfl_sync(0xFFFFFFFFu, next, 0);
    }
}

// The colour of constraint k of a kind, from its colour table (NPH_GPU_COLORS: the overflow).
NPH_D uint32_t colour_of(const ColorTable &tab, uint32_t k)
{
    uint32_t colour = NPH_GPU_COLORS;
    for (uint32_t c = 0; c < NPH_GPU_COLORS; ++c) {
        if (k >= tab.cfirst[c] && k - tab.cfirst[c] < tab.ccount[c]) {
            colour = c;
        }
    }
    return colour;
}

// The colours whose constraints write each body slot (bit c of cmask).
__global__ void __launch_bounds__(kBlock) k_colour_masks(DevSolver S, uint32_t m, uint32_t nj, ColorTable C,
                                                         ColorTable J)
{
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= m + nj) {
        return;
    }
    const bool joint = i >= m;
    const uint32_t k = joint ? i - m : i;
    const uint32_t colour = colour_of(joint ? J : C, k);
    if (colour == NPH_GPU_COLORS) {
        return; // the overflow runs before the pass
    }
    uint32_t a, b;
    bool wa, wb;
    written_bodies(S, joint, k, a, b, wa, wb);
    uint32_t *mask = const_cast<uint32_t *>(S.cmask);
    if (wa) {
        atomicOr(&mask[a], 1u << colour);
    }
    if (wb) {
        atomicOr(&mask[b], 1u << colour);
    }
}

// Each constraint's ranks on the bodies it writes (the earlier colours in their masks): a
// manifold's into hdr.w, a joint's into jrank.
__global__ void __launch_bounds__(kBlock) k_colour_ranks(DevSolver S, uint32_t m, uint32_t nj, ColorTable C,
                                                         ColorTable J, uint32_t extra)
{
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= m + nj) {
        return;
    }
    const bool joint = i >= m;
    const uint32_t k = joint ? i - m : i;
    const uint32_t colour = colour_of(joint ? J : C, k);
    uint32_t a, b;
    bool wa, wb;
    written_bodies(S, joint, k, a, b, wa, wb);
    const uint32_t below = colour < NPH_GPU_COLORS ? (1u << colour) - 1u : 0u;
    const uint32_t above = colour < NPH_GPU_COLORS ? ~((2u << colour) - 1u) : 0u;
    const uint32_t ma = wa ? S.cmask[a] : 0u, mb = wb ? S.cmask[b] : 0u;
    const uint32_t ra = wa ? (uint32_t)__popc(ma & below) + extra : 0u;
    const uint32_t rb = wb ? (uint32_t)__popc(mb & below) + extra : 0u;
    const uint32_t rank = ra | (rb << kRankBits) | ((ma & above) != 0u ? kRankLaterA : 0u) |
                          ((mb & above) != 0u ? kRankLaterB : 0u);
    if (joint) {
        S.jrank[k] = rank;
    } else {
        S.hdr[k].w = rank;
    }
}

__global__ void __launch_bounds__(kBlock) k_integrate_velocity(BodyArrays B, uint32_t n, float h)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        integrate_velocity(B, i, h);
    }
}

__global__ void __launch_bounds__(kBlock) k_integrate_position(BodyArrays B, uint32_t n, float h)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        integrate_position(B, i, h);
    }
}

// store_group (solver.c:475-499) on staged records.
__global__ void __launch_bounds__(kStage) k_store_contacts(DevSolver S, NphGpuContact *contacts,
                                                           uint32_t m)
{
    __shared__ NphGpuContact rec[kStage];
    const uint32_t first = blockIdx.x * kStage;
    const uint32_t count = min(kStage, m - first);
    stage_in<uint4>(contacts + first, count, rec);
    __syncthreads();
    if (threadIdx.x < count) {
        store_manifold(S, first + threadIdx.x, rec[threadIdx.x]);
    }
    __syncthreads();
    stage_out<uint4>(rec, count, contacts + first);
}

// The joints' accumulated impulses back into their records.
// The impulses (and a slider's or 6-DOF joint's rows and blocks) written into the records in
// place: the settings are not rewritten.
__global__ void __launch_bounds__(kBlock) k_store_joints(DevSolver S, NphGpuJoint *joints, uint32_t nj)
{
    const uint32_t j = blockIdx.x * kBlock + threadIdx.x;
    if (j < nj) {
        store_joint(S, j, joints[j]);
    }
}

// finalize_body, solver.c:304-324, on staged records.
__global__ void __launch_bounds__(kStage) k_finalize(BodyArrays B, NphGpuBody *bodies, uint32_t n,
                                                     float dt)
{
    __shared__ NphGpuBody rec[kStage];
    const uint32_t first = blockIdx.x * kStage;
    const uint32_t count = min(kStage, n - first);
    stage_in<uint4>(bodies + first, count, rec);
    __syncthreads();
    if (threadIdx.x < count) {
        finalize_body(B, first + threadIdx.x, rec[threadIdx.x], dt);
    }
    __syncthreads();
    stage_out<uint4>(rec, count, bodies + first);
}

// The packed drop-in's conversions (nph_gpu_phys_solve_packed): a block stages its records
// through shared memory in 4-byte words both ways, so the global reads and writes are
// coalesced whatever the records' sizes.
constexpr uint32_t kConvert = 64;
static_assert(sizeof(NphGpuBodyInput) % 4 == 0 && sizeof(NphGpuContactInput) % 4 == 0 &&
                  sizeof(NphGpuBodyOutput) % 4 == 0 && sizeof(NphGpuContactOutput) % 4 == 0 &&
                  sizeof(NphGpuJointOutput) % 4 == 0 && sizeof(NphGpuJoint) % 4 == 0,
              "packed records stage in 4-byte words");

__device__ void expand_body(const NphGpuBodyInput &i, NphGpuBody &o)
{
    for (uint32_t k = 0; k < 3u; ++k) {
        o.center[k] = i.center[k];
        o.origin[k] = 0.0;
        o.local_center[k] = i.local_center[k];
        o.linear_velocity[k] = i.linear_velocity[k];
        o.angular_velocity[k] = i.angular_velocity[k];
        o.force[k] = i.force[k];
        o.torque[k] = i.torque[k];
    }
    for (uint32_t k = 0; k < 4u; ++k) {
        o.rotation[k] = i.rotation[k];
    }
    for (uint32_t k = 0; k < 9u; ++k) {
        o.inertia[k] = i.inertia[k];
        o.inv_inertia[k] = i.inv_inertia[k];
    }
    o.inv_mass = i.inv_mass;
    o.linear_damping = i.linear_damping;
    o.angular_damping = i.angular_damping;
    o.gravity_scale = i.gravity_scale;
    o.sleep_threshold = i.sleep_threshold;
    o.sleep_time = i.sleep_time;
    o.max_extent = i.max_extent;
    o.type = i.type;
    o.flags = i.flags;
    o.locks = i.locks;
    o.pad = 0u;
}

__device__ void expand_contact(const NphGpuContactInput &i, NphGpuContact &o)
{
    o.body_a = i.body_a;
    o.body_b = i.body_b;
    o.flags = i.flags;
    o.point_count = i.point_count;
    for (uint32_t k = 0; k < 3u; ++k) {
        o.normal[k] = i.normal[k];
    }
    o.friction = i.friction;
    o.restitution = i.restitution;
    o.pad[0] = o.pad[1] = o.pad[2] = 0u;
    for (uint32_t p = 0; p < NPH_GPU_MAX_POINTS; ++p) {
        const NphGpuContactPointInput &a = i.points[p];
        NphGpuContactPoint &b = o.points[p];
        for (uint32_t k = 0; k < 3u; ++k) {
            b.anchor_a[k] = a.anchor_a[k];
            b.anchor_b[k] = a.anchor_b[k];
            b.tangent_impulse[k] = a.tangent_impulse[k];
        }
        b.separation = a.separation;
        b.normal_impulse = a.normal_impulse;
        b.max_normal_impulse = 0.0f;
        b.relative_velocity = 0.0f;
        b.id = a.id;
    }
}

__device__ void pack_body(const NphGpuBody &i, NphGpuBodyOutput &o)
{
    for (uint32_t k = 0; k < 3u; ++k) {
        o.center[k] = i.center[k];
        o.origin[k] = i.origin[k];
        o.linear_velocity[k] = i.linear_velocity[k];
        o.angular_velocity[k] = i.angular_velocity[k];
    }
    for (uint32_t k = 0; k < 4u; ++k) {
        o.rotation[k] = i.rotation[k];
    }
    o.sleep_time = i.sleep_time;
    o.pad = 0u;
}

__device__ void pack_contact(const NphGpuContact &i, NphGpuContactOutput &o)
{
    o.flags = i.flags;
    for (uint32_t p = 0; p < NPH_GPU_MAX_POINTS; ++p) {
        const NphGpuContactPoint &a = i.points[p];
        NphGpuContactPointOutput &b = o.points[p];
        b.normal_impulse = a.normal_impulse;
        b.max_normal_impulse = a.max_normal_impulse;
        for (uint32_t k = 0; k < 3u; ++k) {
            b.tangent_impulse[k] = a.tangent_impulse[k];
        }
        b.relative_velocity = a.relative_velocity;
    }
}

__device__ void pack_joint(const NphGpuJoint &i, NphGpuJointOutput &o)
{
    for (uint32_t k = 0; k < 3u; ++k) {
        o.linear_impulse[k] = i.linear_impulse[k];
        o.angular_impulse[k] = i.angular_impulse[k];
        o.friction_impulse[k] = i.friction_impulse[k];
    }
    o.lower_impulse = i.lower_impulse;
    o.upper_impulse = i.upper_impulse;
    o.swing_impulse = i.swing_impulse;
    o.motor_impulse = i.motor_impulse;
    o.spring_impulse = i.spring_impulse;
    for (uint32_t a = 0; a < NPH_GPU_D6_AXES; ++a) {
        for (uint32_t r = 0; r < 4u; ++r) {
            o.axis_impulse[a][r] = i.axis_impulse[a][r];
        }
    }
    o.flags = i.flags;
}

// Records of type In to records of type Out, kConvert a block.
template <typename In, typename Out, int kKind>
__global__ void __launch_bounds__(kConvert) k_convert(const In *in, Out *out, uint32_t count)
{
    __shared__ In src[kConvert];
    __shared__ Out dst[kConvert];
    const uint32_t first = blockIdx.x * kConvert;
    const uint32_t n = min(kConvert, count - first);
    stage_in<uint32_t>(in + first, n, src);
    __syncthreads();
    if (threadIdx.x < n) {
        if constexpr (kKind == 0) {
            expand_body(src[threadIdx.x], dst[threadIdx.x]);
        } else if constexpr (kKind == 1) {
            expand_contact(src[threadIdx.x], dst[threadIdx.x]);
        } else if constexpr (kKind == 2) {
            pack_body(src[threadIdx.x], dst[threadIdx.x]);
        } else if constexpr (kKind == 3) {
            pack_contact(src[threadIdx.x], dst[threadIdx.x]);
        } else {
            pack_joint(src[threadIdx.x], dst[threadIdx.x]);
        }
    }
    __syncthreads();
    stage_out<uint32_t>(dst, n, out + first);
}

template <typename In, typename Out, int kKind>
void launch_convert(const In *in, Out *out, uint32_t count, cudaStream_t st)
{
    if (count > 0u) {
        k_convert<In, Out, kKind><<<(count + kConvert - 1u) / kConvert, kConvert, 0, st>>>(in, out, count);
    }
}

// post_finalize, solver.c:851-857: a driven joint's bodies stay awake.
__global__ void __launch_bounds__(kBlock) k_driven(DevSolver S, NphGpuBody *bodies, uint32_t n,
                                                   uint32_t nj)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nj) {
        return;
    }
    uint32_t sa, sb, flags;
    joint_head(S, j, sa, sb, flags);
    if ((flags & kJDriven) != 0u) {
        if (sa < n) {
            bodies[sa].sleep_time = 0.0f;
        }
        if (sb < n) {
            bodies[sb].sleep_time = 0.0f;
        }
    }
}

// ------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------

static uint32_t blocks_for(uint64_t count) { return (uint32_t)((count + kBlock - 1) / kBlock); }
static uint32_t stage_blocks(uint64_t count) { return (uint32_t)((count + kStage - 1) / kStage); }

// solver.c:48-65 on the host, in FP32 as the reference.
static Soft host_make_soft(float hertz, float zeta, float h)
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

static float minf_ref(float a, float b) { return a < b ? a : b; }

// phys_solve's step constants, solver.c:985-1017: the soft step's springs, or TGS's rigid
// rows with a fifth of the error taken back a substep and a linear slop left alone.
StepConsts make_step_consts(const NphGpuWorldParams &p, float dt)
{
    StepConsts K;
    std::memset(&K, 0, sizeof K);
    K.dt = dt;
    K.h = dt / (float)p.substeps;
    K.inv_h = 1.0f / K.h;
    K.push_max = p.contact_push_max_velocity;
    K.restitution_threshold = p.restitution_threshold;
    const float contact_hertz = p.contact_hertz > 0.0f ? p.contact_hertz : 0.125f * K.inv_h;
    const float joint_hertz = p.joint_hertz > 0.0f ? p.joint_hertz : 0.25f * K.inv_h;
    const float hertz = minf_ref(contact_hertz, 0.25f * K.inv_h);
    K.contact_soft = host_make_soft(hertz, p.contact_damping_ratio, K.h);
    K.static_soft = host_make_soft(2.0f * hertz, p.contact_damping_ratio, K.h);
    K.joint_soft = host_make_soft(minf_ref(joint_hertz, 0.25f * K.inv_h), p.joint_damping_ratio, K.h);
    const float max_rotation = 0.25f * 3.14159265f * K.inv_h;
    K.max_angular_speed_sq = max_rotation * max_rotation;
    K.max_linear_speed_sq = p.max_linear_speed * p.max_linear_speed;
    K.gravity[0] = p.gravity[0];
    K.gravity[1] = p.gravity[1];
    K.gravity[2] = p.gravity[2];
    K.solver = p.solver;
    if (p.solver == NPH_GPU_SOLVER_TGS) {
        const Soft hard = Soft{0.2f * K.inv_h, 1.0f, 0.0f};
        K.contact_soft = hard;
        K.static_soft = hard;
        K.joint_soft = hard;
        K.slop = 0.005f; // NPH_PHYSICS_LINEAR_SLOP, types.h:38
        K.scale_hits = 1u;
    }
    return K;
}

// ---------------------------------------------------------------------------------------
// The island sleep decision (phys_island_sleep_and_split, island.c:675-735)
// ---------------------------------------------------------------------------------------

// Floats as keys that order as the floats do (non-NaN), for atomic min and max.
__device__ __forceinline__ uint32_t order_key(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) != 0u ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float order_value(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) != 0u ? (k & 0x7FFFFFFFu) : ~k);
}

__global__ void __launch_bounds__(256) k_island_init(uint32_t *tmin, uint32_t *tmax, uint32_t islands,
                                                     unsigned long long *split)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < islands) {
        tmin[k] = order_key(1e30f);
        tmax[k] = order_key(0.0f);
    }
    if (k == 0u) {
        *split = 0ull;
    }
}

// Each island's stillest and sleepiest body clock (a body without sleep counts as just
// moved), and each kinematic body's own verdict.
__global__ void __launch_bounds__(256) k_island_bounds(const NphGpuBody *bodies, uint32_t n,
                                                       const uint32_t *island_of, uint32_t islands,
                                                       float time_to_sleep, uint32_t *tmin, uint32_t *tmax,
                                                       uint8_t *kinematic, uint32_t *err)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const NphGpuBody &b = bodies[i];
    const bool may_sleep = (b.flags & NPH_GPU_BODY_ENABLE_SLEEP) != 0u;
    const uint32_t k = island_of[i];
    if (k != NPH_GPU_NULL) {
        if (k >= islands) {
            atomicOr(err, kErrBadIndex);
        } else {
            const uint32_t key = order_key(may_sleep ? b.sleep_time : 0.0f);
            atomicMin(&tmin[k], key);
            atomicMax(&tmax[k], key);
        }
    }
    kinematic[i] = (b.type == NPH_GPU_BODY_KINEMATIC && may_sleep && b.sleep_time >= time_to_sleep) ? 1u : 0u;
}

// Whole islands whose stillest body is ready sleep; of those that lost constraints, the one
// whose sleepiest body is most ready (the first such in the list) is split instead.
__global__ void __launch_bounds__(256) k_island_decide(const uint32_t *tmin, const uint32_t *tmax,
                                                       const uint32_t *removed, uint32_t islands,
                                                       float time_to_sleep, uint8_t *sleep,
                                                       unsigned long long *split)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= islands) {
        return;
    }
    const float t = order_value(tmin[k]);
    const float sleepiest = order_value(tmax[k]);
    uint8_t asleep = 0u;
    if (removed[k] > 0u) {
        if (sleepiest >= time_to_sleep && sleepiest > 0.0f) {
            atomicMax(split, ((unsigned long long)order_key(sleepiest) << 32) | (0xFFFFFFFFull - k));
        }
    } else if (t >= time_to_sleep) {
        asleep = 1u;
    }
    sleep[k] = asleep;
}

// hit_events (solver.c:919-960) for one manifold: with NPH_GPU_CONTACT_HIT_EVENTS, its point of
// fastest approach above the threshold among those with a positive max_normal_impulse (the
// first on a tie: only a strictly faster point replaces it).
__device__ __forceinline__ bool hit_point(const NphGpuContact &c, float threshold, uint32_t &point, float &speed)
{
    if ((c.flags & NPH_GPU_CONTACT_HIT_EVENTS) == 0u) {
        return false;
    }
    const uint32_t pc = c.point_count <= NPH_GPU_MAX_POINTS ? c.point_count : 0u;
    float best = threshold;
    uint32_t found = NPH_GPU_NULL;
    for (uint32_t k = 0; k < pc; ++k) {
        const float approach = -c.points[k].relative_velocity;
        if (approach > best && c.points[k].max_normal_impulse > 0.0f) {
            best = approach;
            found = k;
        }
    }
    point = found;
    speed = best;
    return found != NPH_GPU_NULL;
}

constexpr uint32_t kHitBlock = 256;
constexpr uint32_t kHitScanThreads = 1024;

// The hits of each block of manifolds.
__global__ void __launch_bounds__(kHitBlock) k_hit_count(const NphGpuContact *contacts, uint32_t m, float threshold,
                                                         uint32_t *block_hits)
{
    const uint32_t g = blockIdx.x * kHitBlock + threadIdx.x;
    uint32_t point = 0u;
    float speed = 0.0f;
    const bool hit = g < m && hit_point(contacts[g], threshold, point, speed);
    const uint32_t n = (uint32_t)__syncthreads_count(hit ? 1 : 0);
    if (threadIdx.x == 0u) {
        block_hits[blockIdx.x] = n;
    }
}

// The blocks' hit counts turned into each block's first event, in place, and the total after
// them: each thread sums a run of blocks, one block-wide scan of the runs, then each run again.
__global__ void __launch_bounds__(kHitScanThreads) k_hit_scan(uint32_t *block_hits, uint32_t blocks)
{
    __shared__ uint32_t part[kHitScanThreads];
    const uint32_t t = threadIdx.x;
    const uint32_t per = (blocks + kHitScanThreads - 1u) / kHitScanThreads;
    const uint32_t first = min(blocks, t * per), end = min(blocks, first + per);
    uint32_t sum = 0u;
    for (uint32_t i = first; i < end; ++i) {
        sum += block_hits[i];
    }
    part[t] = sum;
    __syncthreads();
    for (uint32_t d = 1u; d < kHitScanThreads; d <<= 1u) {
        const uint32_t v = t >= d ? part[t - d] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = part[t] - sum;
    for (uint32_t i = first; i < end; ++i) {
        const uint32_t h = block_hits[i];
        block_hits[i] = run;
        run += h;
    }
    if (t == kHitScanThreads - 1u) {
        block_hits[blocks] = part[t];
    }
}

// Each hit at its block's first event plus the hits before it in the block: manifold order.
__global__ void __launch_bounds__(kHitBlock) k_hit_write(const NphGpuContact *contacts, uint32_t m, float threshold,
                                                         const uint32_t *block_first, NphGpuHitEvent *out)
{
    __shared__ uint32_t warp_hits[kHitBlock / 32u];
    const uint32_t g = blockIdx.x * kHitBlock + threadIdx.x;
    uint32_t point = 0u;
    float speed = 0.0f;
    const bool hit = g < m && hit_point(contacts[g], threshold, point, speed);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5u;
    const uint32_t ballot = __ballot_sync(0xFFFFFFFFu, hit);
    if (lane == 0u) {
        warp_hits[warp] = (uint32_t)__popc(ballot);
    }
    __syncthreads();
    uint32_t at = block_first[blockIdx.x] + (uint32_t)__popc(ballot & ((1u << lane) - 1u));
    for (uint32_t w = 0; w < warp; ++w) {
        at += warp_hits[w];
    }
    if (hit) {
        out[at] = NphGpuHitEvent{g, point, speed, 0u}; // world 0: the caller numbers batches' worlds
    }
}

} // namespace nph

using namespace nph;

struct NphGpuSolver {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t side = nullptr; // a colour's joints run here beside its contacts
    cudaEvent_t fork_event = nullptr, join_event = nullptr;
    bool use_graph = true;
    // Capacities of the device arrays.
    uint32_t bcap = 0, fcap = 0, mcap = 0, jcap = 0;
    uint64_t memory_limit = 0; // bytes the record and row arrays may take (0: no limit)
    uint32_t wait_injection = 0; // added to every dependency count (a test hook)
    // The packed drop-in's device arrays (allocated by its first call).
    NphGpuBodyInput *in_bodies = nullptr;
    NphGpuContactInput *in_contacts = nullptr;
    NphGpuBodyOutput *out_bodies = nullptr;
    NphGpuContactOutput *out_contacts = nullptr;
    NphGpuJointOutput *out_joints = nullptr;
    uint32_t pbcap = 0, pmcap = 0, pjcap = 0;
    // Records (device copies of the view's arrays).
    NphGpuBody *d_bodies = nullptr;
    NphGpuBody *d_fixed = nullptr;
    NphGpuContact *d_contacts = nullptr;
    NphGpuJoint *d_joints = nullptr;
    // Solver state.
    float4 *body_rows = nullptr; // vel | pos | prm
    float4 *vel = nullptr, *pos = nullptr, *prm = nullptr, *itg = nullptr;
    uint4 *hdr = nullptr;
    float4 *nrm = nullptr;
    float *rest = nullptr;
    float4 *pa = nullptr, *pb = nullptr, *pt = nullptr, *pi = nullptr;
    float4 *jw = nullptr;
    // The dependency-driven passes: per body slot the colours that write it and the finished
    // constraints of the current pass; done[n + 1] the pass's next warp ticket.
    uint32_t *cmask = nullptr, *done = nullptr;
    uint32_t *jrank = nullptr; // per joint: its ranks on its bodies
    uint32_t *d_err = nullptr;     // [0] error bits, [1..25] points per colour slot
    uint32_t *h_err = nullptr;     // pinned copy of the same 26 words
    // Per-launch timing of a profiled step.
    struct Mark {
        int kind;
        uint64_t units;
        double bytes;
        cudaEvent_t a, b;
    };
    std::vector<Mark> *marks = nullptr;
    std::vector<cudaEvent_t> event_pool;
    size_t events_used = 0;
    // The uploaded world.
    bool uploaded = false;
    uint32_t n = 0, nf = 0, m = 0, nj = 0;
    uint32_t ccount[NPH_GPU_COLOR_SLOTS] = {}, jcount[NPH_GPU_COLOR_SLOTS] = {};
    uint32_t cfirst[NPH_GPU_COLOR_SLOTS] = {}, jfirst[NPH_GPU_COLOR_SLOTS] = {};
    uint32_t driven = 0;
    uint32_t row_joints = 0; // slider, 6-DOF and distance joints: their own launch per colour
    // Pass configuration per pass kind (warm, solve, relax, restitution).
    uint32_t pass_config[4] = {2, 7, 7, 0};
    // The step graph and what it was captured for.
    cudaGraphExec_t graph = nullptr;
    StepConsts graph_consts{};
    uint32_t graph_substeps = 0;
    bool graph_valid = false;
    cudaEvent_t ev[6] = {};
    NphGpuStepStats stats{};
    uint32_t launches = 0;
    // The contact update's staging of the narrow phase's manifolds (capacity mcap).
    NphGpuContact *d_fresh = nullptr;
    uint32_t fresh_cap = 0;
    // The learned warm start: the attached network and its cold-point buffers.
    NphGpuMlp *mlp = nullptr;
    uint32_t lcap = 0;            // cold points the buffers hold
    float *l_feat = nullptr, *l_pred = nullptr, *l_scale = nullptr;
    uint32_t *l_slot = nullptr;
    uint32_t *l_counts = nullptr; // [0] cold points, [1] features written
    // The residual-driven mode's buffers.
    uint32_t rcap = 0;            // residual slots (passes + 1)
    float *r_sq = nullptr, *r_val = nullptr, *r_ref = nullptr, *r_part = nullptr;
    uint32_t *r_state = nullptr;  // [0] done, [1] passes, [2] cold points, [3] predicted
};

namespace {

template <typename T> void dfree(T *&p)
{
    if (p != nullptr) {
        cudaFree(p);
        p = nullptr;
    }
}

template <typename T> bool dalloc(T *&p, size_t count)
{
    dfree(p);
    if (count == 0) {
        count = 1;
    }
    return cudaMalloc((void **)&p, count * sizeof(T)) == cudaSuccess;
}

void drop_graph(NphGpuSolver *s)
{
    if (s->graph != nullptr) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    s->graph_valid = false;
}

// Device bytes of the record and row arrays at these capacities.
uint64_t array_bytes(uint64_t bcap, uint64_t fcap, uint64_t mcap, uint64_t jcap)
{
    return bcap * (sizeof(NphGpuBody) + 13u * sizeof(float4) + 2u * sizeof(uint32_t)) + 2u * sizeof(uint32_t) +
           fcap * sizeof(NphGpuBody) +
           mcap * (sizeof(NphGpuContact) + sizeof(uint4) + sizeof(float4) + sizeof(float) +
                   16u * sizeof(float4)) +
           jcap * (sizeof(NphGpuJoint) + (uint64_t)kJointRows * sizeof(float4) + sizeof(uint32_t));
}

// Device bytes of the packed drop-in's arrays at these capacities.
uint64_t packed_bytes(uint64_t bcap, uint64_t mcap, uint64_t jcap)
{
    return bcap * (sizeof(NphGpuBodyInput) + sizeof(NphGpuBodyOutput)) +
           mcap * (sizeof(NphGpuContactInput) + sizeof(NphGpuContactOutput)) + jcap * sizeof(NphGpuJointOutput);
}

uint64_t grown(uint32_t need, uint32_t cap) { return need > cap ? (uint64_t)need + need / 8u + 1u : cap; }

// Grows the device arrays to hold the view (between steps only), and the packed drop-in's when
// `packed`. A growth the solver's memory limit does not allow is refused before any array is
// touched: the world stays as it was.
NphGpuResult ensure_capacity(NphGpuSolver *s, uint32_t n, uint32_t nf, uint32_t m, uint32_t nj,
                             bool packed = false)
{
    if (s->memory_limit != 0u) {
        const uint64_t bcap = n + 1u > s->bcap ? (uint64_t)(n + 1u) + (n + 1u) / 8u : s->bcap;
        const uint64_t fcap = nf > s->fcap ? (uint64_t)nf + nf / 8u + 1u : s->fcap;
        const uint64_t mcap = m > s->mcap ? (uint64_t)m + m / 8u + 1u : s->mcap;
        const uint64_t jcap = nj > s->jcap ? (uint64_t)nj + nj / 8u + 1u : s->jcap;
        uint64_t total = array_bytes(bcap, fcap, mcap, jcap);
        if (packed || s->pbcap > 0u) {
            total += packed_bytes(packed ? grown(n, s->pbcap) : s->pbcap, packed ? grown(m, s->pmcap) : s->pmcap,
                                  packed ? grown(nj, s->pjcap) : s->pjcap);
        }
        if (total > s->memory_limit) {
            return NPH_GPU_OUT_OF_MEMORY;
        }
    }
    bool ok = true;
    if (packed && n > s->pbcap) {
        const uint32_t cap = (uint32_t)grown(n, 0u);
        ok = dalloc(s->in_bodies, cap) && dalloc(s->out_bodies, cap);
        s->pbcap = ok ? cap : 0;
    }
    if (ok && packed && m > s->pmcap) {
        const uint32_t cap = (uint32_t)grown(m, 0u);
        ok = dalloc(s->in_contacts, cap) && dalloc(s->out_contacts, cap);
        s->pmcap = ok ? cap : 0;
    }
    if (ok && packed && nj > s->pjcap) {
        const uint32_t cap = (uint32_t)grown(nj, 0u);
        ok = dalloc(s->out_joints, cap);
        s->pjcap = ok ? cap : 0;
    }
    if (n + 1u > s->bcap) {
        const uint32_t cap = n + 1u + (n + 1u) / 8u;
        // vel, pos and prm in one allocation: the body rows the constraint passes gather.
        ok = ok && dalloc(s->d_bodies, cap) && dalloc(s->body_rows, 7ull * cap) &&
             dalloc(s->itg, 6ull * cap) && dalloc(s->cmask, cap) && dalloc(s->done, cap + 2ull);
        if (ok) {
            s->vel = s->body_rows;
            s->pos = s->body_rows + 2ull * cap;
            s->prm = s->body_rows + 4ull * cap;
        }
        s->bcap = ok ? cap : 0;
    }
    if (ok && nf > s->fcap) {
        const uint32_t cap = nf + nf / 8u + 1u;
        ok = dalloc(s->d_fixed, cap);
        s->fcap = ok ? cap : 0;
    }
    if (ok && m > s->mcap) {
        const uint32_t cap = m + m / 8u + 1u;
        ok = dalloc(s->d_contacts, cap) && dalloc(s->hdr, cap) && dalloc(s->nrm, cap) &&
             dalloc(s->rest, cap) && dalloc(s->pa, 4ull * cap) && dalloc(s->pb, 4ull * cap) &&
             dalloc(s->pt, 4ull * cap) && dalloc(s->pi, 4ull * cap);
        s->mcap = ok ? cap : 0;
    }
    if (ok && nj > s->jcap) {
        const uint32_t cap = nj + nj / 8u + 1u;
        ok = dalloc(s->d_joints, cap) && dalloc(s->jw, (size_t)kJointRows * cap) && dalloc(s->jrank, cap);
        s->jcap = ok ? cap : 0;
    }
    if (!ok) {
        s->uploaded = false;
        drop_graph(s);
        cudaGetLastError();
        return NPH_GPU_OUT_OF_MEMORY;
    }
    return NPH_GPU_OK;
}

DevSolver dev_solver(const NphGpuSolver *s)
{
    DevSolver S;
    S.vel = s->vel;
    S.pos = s->pos;
    S.prm = s->prm;
    S.hdr = s->hdr;
    S.nrm = s->nrm;
    S.rest = s->rest;
    S.pa = s->pa;
    S.pb = s->pb;
    S.pt = s->pt;
    S.pi = s->pi;
    S.mcap = s->mcap;
    S.jw = s->jw;
    S.jcap = s->jcap;
    S.cmask = s->cmask;
    S.done = s->done;
    S.jrank = s->jrank;
    return S;
}

BodyArrays body_arrays(const NphGpuSolver *s)
{
    return BodyArrays{s->vel, s->pos, s->prm, s->itg};
}

// Kernel kinds of a profiled step, and the reference data model's live bytes per unit.
enum Kind : int {
    kKPrepareBodies = 0,
    kKPrepareConstraints,
    kKIntegrateVelocity,
    kKWarm,
    kKSolve,
    kKIntegratePosition,
    kKRelax,
    kKRestitution,
    kKStoreFinalize,
    kKOverflow,
    kKDriven,
    kKJoints,
    kKinds
};
const char *const kKindNames[kKinds] = {"prepare_bodies", "prepare_constraints", "integrate_velocity",
                                        "warm_start", "solve", "integrate_position", "relax",
                                        "restitution", "store_finalize", "overflow", "driven",
                                        "joints"};

cudaEvent_t next_event(NphGpuSolver *s)
{
    if (s->events_used == s->event_pool.size()) {
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        s->event_pool.push_back(e);
    }
    return s->event_pool[s->events_used++];
}

void mark_begin(NphGpuSolver *s, int kind, uint64_t units, double bytes)
{
    if (s->marks == nullptr) {
        return;
    }
    NphGpuSolver::Mark m{kind, units, bytes, next_event(s), next_event(s)};
    cudaEventRecord(m.a, s->stream);
    s->marks->push_back(m);
}

void mark_end(NphGpuSolver *s)
{
    if (s->marks != nullptr) {
        cudaEventRecord(s->marks->back().b, s->stream);
    }
}

// Points per colour slot (filled by the last prepare), for the byte counts.
uint64_t color_points(const NphGpuSolver *s, uint32_t c) { return s->h_err[1 + c]; }

template <int P> void enqueue_pass(NphGpuSolver *s, const StepConsts &K)
{
    const DevSolver S = dev_solver(s);
    const uint32_t o = NPH_GPU_OVERFLOW;
    const uint32_t oj = P == kRestitution ? 0u : s->jcount[o];
    const int kind = P == kWarm ? kKWarm : P == kSolve ? kKSolve : P == kRelax ? kKRelax : kKRestitution;
    auto bytes = [&](uint32_t c, uint32_t jc) -> double {
        const double m = s->ccount[c];
        const double pts = s->marks != nullptr ? (double)color_points(s, c) : 4.0 * m;
        switch (P) {
        case kWarm: return 120.0 * pts + 330.0 * jc;
        case kSolve: return 224.0 * m + 148.0 * pts + 330.0 * jc;
        case kRelax: return 212.0 * m + 148.0 * pts + 330.0 * jc;
        default: return 40.0 * m;
        }
    };
    if (s->ccount[o] > 0u || oj > 0u) {
        mark_begin(s, kKOverflow, (uint64_t)s->ccount[o] + oj, bytes(o, oj));
        k_overflow<P><<<1, 32, 0, s->stream>>>(S, s->cfirst[o], s->ccount[o], s->jfirst[o], oj, K);
        mark_end(s);
        s->launches++;
    }
    const uint32_t cfg = s->pass_config[P];
    if constexpr (P != kRestitution) {
    if (kPassConfigs[cfg].staged == 5u) {
        // Every colour in one dependency-driven launch (k_pass_flow).
        FlowTable F{};
        uint32_t tickets = 0, ranges = 0;
        uint64_t units = 0;
        double flow_bytes = 0.0;
        for (uint32_t c = 0; c < NPH_GPU_COLORS; ++c) {
            for (uint32_t half = 0; half < 2u; ++half) { // the colour's joints, then its contacts
                const bool joint = half == 0u;
                const uint32_t count = joint ? s->jcount[c] : s->ccount[c];
                if (count > 0u) {
                    F.ticket[ranges] = tickets;
                    F.first[ranges] = joint ? s->jfirst[c] : s->cfirst[c];
                    F.count[ranges] = count;
                    F.colour_kind[ranges] = c | (joint ? kFlowJoints : 0u);
                    tickets += (count + 31u) / 32u;
                    ranges += 1u;
                }
            }
            units += (uint64_t)s->ccount[c] + s->jcount[c];
            flow_bytes += bytes(c, s->jcount[c]);
        }
        F.ranges = ranges;
        F.tickets = tickets;
        if (tickets == 0u) {
            return;
        }
        static const uint32_t sms = [] {
            int dev = 0, n = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
            return (uint32_t)n;
        }();
        const uint32_t grid = std::min<uint32_t>(tickets, sms * kPassConfigs[cfg].min_blocks);
        const size_t smem = P == kWarm ? 0 : (size_t)kPointSlots * 32u * sizeof(float4);
        uint32_t *ticket = s->done + s->n + 1u;
        cudaMemsetAsync(s->done, 0, (s->n + 2ull) * sizeof(uint32_t), s->stream);
        mark_begin(s, kind, units, flow_bytes);
        switch (kPassConfigs[cfg].min_blocks) {
        case 16: k_pass_flow<P, 16><<<grid, 32, smem, s->stream>>>(S, F, K, ticket, s->d_err); break;
        case 20: k_pass_flow<P, 20><<<grid, 32, smem, s->stream>>>(S, F, K, ticket, s->d_err); break;
        default: k_pass_flow<P, 18><<<grid, 32, smem, s->stream>>>(S, F, K, ticket, s->d_err); break;
        }
        mark_end(s);
        s->launches++;
        return;
    }
    }
    for (uint32_t c = 0; c < NPH_GPU_COLORS; ++c) {
        const uint32_t jc = P == kRestitution ? 0u : s->jcount[c];
        const uint32_t cc = s->ccount[c];
        if (jc == 0u && cc == 0u) {
            continue;
        }
        // The colour's joints beside its contacts: forked to the side stream and joined back
        // (sequential on the solver's stream when a profiled step times each launch).
        const bool fork = jc > 0u && cc > 0u && s->marks == nullptr;
        if (jc > 0u) {
            cudaStream_t js = s->stream;
            if (fork) {
                cudaEventRecord(s->fork_event, s->stream);
                cudaStreamWaitEvent(s->side, s->fork_event, 0);
                js = s->side;
            }
            mark_begin(s, kKJoints, jc, 330.0 * jc);
            if (s->row_joints > 0u) {
                k_joint_pass<P, kJointsPlain><<<blocks_for(jc), kBlock, 0, js>>>(S, s->jfirst[c], jc, K);
                k_joint_pass<P, kJointsRows><<<blocks_for(jc), kBlock, 0, js>>>(S, s->jfirst[c], jc, K);
                s->launches++;
            } else {
                k_joint_pass<P, kJointsPlain><<<blocks_for(jc), kBlock, 0, js>>>(S, s->jfirst[c], jc, K);
            }
            mark_end(s);
            s->launches++;
        }
        if (cc > 0u) {
            mark_begin(s, kind, cc, bytes(c, 0u));
            launch_pass<P>(s->pass_config[P], cc, s->stream, S, s->cfirst[c], K);
            mark_end(s);
            s->launches++;
        }
        if (fork) {
            cudaEventRecord(s->join_event, s->side);
            cudaStreamWaitEvent(s->stream, s->join_event, 0);
        }
    }
}

// The step's prepare stage: bodies, then joints and contacts (solver.c:1032-1041).
void enqueue_prepare(NphGpuSolver *s, const StepConsts &K)
{
    const DevSolver S = dev_solver(s);
    const BodyArrays B = body_arrays(s);
    const double n = s->n;
    mark_begin(s, kKPrepareBodies, s->n, 368.0 * n);
    k_prepare_bodies<<<stage_blocks(s->n + 1u), kStage, 0, s->stream>>>(B, s->d_bodies, s->n, K,
                                                                         s->d_err);
    mark_end(s);
    s->launches++;
    ColorTable T;
    std::memcpy(T.cfirst, s->cfirst, sizeof T.cfirst);
    std::memcpy(T.ccount, s->ccount, sizeof T.ccount);
    cudaMemsetAsync(s->d_err + 1, 0, NPH_GPU_COLOR_SLOTS * sizeof(uint32_t), s->stream);
    if (s->nj > 0u) {
        mark_begin(s, kKPrepareConstraints, s->nj, 330.0 * s->nj);
        k_prepare_joints<<<blocks_for(s->nj), kBlock, 0, s->stream>>>(
            S, s->d_joints, s->d_bodies, s->d_fixed, s->n, s->nf, s->nj, K.h, s->d_err);
        mark_end(s);
        s->launches++;
    }
    if (s->m > 0u) {
        mark_begin(s, kKPrepareConstraints, s->m, 936.0 * s->m);
        k_prepare_contacts<<<stage_blocks(s->m), kStage, 0, s->stream>>>(
            S, s->d_contacts, s->d_fixed, s->n, s->nf, s->m, T, s->d_err, s->d_err + 1);
        mark_end(s);
        s->launches++;
    }
    bool flow = false;
    for (uint32_t p = kWarm; p <= kRelax; ++p) {
        flow = flow || kPassConfigs[s->pass_config[p]].staged == 5u;
    }
    if (flow && s->m + s->nj > 0u) {
        // The colours that write each body, for the dependency-driven passes.
        ColorTable J;
        std::memcpy(J.cfirst, s->jfirst, sizeof J.cfirst);
        std::memcpy(J.ccount, s->jcount, sizeof J.ccount);
        cudaMemsetAsync(s->cmask, 0, (s->n + 1ull) * sizeof(uint32_t), s->stream);
        mark_begin(s, kKPrepareConstraints, (uint64_t)s->m + s->nj, 56.0 * (s->m + s->nj));
        k_colour_masks<<<blocks_for((uint64_t)s->m + s->nj), kBlock, 0, s->stream>>>(S, s->m, s->nj, T, J);
        k_colour_ranks<<<blocks_for((uint64_t)s->m + s->nj), kBlock, 0, s->stream>>>(S, s->m, s->nj, T, J,
                                                                                     s->wait_injection);
        mark_end(s);
        s->launches += 2u;
    }
}

// The feature scales: g = |gravity| (1 m/s^2 without gravity) and h.
FeatureConsts feature_consts(const StepConsts &K)
{
    const double gx = K.gravity[0], gy = K.gravity[1], gz = K.gravity[2];
    const double gl = std::sqrt(gx * gx + gy * gy + gz * gz);
    const double g = gl > 0.0 ? gl : 1.0;
    FeatureConsts F;
    F.gh = (float)(g * K.h);
    F.inv_gh = (float)(1.0 / (g * K.h));
    F.gdir[0] = gl > 0.0 ? (float)(gx / gl) : 0.0f;
    F.gdir[1] = gl > 0.0 ? (float)(gy / gl) : 0.0f;
    F.gdir[2] = gl > 0.0 ? (float)(gz / gl) : 0.0f;
    return F;
}

// The learned warm start of the cold points (after prepare): their features, the network's
// predictions, and the predictions written as their warm-start impulses.
void enqueue_learned_init(NphGpuSolver *s, const StepConsts &K)
{
    if (s->mlp == nullptr || s->m == 0u || s->lcap == 0u || K.solver != NPH_GPU_SOLVER_SOFT_STEP) {
        return; // the model is the soft step's; TGS warm-starts as the reference does
    }
    const DevSolver S = dev_solver(s);
    cudaMemsetAsync(s->l_counts, 0, 2 * sizeof(uint32_t), s->stream);
    k_cold_features<<<blocks_for(s->m), 256, 0, s->stream>>>(S, s->m, feature_consts(K), s->l_feat, s->l_scale,
                                                             s->l_slot, s->l_counts, s->lcap, 1u);
    nph_mlp_forward_device_count(s->mlp, s->l_feat, s->l_counts + 1, s->lcap, s->l_pred, s->stream);
    k_apply_predictions<<<blocks_for(s->lcap), 256, 0, s->stream>>>(S, s->l_pred, s->l_scale, s->l_slot,
                                                                    s->l_counts, s->lcap);
    s->launches += 3;
}

// One step's launches on the solver's stream (the stage list, solver.c:1032-1067).
void enqueue_step(NphGpuSolver *s, const StepConsts &K, uint32_t substeps)
{
    const DevSolver S = dev_solver(s);
    const BodyArrays B = body_arrays(s);
    const double n = s->n;
    s->launches = 0;
    enqueue_prepare(s, K);
    enqueue_learned_init(s, K);
    for (uint32_t sub = 0; sub < substeps; ++sub) {
        mark_begin(s, kKIntegrateVelocity, s->n, 84.0 * n);
        k_integrate_velocity<<<blocks_for(s->n), kBlock, 0, s->stream>>>(B, s->n, K.h);
        mark_end(s);
        enqueue_pass<kWarm>(s, K);
        enqueue_pass<kSolve>(s, K);
        mark_begin(s, kKIntegratePosition, s->n, 84.0 * n);
        k_integrate_position<<<blocks_for(s->n), kBlock, 0, s->stream>>>(B, s->n, K.h);
        mark_end(s);
        if (K.solver == NPH_GPU_SOLVER_SOFT_STEP) {
            enqueue_pass<kRelax>(s, K);
        }
        s->launches += 2;
    }
    if (K.solver == NPH_GPU_SOLVER_TGS) {
        enqueue_pass<kRelax>(s, K); // TGS's velocity iteration: the bias velocity taken back once
    }
    enqueue_pass<kRestitution>(s, K);
    if (s->m > 0u) {
        mark_begin(s, kKStoreFinalize, s->m, 160.0 * s->m);
        k_store_contacts<<<stage_blocks(s->m), kStage, 0, s->stream>>>(S, s->d_contacts, s->m);
        mark_end(s);
        s->launches++;
    }
    if (s->nj > 0u) {
        mark_begin(s, kKStoreFinalize, s->nj, 330.0 * s->nj);
        k_store_joints<<<blocks_for(s->nj), kBlock, 0, s->stream>>>(S, s->d_joints, s->nj);
        mark_end(s);
        s->launches++;
    }
    mark_begin(s, kKStoreFinalize, s->n, 200.0 * n);
    k_finalize<<<stage_blocks(s->n), kStage, 0, s->stream>>>(B, s->d_bodies, s->n, K.dt);
    mark_end(s);
    s->launches++;
    if (s->driven > 0u) {
        mark_begin(s, kKDriven, s->nj, 0.0);
        k_driven<<<blocks_for(s->nj), kBlock, 0, s->stream>>>(S, s->d_bodies, s->n, s->nj);
        mark_end(s);
        s->launches++;
    }
}

NphGpuResult check_cuda(cudaError_t e)
{
    if (e == cudaSuccess) {
        return NPH_GPU_OK;
    }
    if (e == cudaErrorMemoryAllocation) {
        return NPH_GPU_OUT_OF_MEMORY;
    }
    return NPH_GPU_DEVICE_LOST;
}

// Replays (capturing first if needed) one step as a graph, or launches it directly.
NphGpuResult ensure_learned(NphGpuSolver *s);

NphGpuResult launch_step(NphGpuSolver *s, const StepConsts &K, uint32_t substeps)
{
    const NphGpuResult lr = ensure_learned(s);
    if (lr != NPH_GPU_OK) {
        return lr;
    }
    if (!s->use_graph) {
        enqueue_step(s, K, substeps);
        return check_cuda(cudaGetLastError());
    }
    if (!s->graph_valid || s->graph_substeps != substeps ||
        std::memcmp(&s->graph_consts, &K, sizeof K) != 0) {
        drop_graph(s);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            return check_cuda(e);
        }
        enqueue_step(s, K, substeps);
        e = cudaStreamEndCapture(s->stream, &g);
        if (e != cudaSuccess) {
            return check_cuda(e);
        }
        e = cudaGraphInstantiate(&s->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            s->graph = nullptr;
            return check_cuda(e);
        }
        s->graph_consts = K;
        s->graph_substeps = substeps;
        s->graph_valid = true;
    }
    return check_cuda(cudaGraphLaunch(s->graph, s->stream));
}

NphGpuResult validate_params(const NphGpuWorldParams *p, float dt)
{
    if (p == nullptr || !(dt > 0.0f) || p->substeps == 0u || p->substeps > 64u) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if ((p->solver != NPH_GPU_SOLVER_SOFT_STEP && p->solver != NPH_GPU_SOLVER_TGS) ||
        p->enable_continuous != 0u) {
        return NPH_GPU_UNSUPPORTED;
    }
    return NPH_GPU_OK;
}

// The learned warm start and its convergence runs are the soft step's.
static NphGpuResult validate_soft_params(const NphGpuWorldParams *p, float dt)
{
    const NphGpuResult r = validate_params(p, dt);
    return r == NPH_GPU_OK && p->solver != NPH_GPU_SOLVER_SOFT_STEP ? NPH_GPU_UNSUPPORTED : r;
}

NphGpuResult validate_view(const NphGpuWorldView *v)
{
    if (v == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    uint64_t nc = 0, nj = 0;
    for (uint32_t c = 0; c < NPH_GPU_COLOR_SLOTS; ++c) {
        nc += v->contact_color_counts[c];
        nj += v->joint_color_counts[c];
    }
    if (nc != v->contact_count || nj != v->joint_count) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if ((v->body_count > 0 && v->bodies == nullptr) || (v->fixed_count > 0 && v->fixed_bodies == nullptr) ||
        (v->contact_count > 0 && v->contacts == nullptr) || (v->joint_count > 0 && v->joints == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if ((uint64_t)v->body_count + v->fixed_count >= 0xFFFFFFF0ull) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    return NPH_GPU_OK;
}

// Checks a view's counts and joint records, grows the arrays, and takes the view's shape
// (its counts and colour tables); the records are the caller's to copy.
NphGpuResult upload_shape(NphGpuSolver *s, const NphGpuWorldView *v, bool packed)
{
    NphGpuResult r = validate_view(v);
    if (r != NPH_GPU_OK) {
        return r;
    }
    // The joint records first: a refused view leaves the solver as it was.
    uint32_t driven = 0, row_joints = 0;
    for (uint32_t j = 0; j < v->joint_count; ++j) {
        const NphGpuJoint &jr = v->joints[j];
        const int bad = nph_joint_check(&jr);
        if (bad != NPH_GPU_OK) {
            return (NphGpuResult)bad;
        }
        driven += nph_joint_is_driven(&jr) ? 1u : 0u;
        row_joints += (nph_joint_has_axes(jr.type) || jr.type == NPH_GPU_JOINT_DISTANCE) ? 1u : 0u;
    }
    r = ensure_capacity(s, v->body_count, v->fixed_count, v->contact_count, v->joint_count, packed);
    if (r != NPH_GPU_OK) {
        return r;
    }
    const bool same_shape = s->uploaded && s->n == v->body_count && s->nf == v->fixed_count &&
                            s->m == v->contact_count && s->nj == v->joint_count &&
                            std::memcmp(s->ccount, v->contact_color_counts, sizeof s->ccount) == 0 &&
                            std::memcmp(s->jcount, v->joint_color_counts, sizeof s->jcount) == 0;
    s->n = v->body_count;
    s->nf = v->fixed_count;
    s->m = v->contact_count;
    s->nj = v->joint_count;
    uint32_t cf = 0, jf = 0;
    for (uint32_t c = 0; c < NPH_GPU_COLOR_SLOTS; ++c) {
        s->ccount[c] = v->contact_color_counts[c];
        s->jcount[c] = v->joint_color_counts[c];
        s->cfirst[c] = cf;
        s->jfirst[c] = jf;
        cf += s->ccount[c];
        jf += s->jcount[c];
    }
    if (!same_shape || driven != s->driven || (row_joints > 0u) != (s->row_joints > 0u)) {
        drop_graph(s);
    }
    s->driven = driven;
    s->row_joints = row_joints;
    return NPH_GPU_OK;
}

NphGpuResult upload(NphGpuSolver *s, const NphGpuWorldView *v)
{
    const NphGpuResult r = upload_shape(s, v, false);
    if (r != NPH_GPU_OK) {
        return r;
    }
    cudaMemcpyAsync(s->d_bodies, v->bodies, sizeof(NphGpuBody) * s->n, cudaMemcpyHostToDevice, s->stream);
    if (s->nf > 0) {
        cudaMemcpyAsync(s->d_fixed, v->fixed_bodies, sizeof(NphGpuBody) * s->nf, cudaMemcpyHostToDevice,
                        s->stream);
    }
    if (s->m > 0) {
        cudaMemcpyAsync(s->d_contacts, v->contacts, sizeof(NphGpuContact) * s->m, cudaMemcpyHostToDevice,
                        s->stream);
    }
    if (s->nj > 0) {
        cudaMemcpyAsync(s->d_joints, v->joints, sizeof(NphGpuJoint) * s->nj, cudaMemcpyHostToDevice,
                        s->stream);
    }
    cudaMemsetAsync(s->d_err, 0, 32 * sizeof(uint32_t), s->stream);
    s->uploaded = true;
    return check_cuda(cudaGetLastError());
}

NphGpuResult download(NphGpuSolver *s, NphGpuWorldView *v)
{
    if (!s->uploaded || v == nullptr || v->body_count != s->n || v->contact_count != s->m ||
        v->joint_count != s->nj) {
        return NPH_GPU_INVALID_STATE;
    }
    cudaMemcpyAsync(v->bodies, s->d_bodies, sizeof(NphGpuBody) * s->n, cudaMemcpyDeviceToHost, s->stream);
    if (s->m > 0) {
        cudaMemcpyAsync(v->contacts, s->d_contacts, sizeof(NphGpuContact) * s->m, cudaMemcpyDeviceToHost,
                        s->stream);
    }
    if (s->nj > 0) {
        cudaMemcpyAsync(v->joints, s->d_joints, sizeof(NphGpuJoint) * s->nj, cudaMemcpyDeviceToHost,
                        s->stream);
    }
    return check_cuda(cudaStreamSynchronize(s->stream));
}

// The packed drop-in's upload: the packed records up, expanded into the solver's records on the
// device (the fields the stage only writes start at zero).
NphGpuResult upload_packed(NphGpuSolver *s, const NphGpuPackedInput *in)
{
    if (in == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    NphGpuWorldView shape;
    std::memset(&shape, 0, sizeof shape);
    shape.bodies = (NphGpuBody *)in->bodies; // for the null checks only: never read as records
    shape.body_count = in->body_count;
    shape.fixed_count = in->fixed_count;
    shape.fixed_bodies = in->fixed_bodies;
    shape.contacts = (NphGpuContact *)in->contacts;
    shape.contact_count = in->contact_count;
    shape.joint_count = in->joint_count;
    shape.joints = (NphGpuJoint *)in->joints;
    std::memcpy(shape.contact_color_counts, in->contact_color_counts, sizeof shape.contact_color_counts);
    std::memcpy(shape.joint_color_counts, in->joint_color_counts, sizeof shape.joint_color_counts);
    const NphGpuResult r = upload_shape(s, &shape, true);
    if (r != NPH_GPU_OK) {
        return r;
    }
    cudaMemcpyAsync(s->in_bodies, in->bodies, sizeof(NphGpuBodyInput) * s->n, cudaMemcpyHostToDevice, s->stream);
    if (s->nf > 0) {
        cudaMemcpyAsync(s->d_fixed, in->fixed_bodies, sizeof(NphGpuBody) * s->nf, cudaMemcpyHostToDevice,
                        s->stream);
    }
    if (s->m > 0) {
        cudaMemcpyAsync(s->in_contacts, in->contacts, sizeof(NphGpuContactInput) * s->m,
                        cudaMemcpyHostToDevice, s->stream);
    }
    if (s->nj > 0) {
        cudaMemcpyAsync(s->d_joints, in->joints, sizeof(NphGpuJoint) * s->nj, cudaMemcpyHostToDevice,
                        s->stream);
    }
    launch_convert<NphGpuBodyInput, NphGpuBody, 0>(s->in_bodies, s->d_bodies, s->n, s->stream);
    launch_convert<NphGpuContactInput, NphGpuContact, 1>(s->in_contacts, s->d_contacts, s->m, s->stream);
    cudaMemsetAsync(s->d_err, 0, 32 * sizeof(uint32_t), s->stream);
    s->uploaded = true;
    return check_cuda(cudaGetLastError());
}

// The packed drop-in's download: the written fields packed on the device, one copy per kind.
NphGpuResult download_packed(NphGpuSolver *s, NphGpuPackedOutput *out)
{
    launch_convert<NphGpuBody, NphGpuBodyOutput, 2>(s->d_bodies, s->out_bodies, s->n, s->stream);
    launch_convert<NphGpuContact, NphGpuContactOutput, 3>(s->d_contacts, s->out_contacts, s->m, s->stream);
    launch_convert<NphGpuJoint, NphGpuJointOutput, 4>(s->d_joints, s->out_joints, s->nj, s->stream);
    cudaMemcpyAsync(out->bodies, s->out_bodies, sizeof(NphGpuBodyOutput) * s->n, cudaMemcpyDeviceToHost,
                    s->stream);
    if (s->m > 0) {
        cudaMemcpyAsync(out->contacts, s->out_contacts, sizeof(NphGpuContactOutput) * s->m,
                        cudaMemcpyDeviceToHost, s->stream);
    }
    if (s->nj > 0) {
        cudaMemcpyAsync(out->joints, s->out_joints, sizeof(NphGpuJointOutput) * s->nj, cudaMemcpyDeviceToHost,
                        s->stream);
    }
    return check_cuda(cudaStreamSynchronize(s->stream));
}

NphGpuResult read_error(NphGpuSolver *s)
{
    cudaMemcpyAsync(s->h_err, s->d_err, 32 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    const NphGpuResult r = check_cuda(cudaStreamSynchronize(s->stream));
    if (r != NPH_GPU_OK) {
        return r;
    }
    s->stats.error_word = *s->h_err;
    if ((*s->h_err & kErrWait) != 0u) {
        return NPH_GPU_DEVICE_LOST;
    }
    return *s->h_err != 0u ? NPH_GPU_INVALID_ARGUMENT : NPH_GPU_OK;
}

void fill_stats(NphGpuSolver *s)
{
    uint32_t used = 0;
    for (uint32_t c = 0; c < NPH_GPU_COLORS; ++c) {
        used += (s->ccount[c] > 0u || s->jcount[c] > 0u) ? 1u : 0u;
    }
    s->stats.colors_used = used;
    s->stats.overflow_contacts = s->ccount[NPH_GPU_OVERFLOW];
    s->stats.overflow_joints = s->jcount[NPH_GPU_OVERFLOW];
    s->stats.launches = s->launches;
}

// The cold-point buffers of the learned warm start, for every point slot of the world.
NphGpuResult ensure_learned(NphGpuSolver *s)
{
    const uint64_t want = 4ull * s->m;
    if (s->mlp == nullptr || want <= s->lcap) {
        return NPH_GPU_OK;
    }
    if (want > 0x7FFFFFFFull) {
        return NPH_GPU_TOO_LARGE;
    }
    const uint32_t cap = (uint32_t)(want + want / 8u + 64u);
    drop_graph(s);
    const bool ok = dalloc(s->l_feat, (size_t)cap * NPH_GPU_MLP_INPUTS) && dalloc(s->l_pred, (size_t)cap * 3u) &&
                    dalloc(s->l_scale, cap) && dalloc(s->l_slot, cap) && dalloc(s->l_counts, 2);
    if (!ok) {
        s->lcap = 0;
        cudaGetLastError();
        return NPH_GPU_OUT_OF_MEMORY;
    }
    s->lcap = cap;
    return NPH_GPU_OK;
}

NphGpuResult ensure_residuals(NphGpuSolver *s, uint32_t slots)
{
    if (slots <= s->rcap && s->r_state != nullptr) {
        return NPH_GPU_OK;
    }
    const bool ok = dalloc(s->r_sq, slots) && dalloc(s->r_val, slots) && dalloc(s->r_ref, 1) &&
                    dalloc(s->r_state, 4) && dalloc(s->r_part, kResidualBlocks);
    if (!ok) {
        s->rcap = 0;
        cudaGetLastError();
        return NPH_GPU_OUT_OF_MEMORY;
    }
    s->rcap = slots;
    return NPH_GPU_OK;
}

// One rigid pass of the residual-driven mode: the overflow, then every colour's joints and
// contacts (a colour's joints and contacts share no dynamic body).
void enqueue_converge_pass(NphGpuSolver *s, const StepConsts &K, const uint32_t *done)
{
    const DevSolver S = dev_solver(s);
    const uint32_t o = NPH_GPU_OVERFLOW;
    if (s->ccount[o] > 0u || s->jcount[o] > 0u) {
        k_converge_overflow<<<1, 32, 0, s->stream>>>(S, s->cfirst[o], s->ccount[o], s->jfirst[o], s->jcount[o], K,
                                                     done);
    }
    for (uint32_t c = 0; c < NPH_GPU_COLORS; ++c) {
        if (s->jcount[c] > 0u) {
            k_converge_joint_pass<<<blocks_for(s->jcount[c]), 256, 0, s->stream>>>(S, s->jfirst[c], s->jcount[c], K,
                                                                                   done);
        }
        if (s->ccount[c] > 0u) {
            k_converge_pass<128><<<(s->ccount[c] + 127u) / 128u, 128, 0, s->stream>>>(S, s->cfirst[c], s->ccount[c],
                                                                                      K, done);
        }
    }
}

} // namespace

// ------------------------------------------------------------------------------------
// Internal links (solver_link.h)
// ------------------------------------------------------------------------------------

NphGpuResult nph_solver_bind_device(NphGpuSolver *s, const NphGpuWorldView *v, uint32_t driven,
                                    uint32_t row_joints, NphSolverRecords *out)
{
    if (s == nullptr || v == nullptr || out == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    uint64_t nc = 0, nj = 0;
    for (uint32_t c = 0; c < NPH_GPU_COLOR_SLOTS; ++c) {
        nc += v->contact_color_counts[c];
        nj += v->joint_color_counts[c];
    }
    if (nc != v->contact_count || nj != v->joint_count ||
        (uint64_t)v->body_count + v->fixed_count >= 0xFFFFFFF0ull) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(s->device);
    NphGpuResult r = ensure_capacity(s, v->body_count, v->fixed_count, v->contact_count, v->joint_count);
    if (r != NPH_GPU_OK) {
        return r;
    }
    const bool same_shape = s->uploaded && s->n == v->body_count && s->nf == v->fixed_count &&
                            s->m == v->contact_count && s->nj == v->joint_count &&
                            std::memcmp(s->ccount, v->contact_color_counts, sizeof s->ccount) == 0 &&
                            std::memcmp(s->jcount, v->joint_color_counts, sizeof s->jcount) == 0;
    s->n = v->body_count;
    s->nf = v->fixed_count;
    s->m = v->contact_count;
    s->nj = v->joint_count;
    uint32_t cf = 0, jf = 0;
    for (uint32_t c = 0; c < NPH_GPU_COLOR_SLOTS; ++c) {
        s->ccount[c] = v->contact_color_counts[c];
        s->jcount[c] = v->joint_color_counts[c];
        s->cfirst[c] = cf;
        s->jfirst[c] = jf;
        cf += s->ccount[c];
        jf += s->jcount[c];
    }
    if (!same_shape || driven != s->driven || (row_joints > 0u) != (s->row_joints > 0u)) {
        drop_graph(s);
    }
    s->driven = driven;
    s->row_joints = row_joints;
    cudaMemsetAsync(s->d_err, 0, 32 * sizeof(uint32_t), s->stream);
    s->uploaded = true;
    return nph_solver_records(s, out);
}

NphGpuResult nph_solver_records(NphGpuSolver *s, NphSolverRecords *out)
{
    if (s == nullptr || out == nullptr || !s->uploaded) {
        return NPH_GPU_INVALID_STATE;
    }
    out->bodies = s->d_bodies;
    out->fixed = s->d_fixed;
    out->contacts = s->d_contacts;
    out->joints = s->d_joints;
    return NPH_GPU_OK;
}

NphGpuResult nph_solver_check(NphGpuSolver *s)
{
    if (s == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(s->device);
    return read_error(s);
}

NphGpuResult nph_hits_scan(const NphGpuContact *contacts, uint32_t m, float threshold, cudaStream_t st,
                           NphGpuHitEvent *events, uint32_t capacity, uint32_t *count)
{
    *count = 0u;
    if (m == 0u) {
        return NPH_GPU_OK;
    }
    const uint32_t blocks = (m + kHitBlock - 1u) / kHitBlock;
    uint32_t *d_blocks = nullptr;
    NphGpuHitEvent *d_out = nullptr;
    NphGpuResult r = dalloc(d_blocks, blocks + 1u) && dalloc(d_out, m) ? NPH_GPU_OK : NPH_GPU_OUT_OF_MEMORY;
    uint32_t total = 0u;
    if (r == NPH_GPU_OK) {
        k_hit_count<<<blocks, kHitBlock, 0, st>>>(contacts, m, threshold, d_blocks);
        k_hit_scan<<<1, kHitScanThreads, 0, st>>>(d_blocks, blocks);
        k_hit_write<<<blocks, kHitBlock, 0, st>>>(contacts, m, threshold, d_blocks, d_out);
        cudaMemcpyAsync(&total, d_blocks + blocks, sizeof total, cudaMemcpyDeviceToHost, st);
        r = check_cuda(cudaStreamSynchronize(st));
    }
    const uint32_t n = std::min(total, capacity);
    if (r == NPH_GPU_OK && n > 0u) {
        r = check_cuda(cudaMemcpy(events, d_out, sizeof(NphGpuHitEvent) * n, cudaMemcpyDeviceToHost));
    }
    if (r == NPH_GPU_OK) {
        *count = total;
    }
    cudaGetLastError();
    dfree(d_blocks);
    dfree(d_out);
    return r;
}

// ------------------------------------------------------------------------------------
// The C ABI
// ------------------------------------------------------------------------------------

extern "C" {

NPH_GPU_API NphGpuResult nph_gpu_solver_create(const NphGpuSolverDesc *desc, NphGpuSolver **out)
{
    if (out == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    *out = nullptr;
    NphGpuSolverDesc d{};
    if (desc != nullptr) {
        d = *desc;
    } else {
        d.use_graph = 1;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return NPH_GPU_DEVICE_LOST;
    }
    if (d.device < 0 || d.device >= count) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    NphGpuSolver *s = new (std::nothrow) NphGpuSolver();
    if (s == nullptr) {
        return NPH_GPU_OUT_OF_MEMORY;
    }
    s->device = d.device;
    s->use_graph = d.use_graph != 0u;
    if (cudaSetDevice(d.device) != cudaSuccess) {
        delete s;
        return NPH_GPU_DEVICE_LOST;
    }
    if (d.stream != nullptr) {
        s->stream = (cudaStream_t)d.stream;
    } else {
        if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete s;
            return NPH_GPU_DEVICE_LOST;
        }
        s->own_stream = true;
    }
    bool ok = cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&s->fork_event, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&s->join_event, cudaEventDisableTiming) == cudaSuccess &&
              dalloc(s->d_err, 32) && cudaMallocHost((void **)&s->h_err, 32 * sizeof(uint32_t)) == cudaSuccess;
    for (auto &e : s->ev) {
        ok = ok && cudaEventCreate(&e) == cudaSuccess;
    }
    if (ok) {
        ok = ensure_capacity(s, d.body_capacity, 0, d.contact_capacity, d.joint_capacity) == NPH_GPU_OK;
    }
    allow_tiles<kWarm>();
    allow_tiles<kSolve>();
    allow_tiles<kRelax>();
    allow_tiles<kRestitution>();
    if (!ok) {
        nph_gpu_solver_destroy(s);
        return NPH_GPU_OUT_OF_MEMORY;
    }
    *out = s;
    return NPH_GPU_OK;
}

NPH_GPU_API void nph_gpu_solver_destroy(NphGpuSolver *s)
{
    if (s == nullptr) {
        return;
    }
    cudaSetDevice(s->device);
    if (s->stream != nullptr) {
        cudaStreamSynchronize(s->stream);
    }
    drop_graph(s);
    dfree(s->d_bodies);
    dfree(s->d_fixed);
    dfree(s->d_contacts);
    dfree(s->d_joints);
    dfree(s->body_rows);
    s->vel = s->pos = s->prm = nullptr;
    dfree(s->itg);
    dfree(s->cmask);
    dfree(s->done);
    dfree(s->jrank);
    dfree(s->hdr);
    dfree(s->nrm);
    dfree(s->rest);
    dfree(s->pa);
    dfree(s->pb);
    dfree(s->pt);
    dfree(s->pi);
    dfree(s->jw);
    dfree(s->d_fresh);
    dfree(s->l_feat);
    dfree(s->l_pred);
    dfree(s->l_scale);
    dfree(s->l_slot);
    dfree(s->l_counts);
    dfree(s->r_sq);
    dfree(s->r_part);
    dfree(s->r_val);
    dfree(s->r_ref);
    dfree(s->r_state);
    dfree(s->d_err);
    dfree(s->in_bodies);
    dfree(s->in_contacts);
    dfree(s->out_bodies);
    dfree(s->out_contacts);
    dfree(s->out_joints);
    if (s->h_err != nullptr) {
        cudaFreeHost(s->h_err);
    }
    for (auto &e : s->ev) {
        if (e != nullptr) {
            cudaEventDestroy(e);
        }
    }
    for (auto &e : s->event_pool) {
        cudaEventDestroy(e);
    }
    if (s->fork_event != nullptr) {
        cudaEventDestroy(s->fork_event);
    }
    if (s->join_event != nullptr) {
        cudaEventDestroy(s->join_event);
    }
    if (s->side != nullptr) {
        cudaStreamSynchronize(s->side);
        cudaStreamDestroy(s->side);
    }
    if (s->own_stream && s->stream != nullptr) {
        cudaStreamDestroy(s->stream);
    }
    delete s;
}

NPH_GPU_API NphGpuResult nph_gpu_world_upload(NphGpuSolver *s, const NphGpuWorldView *view)
{
    if (s == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(s->device);
    NphGpuResult r = upload(s, view);
    if (r == NPH_GPU_OK) {
        r = check_cuda(cudaStreamSynchronize(s->stream));
    }
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_world_step_async(NphGpuSolver *s, const NphGpuWorldParams *params,
                                                  float dt, uint32_t steps)
{
    if (s == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    NphGpuResult r = validate_params(params, dt);
    if (r != NPH_GPU_OK) {
        return r;
    }
    if (!s->uploaded) {
        return NPH_GPU_INVALID_STATE;
    }
    cudaSetDevice(s->device);
    const StepConsts K = make_step_consts(*params, dt);
    for (uint32_t i = 0; i < steps && r == NPH_GPU_OK; ++i) {
        r = launch_step(s, K, params->substeps);
    }
    fill_stats(s);
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_world_download(NphGpuSolver *s, NphGpuWorldView *view)
{
    if (s == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(s->device);
    NphGpuResult r = read_error(s);
    if (r != NPH_GPU_OK) {
        return r;
    }
    return download(s, view);
}

NPH_GPU_API NphGpuResult nph_gpu_solver_synchronize(NphGpuSolver *s)
{
    if (s == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(s->device);
    return check_cuda(cudaStreamSynchronize(s->stream));
}

NPH_GPU_API NphGpuResult nph_gpu_phys_solve(NphGpuSolver *s, const NphGpuWorldParams *params, float dt,
                                            NphGpuWorldView *view)
{
    if (s == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    NphGpuResult r = validate_params(params, dt);
    if (r != NPH_GPU_OK) {
        return r;
    }
    cudaSetDevice(s->device);
    if (view != nullptr && view->body_count == 0u) {
        return validate_view(view); // phys_solve with no awake body does nothing (solver.c:963-966)
    }
    cudaEventRecord(s->ev[0], s->stream);
    r = upload(s, view);
    if (r != NPH_GPU_OK) {
        return r;
    }
    cudaEventRecord(s->ev[1], s->stream);
    const StepConsts K = make_step_consts(*params, dt);
    r = launch_step(s, K, params->substeps);
    if (r != NPH_GPU_OK) {
        return r;
    }
    cudaEventRecord(s->ev[2], s->stream);
    r = read_error(s);
    if (r != NPH_GPU_OK) {
        return r; // the view is untouched: the step did not happen
    }
    cudaEventRecord(s->ev[3], s->stream);
    r = download(s, view);
    if (r != NPH_GPU_OK) {
        return r;
    }
    cudaEventRecord(s->ev[4], s->stream);
    cudaEventSynchronize(s->ev[4]);
    cudaEventElapsedTime(&s->stats.upload_ms, s->ev[0], s->ev[1]);
    cudaEventElapsedTime(&s->stats.device_ms, s->ev[1], s->ev[2]);
    cudaEventElapsedTime(&s->stats.download_ms, s->ev[3], s->ev[4]);
    fill_stats(s);
    return NPH_GPU_OK;
}

NPH_GPU_API NphGpuResult nph_gpu_phys_solve_packed(NphGpuSolver *s, const NphGpuWorldParams *params, float dt,
                                                   const NphGpuPackedInput *in, NphGpuPackedOutput *out)
{
    if (s == nullptr || in == nullptr || out == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    NphGpuResult r = validate_params(params, dt);
    if (r != NPH_GPU_OK) {
        return r;
    }
    if ((in->body_count > 0 && out->bodies == nullptr) || (in->contact_count > 0 && out->contacts == nullptr) ||
        (in->joint_count > 0 && out->joints == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(s->device);
    if (in->body_count == 0u) {
        uint64_t nc = 0, nj = 0;
        for (uint32_t c = 0; c < NPH_GPU_COLOR_SLOTS; ++c) {
            nc += in->contact_color_counts[c];
            nj += in->joint_color_counts[c];
        }
        return nc == in->contact_count && nj == in->joint_count ? NPH_GPU_OK : NPH_GPU_INVALID_ARGUMENT;
    }
    cudaEventRecord(s->ev[0], s->stream);
    r = upload_packed(s, in);
    if (r != NPH_GPU_OK) {
        return r;
    }
    cudaEventRecord(s->ev[1], s->stream);
    const StepConsts K = make_step_consts(*params, dt);
    r = launch_step(s, K, params->substeps);
    if (r != NPH_GPU_OK) {
        return r;
    }
    cudaEventRecord(s->ev[2], s->stream);
    r = read_error(s);
    if (r != NPH_GPU_OK) {
        return r; // the outputs are untouched: the step did not happen
    }
    cudaEventRecord(s->ev[3], s->stream);
    r = download_packed(s, out);
    if (r != NPH_GPU_OK) {
        return r;
    }
    cudaEventRecord(s->ev[4], s->stream);
    cudaEventSynchronize(s->ev[4]);
    cudaEventElapsedTime(&s->stats.upload_ms, s->ev[0], s->ev[1]);
    cudaEventElapsedTime(&s->stats.device_ms, s->ev[1], s->ev[2]);
    cudaEventElapsedTime(&s->stats.download_ms, s->ev[3], s->ev[4]);
    fill_stats(s);
    return NPH_GPU_OK;
}

NPH_GPU_API NphGpuResult nph_gpu_world_profile_step(NphGpuSolver *s, const NphGpuWorldParams *params,
                                                    float dt, NphGpuKernelTime *out, uint32_t capacity,
                                                    uint32_t *count)
{
    if (s == nullptr || out == nullptr || count == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    NphGpuResult r = validate_params(params, dt);
    if (r != NPH_GPU_OK) {
        return r;
    }
    if (!s->uploaded) {
        return NPH_GPU_INVALID_STATE;
    }
    cudaSetDevice(s->device);
    // The points per colour of the last prepare: run one prepare's worth first when needed.
    r = read_error(s);
    if (r != NPH_GPU_OK) {
        return r;
    }
    const StepConsts K = make_step_consts(*params, dt);
    std::vector<NphGpuSolver::Mark> marks;
    marks.reserve(1024);
    s->marks = &marks;
    s->events_used = 0;
    enqueue_step(s, K, params->substeps);
    s->marks = nullptr;
    r = check_cuda(cudaStreamSynchronize(s->stream));
    if (r != NPH_GPU_OK) {
        return r;
    }
    NphGpuKernelTime kinds[kKinds];
    std::memset(kinds, 0, sizeof kinds);
    for (const auto &m : marks) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, m.a, m.b);
        NphGpuKernelTime &k = kinds[m.kind];
        k.launches += 1;
        k.units += m.units;
        k.total_ms += ms;
        k.algorithmic_bytes += m.bytes;
    }
    uint32_t n = 0;
    for (int k = 0; k < kKinds; ++k) {
        if (kinds[k].launches == 0) {
            continue;
        }
        if (n < capacity) {
            out[n] = kinds[k];
            std::strncpy(out[n].name, kKindNames[k], sizeof out[n].name - 1);
        }
        ++n;
    }
    *count = n < capacity ? n : capacity;
    fill_stats(s);
    return NPH_GPU_OK;
}

NPH_GPU_API NphGpuResult nph_gpu_solver_set_pass_config(NphGpuSolver *s, uint32_t pass,
                                                         uint32_t config)
{
    if (s == nullptr || pass >= 4u || config >= kPassConfigCount) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if (s->pass_config[pass] != config) {
        s->pass_config[pass] = config;
        drop_graph(s);
    }
    return NPH_GPU_OK;
}

NPH_GPU_API uint32_t nph_gpu_pass_config_count(void) { return kPassConfigCount; }

NPH_GPU_API NphGpuResult nph_gpu_solver_autotune(NphGpuSolver *s, const NphGpuWorldParams *params,
                                                 float dt, uint32_t rounds, uint32_t *chosen)
{
    if (s == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    NphGpuResult r = validate_params(params, dt);
    if (r != NPH_GPU_OK) {
        return r;
    }
    if (!s->uploaded) {
        return NPH_GPU_INVALID_STATE;
    }
    cudaSetDevice(s->device);
    const StepConsts K = make_step_consts(*params, dt);
    const int kinds[4] = {kKWarm, kKSolve, kKRelax, kKRestitution};
    double best_ms[4];
    uint32_t best[4];
    for (uint32_t p = 0; p < 4; ++p) {
        best_ms[p] = 1e300;
        best[p] = s->pass_config[p];
    }
    rounds = rounds == 0u ? 1u : rounds;
    double flow_ms[4];
    uint32_t flow[4];
    for (uint32_t p = 0; p < 4; ++p) {
        flow_ms[p] = 1e300;
        flow[p] = kPassConfigCount;
    }
    for (uint32_t c = 0; c < kPassConfigCount; ++c) {
        for (uint32_t p = 0; p < 4; ++p) {
            s->pass_config[p] = c;
        }
        double ms[4] = {0.0, 0.0, 0.0, 0.0};
        for (uint32_t round = 0; round <= rounds; ++round) {
            std::vector<NphGpuSolver::Mark> marks;
            marks.reserve(1024);
            s->marks = &marks;
            s->events_used = 0;
            enqueue_step(s, K, params->substeps);
            s->marks = nullptr;
            r = check_cuda(cudaStreamSynchronize(s->stream));
            if (r != NPH_GPU_OK) {
                return r;
            }
            if (round == 0u) {
                continue; // the first step of a configuration warms its kernels
            }
            for (const auto &m : marks) {
                float t = 0.0f;
                cudaEventElapsedTime(&t, m.a, m.b);
                for (uint32_t p = 0; p < 4; ++p) {
                    if (m.kind == kinds[p]) {
                        ms[p] += t;
                    }
                }
            }
        }
        for (uint32_t p = 0; p < 4; ++p) {
            if (ms[p] < best_ms[p]) {
                best_ms[p] = ms[p];
                best[p] = c;
            }
            if (kPassConfigs[c].staged == 5u && ms[p] < flow_ms[p]) {
                flow_ms[p] = ms[p];
                flow[p] = c;
            }
        }
    }
    // Launch by launch, a dependency-driven pass counts its colours' joints and a colour a
    // launch does not (its joints are a kind of their own, beside it in the step's graph), so
    // the two forms are compared once more over whole steps of the graph: the chosen set
    // against the same with solve and relax dependency-driven.
    if (s->use_graph && flow[kSolve] < kPassConfigCount && flow[kRelax] < kPassConfigCount &&
        (best[kSolve] != flow[kSolve] || best[kRelax] != flow[kRelax])) {
        auto step_ms = [&](const uint32_t cfg[4], double &out) -> NphGpuResult {
            std::memcpy(s->pass_config, cfg, 4 * sizeof(uint32_t));
            drop_graph(s);
            NphGpuResult q = launch_step(s, K, params->substeps); // captures and warms
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            cudaEventRecord(e0, s->stream);
            for (uint32_t i = 0; i < rounds + 1u && q == NPH_GPU_OK; ++i) {
                q = launch_step(s, K, params->substeps);
            }
            cudaEventRecord(e1, s->stream);
            if (q == NPH_GPU_OK) {
                q = check_cuda(cudaEventSynchronize(e1));
            }
            float t = 0.0f;
            if (q == NPH_GPU_OK) {
                cudaEventElapsedTime(&t, e0, e1);
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            out = t;
            return q;
        };
        uint32_t with_flow[4];
        std::memcpy(with_flow, best, sizeof with_flow);
        with_flow[kSolve] = flow[kSolve];
        with_flow[kRelax] = flow[kRelax];
        double plain_ms = 0.0, flow_step_ms = 0.0;
        r = step_ms(best, plain_ms);
        if (r == NPH_GPU_OK) {
            r = step_ms(with_flow, flow_step_ms);
        }
        if (r != NPH_GPU_OK) {
            return r;
        }
        if (flow_step_ms < plain_ms) {
            std::memcpy(best, with_flow, sizeof best);
        }
    }
    for (uint32_t p = 0; p < 4; ++p) {
        s->pass_config[p] = best[p];
        if (chosen != nullptr) {
            chosen[p] = best[p];
        }
    }
    drop_graph(s);
    return NPH_GPU_OK;
}

NPH_GPU_API NphGpuResult nph_gpu_solver_stats(const NphGpuSolver *s, NphGpuStepStats *out)
{
    if (s == nullptr || out == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    *out = s->stats;
    return NPH_GPU_OK;
}

NPH_GPU_API void *nph_gpu_solver_stream(const NphGpuSolver *s)
{
    return s != nullptr ? (void *)s->stream : nullptr;
}

NPH_GPU_API NphGpuResult nph_gpu_solver_set_memory_limit(NphGpuSolver *s, uint64_t bytes)
{
    if (s == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    s->memory_limit = bytes;
    return NPH_GPU_OK;
}

NPH_GPU_API uint64_t nph_gpu_solver_memory(const NphGpuSolver *s)
{
    return s != nullptr ? array_bytes(s->bcap, s->fcap, s->mcap, s->jcap) : 0u;
}

NPH_GPU_API NphGpuResult nph_gpu_solver_set_wait_injection(NphGpuSolver *s, uint32_t extra)
{
    if (s == nullptr || extra > 64u) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if (s->wait_injection != extra) {
        s->wait_injection = extra;
        drop_graph(s);
    }
    return NPH_GPU_OK;
}

} // extern "C"

int nph_solver_device(const NphGpuSolver *s) { return s != nullptr ? s->device : 0; }

extern "C" {

NPH_GPU_API NphGpuResult nph_gpu_world_update_contacts(NphGpuSolver *s, const NphGpuContact *fresh,
                                                       uint32_t count)
{
    if (s == nullptr || (count > 0 && fresh == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if (!s->uploaded || count != s->m) {
        return NPH_GPU_INVALID_STATE;
    }
    if (count == 0) {
        return NPH_GPU_OK;
    }
    for (uint32_t g = 0; g < count; ++g) {
        if (fresh[g].point_count < 1u || fresh[g].point_count > NPH_GPU_MAX_POINTS) {
            return NPH_GPU_INVALID_ARGUMENT;
        }
    }
    cudaSetDevice(s->device);
    if (s->fresh_cap < count) {
        if (!dalloc(s->d_fresh, s->mcap)) {
            s->fresh_cap = 0;
            cudaGetLastError();
            return NPH_GPU_OUT_OF_MEMORY;
        }
        s->fresh_cap = s->mcap;
    }
    cudaMemcpyAsync(s->d_fresh, fresh, sizeof(NphGpuContact) * count, cudaMemcpyHostToDevice, s->stream);
    k_warm_update<<<(count + 127u) / 128u, 128, 0, s->stream>>>(s->d_contacts, s->d_fresh, count);
    return check_cuda(cudaStreamSynchronize(s->stream));
}

NPH_GPU_API NphGpuResult nph_gpu_solver_set_warm_start_model(NphGpuSolver *s, NphGpuMlp *mlp)
{
    if (s == nullptr || (mlp != nullptr && nph_mlp_device(mlp) != s->device)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    s->mlp = mlp;
    drop_graph(s);
    return ensure_learned(s);
}

NPH_GPU_API NphGpuResult nph_gpu_world_sleep_decision(NphGpuSolver *s, const uint32_t *island_of,
                                                     uint32_t island_count, const uint32_t *removed,
                                                     float time_to_sleep, uint8_t *sleep, uint32_t *split,
                                                     uint8_t *kinematic_sleep)
{
    if (s == nullptr || split == nullptr || (s->n > 0u && (island_of == nullptr || kinematic_sleep == nullptr)) ||
        (island_count > 0u && (removed == nullptr || sleep == nullptr))) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if (!s->uploaded) {
        return NPH_GPU_INVALID_STATE;
    }
    *split = NPH_GPU_NULL;
    cudaSetDevice(s->device);
    const uint32_t n = s->n;
    const uint32_t ni = island_count;
    uint32_t *d_of = nullptr, *d_removed = nullptr, *d_min = nullptr, *d_max = nullptr;
    uint8_t *d_sleep = nullptr, *d_kin = nullptr;
    uint32_t *d_bad = nullptr;
    unsigned long long *d_split = nullptr;
    const bool ok = dalloc(d_bad, 1) && dalloc(d_of, std::max<uint32_t>(n, 1u)) && dalloc(d_kin, std::max<uint32_t>(n, 1u)) &&
                    dalloc(d_removed, std::max<uint32_t>(ni, 1u)) && dalloc(d_min, std::max<uint32_t>(ni, 1u)) &&
                    dalloc(d_max, std::max<uint32_t>(ni, 1u)) && dalloc(d_sleep, std::max<uint32_t>(ni, 1u)) &&
                    dalloc(d_split, 1);
    NphGpuResult r = ok ? NPH_GPU_OK : NPH_GPU_OUT_OF_MEMORY;
    if (r == NPH_GPU_OK) {
        cudaMemsetAsync(d_bad, 0, sizeof(uint32_t), s->stream);
        if (n > 0u) {
            cudaMemcpyAsync(d_of, island_of, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s->stream);
        }
        if (ni > 0u) {
            cudaMemcpyAsync(d_removed, removed, sizeof(uint32_t) * ni, cudaMemcpyHostToDevice, s->stream);
        }
        k_island_init<<<blocks_for(std::max<uint32_t>(ni, 1u)), kBlock, 0, s->stream>>>(d_min, d_max, ni, d_split);
        if (n > 0u) {
            k_island_bounds<<<blocks_for(n), kBlock, 0, s->stream>>>(s->d_bodies, n, d_of, ni, time_to_sleep, d_min,
                                                                     d_max, d_kin, d_bad);
        }
        if (ni > 0u) {
            k_island_decide<<<blocks_for(ni), kBlock, 0, s->stream>>>(d_min, d_max, d_removed, ni, time_to_sleep,
                                                                      d_sleep, d_split);
            cudaMemcpyAsync(sleep, d_sleep, ni, cudaMemcpyDeviceToHost, s->stream);
        }
        if (n > 0u) {
            cudaMemcpyAsync(kinematic_sleep, d_kin, n, cudaMemcpyDeviceToHost, s->stream);
        }
        unsigned long long key = 0ull;
        uint32_t bad = 0u;
        cudaMemcpyAsync(&key, d_split, sizeof key, cudaMemcpyDeviceToHost, s->stream);
        cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, s->stream);
        r = check_cuda(cudaStreamSynchronize(s->stream));
        if (r == NPH_GPU_OK && bad != 0u) {
            r = NPH_GPU_INVALID_ARGUMENT; // an island index past island_count
        }
        if (r == NPH_GPU_OK && key != 0ull) {
            *split = 0xFFFFFFFFu - (uint32_t)(key & 0xFFFFFFFFull);
        }
    }
    cudaGetLastError();
    dfree(d_bad);
    dfree(d_of);
    dfree(d_kin);
    dfree(d_removed);
    dfree(d_min);
    dfree(d_max);
    dfree(d_sleep);
    dfree(d_split);
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_world_hit_events(NphGpuSolver *s, float threshold, NphGpuHitEvent *events,
                                                 uint32_t capacity, uint32_t *count)
{
    if (s == nullptr || count == nullptr || (capacity > 0u && events == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    *count = 0u;
    if (!s->uploaded) {
        return NPH_GPU_INVALID_STATE;
    }
    cudaSetDevice(s->device);
    return nph_hits_scan(s->d_contacts, s->m, threshold, s->stream, events, capacity, count);
}

NPH_GPU_API NphGpuResult nph_gpu_world_features(NphGpuSolver *s, const NphGpuWorldParams *params, float dt,
                                                float *features, float *scale, uint32_t *kind, uint64_t slots)
{
    if (s == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    NphGpuResult r = validate_soft_params(params, dt);
    if (r != NPH_GPU_OK) {
        return r;
    }
    if (!s->uploaded) {
        return NPH_GPU_INVALID_STATE;
    }
    const uint64_t need = 4ull * s->m;
    if (slots < need || (need > 0 && (features == nullptr || scale == nullptr || kind == nullptr))) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if (need == 0) {
        return NPH_GPU_OK;
    }
    cudaSetDevice(s->device);
    const StepConsts K = make_step_consts(*params, dt);
    float *d_feat = nullptr, *d_scale = nullptr;
    uint32_t *d_kind = nullptr;
    if (!dalloc(d_feat, need * NPH_GPU_MLP_INPUTS) || !dalloc(d_scale, need) || !dalloc(d_kind, need)) {
        dfree(d_feat);
        dfree(d_scale);
        dfree(d_kind);
        cudaGetLastError();
        return NPH_GPU_OUT_OF_MEMORY;
    }
    s->marks = nullptr;
    enqueue_prepare(s, K);
    k_all_features<<<blocks_for(s->m), 256, 0, s->stream>>>(dev_solver(s), s->m, feature_consts(K), d_feat,
                                                            d_scale, d_kind);
    cudaMemcpyAsync(features, d_feat, need * NPH_GPU_MLP_INPUTS * sizeof(float), cudaMemcpyDeviceToHost,
                    s->stream);
    cudaMemcpyAsync(scale, d_scale, need * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(kind, d_kind, need * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    r = check_cuda(cudaStreamSynchronize(s->stream));
    dfree(d_feat);
    dfree(d_scale);
    dfree(d_kind);
    if (r == NPH_GPU_OK) {
        r = read_error(s);
    }
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_world_converge(NphGpuSolver *s, const NphGpuWorldParams *params, float dt,
                                                uint32_t learned, float tolerance, uint32_t max_passes,
                                                float reference_residual, float *residuals, float *impulses,
                                                NphGpuConvergeStats *out)
{
    if (s == nullptr || out == nullptr || !(tolerance > 0.0f) || max_passes > 1000000u ||
        learned > NPH_GPU_START_GATED) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    NphGpuResult r = validate_soft_params(params, dt);
    if (r != NPH_GPU_OK) {
        return r;
    }
    if (!s->uploaded || (learned != NPH_GPU_START_PLAIN && s->mlp == nullptr)) {
        return NPH_GPU_INVALID_STATE;
    }
    std::memset(out, 0, sizeof *out);
    cudaSetDevice(s->device);
    const StepConsts K = make_step_consts(*params, dt);
    r = ensure_residuals(s, max_passes + 1u);
    if (r == NPH_GPU_OK) {
        r = ensure_learned(s);
    }
    if (r != NPH_GPU_OK) {
        return r;
    }
    const DevSolver S = dev_solver(s);
    const BodyArrays B = body_arrays(s);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemsetAsync(s->r_sq, 0, (max_passes + 1u) * sizeof(float), s->stream);
    cudaMemsetAsync(s->r_val, 0, (max_passes + 1u) * sizeof(float), s->stream);
    s->marks = nullptr;
    const uint32_t *done = s->r_state;
    const uint32_t res_blocks = std::max<uint32_t>(1u, std::min<uint32_t>(blocks_for(s->m), kResidualBlocks));
    // The start: prepare from the uploaded records, the cold points counted (and started by the
    // network when `net`), the first substep's velocity integration and warm start, and the
    // residual after it against `ref_in` (<= 0: its own). Prepare rebuilds every row the passes
    // use from the records, so a second start replaces the first.
    auto start = [&](bool net, float ref_in) {
        cudaMemsetAsync(s->r_state, 0, 4 * sizeof(uint32_t), s->stream);
        enqueue_prepare(s, K);
        if (s->m > 0u) {
            k_cold_features<<<blocks_for(s->m), 256, 0, s->stream>>>(S, s->m, feature_consts(K), s->l_feat,
                                                                     s->l_scale, s->l_slot, s->r_state + 2,
                                                                     net ? s->lcap : 0u, net ? 1u : 0u);
            if (net) {
                nph_mlp_forward_device_count(s->mlp, s->l_feat, s->r_state + 3, s->lcap, s->l_pred, s->stream);
                k_apply_predictions<<<blocks_for(s->lcap), 256, 0, s->stream>>>(S, s->l_pred, s->l_scale,
                                                                                s->l_slot, s->r_state + 2, s->lcap);
            }
        }
        k_integrate_velocity<<<blocks_for(s->n), kBlock, 0, s->stream>>>(B, s->n, K.h);
        enqueue_pass<kWarm>(s, K);
        k_residual<<<res_blocks, 256, 0, s->stream>>>(S, s->m, K.inv_h, s->r_part, done);
        k_residual_check<<<1, 256, 0, s->stream>>>(s->r_part, res_blocks, s->r_sq, s->r_val, s->r_ref, 0u,
                                                   tolerance, ref_in, s->r_state);
    };
    auto initial = [&](float &v) {
        cudaMemcpyAsync(&v, s->r_val, sizeof v, cudaMemcpyDeviceToHost, s->stream);
        return check_cuda(cudaStreamSynchronize(s->stream));
    };
    const bool use = learned != NPH_GPU_START_PLAIN && s->lcap > 0u;
    bool fell_back = false;
    float reference = reference_residual;
    cudaEventRecord(e0, s->stream);
    if (use && learned == NPH_GPU_START_GATED) {
        // The plain start is the fallback: the network's start is kept only when the plain
        // solver's residual after it is no larger than after the plain start.
        if (!(reference > 0.0f)) {
            start(false, 0.0f);
            r = initial(reference);
        }
        float learned_initial = 0.0f;
        if (r == NPH_GPU_OK) {
            start(true, reference);
            r = initial(learned_initial);
        }
        if (r == NPH_GPU_OK && learned_initial > reference) {
            start(false, reference);
            fell_back = true;
        }
    } else {
        start(use, reference);
    }
    // Passes in chunks of eight; the host stops issuing once the residual reached the tolerance.
    uint32_t state[4] = {0u, 0u, 0u, 0u};
    uint32_t issued = 0;
    while (r == NPH_GPU_OK && issued < max_passes) {
        cudaMemcpyAsync(state, s->r_state, sizeof state, cudaMemcpyDeviceToHost, s->stream);
        r = check_cuda(cudaStreamSynchronize(s->stream));
        if (r != NPH_GPU_OK || state[0] != 0u) {
            break;
        }
        const uint32_t chunk = std::min<uint32_t>(8u, max_passes - issued);
        for (uint32_t q = 0; q < chunk; ++q) {
            const uint32_t p = ++issued;
            enqueue_converge_pass(s, K, done);
            k_residual<<<res_blocks, 256, 0, s->stream>>>(S, s->m, K.inv_h, s->r_part, done);
            k_residual_check<<<1, 256, 0, s->stream>>>(s->r_part, res_blocks, s->r_sq, s->r_val, s->r_ref, p,
                                                       tolerance, reference, s->r_state);
        }
    }
    cudaEventRecord(e1, s->stream);
    float ref = 0.0f;
    cudaMemcpyAsync(state, s->r_state, sizeof state, cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(&ref, s->r_ref, sizeof ref, cudaMemcpyDeviceToHost, s->stream);
    std::vector<float> vals(max_passes + 1u, 0.0f);
    cudaMemcpyAsync(vals.data(), s->r_val, vals.size() * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
    if (r == NPH_GPU_OK) {
        r = check_cuda(cudaStreamSynchronize(s->stream));
    }
    float ms = 0.0f;
    if (r == NPH_GPU_OK) {
        cudaEventElapsedTime(&ms, e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r == NPH_GPU_OK && impulses != nullptr && s->m > 0u) {
        float *d_imp = nullptr;
        if (!dalloc(d_imp, 12ull * s->m)) {
            cudaGetLastError();
            return NPH_GPU_OUT_OF_MEMORY;
        }
        k_slot_impulses<<<blocks_for(s->m), 256, 0, s->stream>>>(S, s->m, d_imp);
        cudaMemcpyAsync(impulses, d_imp, 12ull * s->m * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
        r = check_cuda(cudaStreamSynchronize(s->stream));
        dfree(d_imp);
    }
    if (r == NPH_GPU_OK) {
        r = read_error(s);
    }
    if (r != NPH_GPU_OK) {
        return r;
    }
    const uint32_t passes = state[1];
    if (residuals != nullptr) {
        std::memcpy(residuals, vals.data(), (passes + 1u) * sizeof(float));
    }
    out->passes = passes;
    out->converged = state[0];
    out->cold_points = state[2];
    out->predicted_points = use && !fell_back ? std::min(state[3], s->lcap) : 0u;
    out->fell_back = fell_back ? 1u : 0u;
    out->initial_residual = vals[0];
    out->final_residual = vals[passes];
    out->reference_residual = ref;
    out->ms = ms;
    return NPH_GPU_OK;
}

NPH_GPU_API const char *nph_gpu_version(void)
{
    return "nepheline_b200 0.1.0 (sm_100a)";
}

} // extern "C"

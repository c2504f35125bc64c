// SPDX-License-Identifier: Apache-2.0
//
// Many independent worlds of uneven size solved in one persistent launch. Each block takes a
// whole world at a time from a queue sorted by size (largest first, so the last worlds taken
// are the smallest and the blocks finish together), and runs the world's entire solver stage
// (the stage list of phys_solve, solver.c:1032-1067) inside the block: every stage and every
// colour is a loop over the world's items by the block's threads, with a block barrier
// between them. No block ever waits on another, so no device-wide barrier or spin exists.
//
// Each world's arithmetic is the single-world solver's (the same device functions of
// bodies.cuh, contacts.cuh and joints.cuh on the world's slice of the arrays), so a world in
// a batch gives the same bits as the world solved alone. With `shared_velocities` the
// world's body velocities (the only body rows the constraint passes write) live in shared
// memory for the whole step.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "nepheline_b200.h"

#include "bodies.cuh"
#include "contacts.cuh"
#include "joints.cuh"

namespace nph {
namespace {

// One world of the batch on the device.
struct WorldSlice {
    uint32_t body_first;    // its records in the body record array
    uint32_t slot_first;    // its solver slots (n + 1 with its dummy) in the body rows
    uint32_t n;             // awake bodies
    uint32_t fixed_first;
    uint32_t nf;
    uint32_t contact_first; // manifolds, in the world's colour order
    uint32_t m;
    uint32_t joint_first;
    uint32_t nj;
    uint32_t driven;
    uint32_t cfirst[NPH_GPU_COLOR_SLOTS]; // world-relative
    uint32_t ccount[NPH_GPU_COLOR_SLOTS];
    uint32_t jfirst[NPH_GPU_COLOR_SLOTS];
    uint32_t jcount[NPH_GPU_COLOR_SLOTS];
};

struct BatchArgs {
    const WorldSlice *worlds;
    const uint32_t *order; // world indices, largest first
    uint32_t count;
    uint32_t *next;        // the queue's head
    uint32_t *err;
    NphGpuBody *bodies;
    const NphGpuBody *fixed;
    NphGpuContact *contacts;
    NphGpuJoint *joints;
    float4 *vel, *pos, *prm, *itg;
    uint4 *hdr;
    float4 *nrm;
    float *rest;
    float4 *pa, *pb, *pt, *pi;
    uint32_t mcap;
    float4 *jw;
    uint32_t jcap;
    uint32_t shared_velocities; // the world's velocities in shared memory
    uint32_t max_slots;         // shared velocity rows available (bodies + dummy)
};

enum Pass : int { kWarm = 0, kSolve = 1, kRelax = 2, kRestitution = 3 };

// The world's slice of the arrays: body indices in its rows are world-relative.
__device__ DevSolver world_solver(const BatchArgs &A, const WorldSlice &W, float4 *vel)
{
    DevSolver S;
    S.vel = vel;
    S.pos = A.pos + 2u * W.slot_first;
    S.prm = A.prm + 3u * W.slot_first;
    S.hdr = A.hdr + W.contact_first;
    S.nrm = A.nrm + W.contact_first;
    S.rest = A.rest + W.contact_first;
    S.pa = A.pa + W.contact_first;
    S.pb = A.pb + W.contact_first;
    S.pt = A.pt + W.contact_first;
    S.pi = A.pi + W.contact_first;
    S.mcap = A.mcap;
    S.jw = A.jw + W.joint_first;
    S.jcap = A.jcap;
    return S;
}

template <int P> __device__ void world_pass(const DevSolver &S, const WorldSlice &W, const StepConsts &K)
{
    const uint32_t o = NPH_GPU_OVERFLOW;
    // The overflow: one thread, its joints then its contacts in list order.
    if ((W.ccount[o] > 0u || (P != kRestitution && W.jcount[o] > 0u))) {
        if (threadIdx.x == 0) {
            if (P != kRestitution) {
                for (uint32_t j = 0; j < W.jcount[o]; ++j) {
                    const uint32_t jj = W.jfirst[o] + j;
                    if (P == kWarm) {
                        warm_joint(S, jj);
                    } else {
                        solve_joint<P == kSolve>(S, jj, K);
                    }
                }
            }
            for (uint32_t g = 0; g < W.ccount[o]; ++g) {
                const uint32_t gg = W.cfirst[o] + g;
                if (P == kWarm) {
                    warm_manifold(S, gg);
                } else if (P == kRestitution) {
                    restitution_manifold(S, gg, K);
                } else {
                    solve_manifold<P == kSolve>(S, gg, K);
                }
            }
        }
        __syncthreads();
    }
    for (uint32_t c = 0; c < NPH_GPU_COLORS; ++c) {
        const uint32_t jc = P == kRestitution ? 0u : W.jcount[c];
        const uint32_t cc = W.ccount[c];
        if (jc + cc == 0u) {
            continue;
        }
        for (uint32_t i = threadIdx.x; i < jc + cc; i += blockDim.x) {
            if (i < jc) {
                const uint32_t jj = W.jfirst[c] + i;
                if (P == kWarm) {
                    warm_joint(S, jj);
                } else {
                    solve_joint<P == kSolve>(S, jj, K);
                }
            } else {
                const uint32_t gg = W.cfirst[c] + (i - jc);
                if (P == kWarm) {
                    warm_manifold(S, gg);
                } else if (P == kRestitution) {
                    restitution_manifold(S, gg, K);
                } else {
                    solve_manifold<P == kSolve>(S, gg, K);
                }
            }
        }
        __syncthreads();
    }
}

// The largest point count of manifold g's eight-lane group in its world's colour list.
__device__ uint32_t world_group_points(const NphGpuContact *contacts, const WorldSlice &W, uint32_t g)
{
    uint32_t c = 0;
    while (c + 1u < NPH_GPU_COLOR_SLOTS && g >= W.cfirst[c] + W.ccount[c]) {
        ++c;
    }
    const uint32_t per = c == NPH_GPU_OVERFLOW ? 1u : 8u;
    const uint32_t start = W.cfirst[c] + ((g - W.cfirst[c]) / per) * per;
    const uint32_t end = min(start + per, W.cfirst[c] + W.ccount[c]);
    uint32_t gp = 0;
    for (uint32_t q = start; q < end; ++q) {
        const uint32_t pc = contacts[q].point_count;
        gp = pc <= NPH_GPU_MAX_POINTS && pc > gp ? pc : gp;
    }
    return gp;
}

__device__ void world_step(const BatchArgs &A, const WorldSlice &W, const StepConsts &K,
                           uint32_t substeps, float4 *shared_vel)
{
    const bool in_shared = A.shared_velocities != 0u && W.n + 1u <= A.max_slots;
    float4 *vel = in_shared ? shared_vel : A.vel + 2u * W.slot_first;
    const DevSolver S = world_solver(A, W, vel);
    const BodyArrays B{vel, A.pos + 2u * W.slot_first, A.prm + 3u * W.slot_first,
                       A.itg + 6u * W.slot_first};
    NphGpuBody *bodies = A.bodies + W.body_first;
    const NphGpuBody *fixed = A.fixed + W.fixed_first;
    NphGpuContact *contacts = A.contacts + W.contact_first;
    NphGpuJoint *joints = A.joints + W.joint_first;
    const uint32_t n = W.n;
    // prepare_body (solver.c:131-168), the dummy last.
    for (uint32_t i = threadIdx.x; i <= n; i += blockDim.x) {
        if (i < n) {
            prepare_body(B, i, bodies[i], K);
        } else {
            prepare_dummy(B, n);
        }
    }
    __syncthreads();
    // The joints and the manifolds (prepare_group, phys_joint_prepare).
    const uint32_t total = n + W.nf;
    for (uint32_t i = threadIdx.x; i < W.nj + W.m; i += blockDim.x) {
        if (i < W.nj) {
            const NphGpuJoint &jr = joints[i];
            if (jr.body_a >= total || jr.body_b >= total ||
                (jr.type != NPH_GPU_JOINT_BALL && jr.type != NPH_GPU_JOINT_HINGE)) {
                atomicOr(A.err, kErrBadJoint);
                for (uint32_t r = 0; r < kJointRows; ++r) {
                    S.jw[r * S.jcap + i] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                S.jw[kJrFrameA * S.jcap + i] = make_float4(0.f, 0.f, 0.f, 1.f);
                S.jw[kJrFrameB * S.jcap + i] = make_float4(0.f, 0.f, 0.f, 1.f);
                S.jw[kJrHead * S.jcap + i] =
                    make_float4(__uint_as_float(n), __uint_as_float(n), 0.f, 0.f);
                continue;
            }
            const NphGpuBody &a = jr.body_a < n ? bodies[jr.body_a] : fixed[jr.body_a - n];
            const NphGpuBody &b = jr.body_b < n ? bodies[jr.body_b] : fixed[jr.body_b - n];
            prepare_joint(S, i, jr, a, b, jr.body_a < n ? jr.body_a : n, jr.body_b < n ? jr.body_b : n,
                          K.h);
        } else {
            const uint32_t g = i - W.nj;
            const NphGpuContact &c = contacts[g];
            if (c.body_a >= total || c.body_b >= total) {
                atomicOr(A.err, kErrBadIndex);
                S.hdr[g] = make_uint4(n, n, 0u, 0u);
                continue;
            }
            if (c.point_count < 1u || c.point_count > NPH_GPU_MAX_POINTS) {
                atomicOr(A.err, kErrBadPoints);
                S.hdr[g] = make_uint4(n, n, 0u, 0u);
                continue;
            }
            const NphGpuBody &ra = c.body_a < n ? bodies[c.body_a] : fixed[c.body_a - n];
            const NphGpuBody &rb = c.body_b < n ? bodies[c.body_b] : fixed[c.body_b - n];
            const bool dyn_a = ra.type == NPH_GPU_BODY_DYNAMIC;
            const bool dyn_b = rb.type == NPH_GPU_BODY_DYNAMIC;
            S.nrm[g] = make_float4(c.normal[0], c.normal[1], c.normal[2], c.friction);
            S.rest[g] = c.restitution;
            prepare_manifold(S, g, c, c.body_a < n ? c.body_a : n, c.body_b < n ? c.body_b : n, dyn_a,
                             dyn_b, dyn_a ? ra.inv_mass : 0.0f, dyn_b ? rb.inv_mass : 0.0f,
                             world_group_points(contacts, W, g));
        }
    }
    __syncthreads();
    for (uint32_t sub = 0; sub < substeps; ++sub) {
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            integrate_velocity(B, i, K.h);
        }
        __syncthreads();
        world_pass<kWarm>(S, W, K);
        world_pass<kSolve>(S, W, K);
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            integrate_position(B, i, K.h);
        }
        __syncthreads();
        world_pass<kRelax>(S, W, K);
    }
    world_pass<kRestitution>(S, W, K);
    // store_group, the joints' impulses, finalize_body.
    for (uint32_t g = threadIdx.x; g < W.m; g += blockDim.x) {
        store_manifold(S, g, contacts[g]);
    }
    for (uint32_t j = threadIdx.x; j < W.nj; j += blockDim.x) {
        store_joint(S, j, joints[j]);
    }
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        finalize_body(B, i, bodies[i], K.dt);
    }
    __syncthreads();
    // post_finalize's driven joints (solver.c:851-857).
    if (W.driven > 0u) {
        for (uint32_t j = threadIdx.x; j < W.nj; j += blockDim.x) {
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
    }
    __syncthreads();
}

template <int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
k_worlds(BatchArgs A, StepConsts K, uint32_t substeps)
{
    extern __shared__ float4 shared_vel[];
    __shared__ uint32_t taken;
    for (;;) {
        if (threadIdx.x == 0) {
            taken = atomicAdd(A.next, 1u);
        }
        __syncthreads();
        const uint32_t q = taken;
        __syncthreads();
        if (q >= A.count) {
            return;
        }
        world_step(A, A.worlds[A.order[q]], K, substeps, shared_vel);
    }
}

struct BatchConfig {
    uint32_t threads, min_blocks;
};
constexpr BatchConfig kBatchConfigs[] = {{128, 4}, {256, 2}, {256, 1}, {512, 1}, {1024, 1}};
constexpr uint32_t kBatchConfigCount = sizeof(kBatchConfigs) / sizeof(kBatchConfigs[0]);

} // namespace

StepConsts make_step_consts(const NphGpuWorldParams &p, float dt);

} // namespace nph

using namespace nph;

struct NphGpuBatch {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool use_graph = true;
    uint32_t config = 1;
    uint32_t shared_velocities = 1;
    uint32_t blocks_per_sm = 0; // resident blocks of the chosen kernel (0: not yet known)
    int sms = 148;
    // Device arrays.
    NphGpuBody *d_bodies = nullptr;
    NphGpuBody *d_fixed = nullptr;
    NphGpuContact *d_contacts = nullptr;
    NphGpuJoint *d_joints = nullptr;
    float4 *vel = nullptr, *pos = nullptr, *prm = nullptr, *itg = nullptr;
    uint4 *hdr = nullptr;
    float4 *nrm = nullptr;
    float *rest = nullptr;
    float4 *pa = nullptr, *pb = nullptr, *pt = nullptr, *pi = nullptr;
    float4 *jw = nullptr;
    WorldSlice *d_worlds = nullptr;
    uint32_t *d_order = nullptr;
    uint32_t *d_counters = nullptr; // [0] queue head, [1] error bits
    uint32_t *h_counters = nullptr;
    // Sizes.
    uint32_t world_count = 0;
    uint64_t bodies = 0, slots = 0, fixed = 0, contacts = 0, joints = 0;
    uint64_t max_world_slots = 0;
    std::vector<WorldSlice> worlds;
    // The step graph.
    cudaGraphExec_t graph = nullptr;
    bool graph_valid = false;
    StepConsts graph_consts{};
    uint32_t graph_substeps = 0;
    size_t bytes_held = 0;
};

namespace {

template <typename T> void bfree(T *&p)
{
    if (p != nullptr) {
        cudaFree(p);
        p = nullptr;
    }
}

template <typename T> bool balloc(T *&p, uint64_t count)
{
    bfree(p);
    return cudaMalloc((void **)&p, std::max<uint64_t>(count, 1) * sizeof(T)) == cudaSuccess;
}

void drop_batch_graph(NphGpuBatch *b)
{
    if (b->graph != nullptr) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->graph_valid = false;
}

void free_arrays(NphGpuBatch *b)
{
    drop_batch_graph(b);
    bfree(b->d_bodies);
    bfree(b->d_fixed);
    bfree(b->d_contacts);
    bfree(b->d_joints);
    bfree(b->vel);
    bfree(b->pos);
    bfree(b->prm);
    bfree(b->itg);
    bfree(b->hdr);
    bfree(b->nrm);
    bfree(b->rest);
    bfree(b->pa);
    bfree(b->pb);
    bfree(b->pt);
    bfree(b->pi);
    bfree(b->jw);
    bfree(b->d_worlds);
    bfree(b->d_order);
    b->world_count = 0;
}

NphGpuResult cuda_result(cudaError_t e)
{
    if (e == cudaSuccess) {
        return NPH_GPU_OK;
    }
    return e == cudaErrorMemoryAllocation ? NPH_GPU_OUT_OF_MEMORY : NPH_GPU_DEVICE_LOST;
}

size_t shared_bytes(const NphGpuBatch *b)
{
    if (b->shared_velocities == 0u) {
        return 0;
    }
    // Two velocity rows per slot, up to the largest world, within 160 KiB.
    const uint64_t want = 2ull * b->max_world_slots * sizeof(float4);
    return (size_t)std::min<uint64_t>(want, 160ull << 10);
}

BatchArgs batch_args(const NphGpuBatch *b)
{
    BatchArgs A;
    A.worlds = b->d_worlds;
    A.order = b->d_order;
    A.count = b->world_count;
    A.next = b->d_counters;
    A.err = b->d_counters + 1;
    A.bodies = b->d_bodies;
    A.fixed = b->d_fixed;
    A.contacts = b->d_contacts;
    A.joints = b->d_joints;
    A.vel = b->vel;
    A.pos = b->pos;
    A.prm = b->prm;
    A.itg = b->itg;
    A.hdr = b->hdr;
    A.nrm = b->nrm;
    A.rest = b->rest;
    A.pa = b->pa;
    A.pb = b->pb;
    A.pt = b->pt;
    A.pi = b->pi;
    A.mcap = (uint32_t)std::max<uint64_t>(b->contacts, 1);
    A.jw = b->jw;
    A.jcap = (uint32_t)std::max<uint64_t>(b->joints, 1);
    A.shared_velocities = shared_bytes(b) > 0 ? 1u : 0u;
    A.max_slots = (uint32_t)(shared_bytes(b) / (2 * sizeof(float4)));
    return A;
}

template <int T, int M> void configure_kernel(size_t smem)
{
    cudaFuncSetAttribute(k_worlds<T, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int T, int M> uint32_t resident(size_t smem)
{
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_worlds<T, M>, T, smem);
    return (uint32_t)std::max(blocks, 1);
}

// The chosen kernel's shared-memory limit and residency (outside any stream capture).
void configure_batch_kernel(NphGpuBatch *b)
{
    const size_t smem = shared_bytes(b);
    uint32_t per_sm = 1;
    switch (b->config) {
    case 0: configure_kernel<128, 4>(smem); per_sm = resident<128, 4>(smem); break;
    case 1: configure_kernel<256, 2>(smem); per_sm = resident<256, 2>(smem); break;
    case 2: configure_kernel<256, 1>(smem); per_sm = resident<256, 1>(smem); break;
    case 3: configure_kernel<512, 1>(smem); per_sm = resident<512, 1>(smem); break;
    default: configure_kernel<1024, 1>(smem); per_sm = resident<1024, 1>(smem); break;
    }
    b->blocks_per_sm = per_sm;
}

void enqueue_batch_step(NphGpuBatch *b, const StepConsts &K, uint32_t substeps)
{
    const BatchArgs A = batch_args(b);
    const size_t smem = shared_bytes(b);
    cudaMemsetAsync(b->d_counters, 0, sizeof(uint32_t), b->stream);
    const uint32_t grid =
        std::max<uint32_t>(1, std::min<uint32_t>(b->world_count, b->blocks_per_sm * (uint32_t)b->sms));
    switch (b->config) {
    case 0: k_worlds<128, 4><<<grid, 128, smem, b->stream>>>(A, K, substeps); break;
    case 1: k_worlds<256, 2><<<grid, 256, smem, b->stream>>>(A, K, substeps); break;
    case 2: k_worlds<256, 1><<<grid, 256, smem, b->stream>>>(A, K, substeps); break;
    case 3: k_worlds<512, 1><<<grid, 512, smem, b->stream>>>(A, K, substeps); break;
    default: k_worlds<1024, 1><<<grid, 1024, smem, b->stream>>>(A, K, substeps); break;
    }
}

NphGpuResult launch_batch_step(NphGpuBatch *b, const StepConsts &K, uint32_t substeps)
{
    if (!b->use_graph) {
        configure_batch_kernel(b);
        enqueue_batch_step(b, K, substeps);
        return cuda_result(cudaGetLastError());
    }
    if (!b->graph_valid || b->graph_substeps != substeps || std::memcmp(&b->graph_consts, &K, sizeof K) != 0) {
        drop_batch_graph(b);
        configure_batch_kernel(b);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            return cuda_result(e);
        }
        enqueue_batch_step(b, K, substeps);
        e = cudaStreamEndCapture(b->stream, &g);
        if (e != cudaSuccess) {
            return cuda_result(e);
        }
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b->graph = nullptr;
            return cuda_result(e);
        }
        b->graph_consts = K;
        b->graph_substeps = substeps;
        b->graph_valid = true;
    }
    return cuda_result(cudaGraphLaunch(b->graph, b->stream));
}

NphGpuResult check_world(const NphGpuWorldView &v)
{
    uint64_t nc = 0, nj = 0;
    for (uint32_t c = 0; c < NPH_GPU_COLOR_SLOTS; ++c) {
        nc += v.contact_color_counts[c];
        nj += v.joint_color_counts[c];
    }
    if (nc != v.contact_count || nj != v.joint_count) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if ((v.body_count > 0 && v.bodies == nullptr) || (v.fixed_count > 0 && v.fixed_bodies == nullptr) ||
        (v.contact_count > 0 && v.contacts == nullptr) || (v.joint_count > 0 && v.joints == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    for (uint32_t j = 0; j < v.joint_count; ++j) {
        if (v.joints[j].type != NPH_GPU_JOINT_BALL && v.joints[j].type != NPH_GPU_JOINT_HINGE) {
            return NPH_GPU_UNSUPPORTED;
        }
    }
    return NPH_GPU_OK;
}

} // namespace

extern "C" {

NPH_GPU_API NphGpuResult nph_gpu_batch_create(const NphGpuSolverDesc *desc, NphGpuBatch **out)
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
    NphGpuBatch *b = new (std::nothrow) NphGpuBatch();
    if (b == nullptr) {
        return NPH_GPU_OUT_OF_MEMORY;
    }
    b->device = d.device;
    b->use_graph = d.use_graph != 0u;
    cudaSetDevice(d.device);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, d.device);
    if (d.stream != nullptr) {
        b->stream = (cudaStream_t)d.stream;
    } else if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess) {
        b->own_stream = true;
    } else {
        delete b;
        return NPH_GPU_DEVICE_LOST;
    }
    if (!balloc(b->d_counters, 4) ||
        cudaMallocHost((void **)&b->h_counters, 4 * sizeof(uint32_t)) != cudaSuccess) {
        nph_gpu_batch_destroy(b);
        return NPH_GPU_OUT_OF_MEMORY;
    }
    *out = b;
    return NPH_GPU_OK;
}

NPH_GPU_API void nph_gpu_batch_destroy(NphGpuBatch *b)
{
    if (b == nullptr) {
        return;
    }
    cudaSetDevice(b->device);
    if (b->stream != nullptr) {
        cudaStreamSynchronize(b->stream);
    }
    free_arrays(b);
    bfree(b->d_counters);
    if (b->h_counters != nullptr) {
        cudaFreeHost(b->h_counters);
    }
    if (b->own_stream && b->stream != nullptr) {
        cudaStreamDestroy(b->stream);
    }
    delete b;
}

NPH_GPU_API void *nph_gpu_batch_stream(const NphGpuBatch *b)
{
    return b != nullptr ? (void *)b->stream : nullptr;
}

NPH_GPU_API NphGpuResult nph_gpu_batch_upload(NphGpuBatch *b, const NphGpuWorldView *worlds,
                                              uint32_t count)
{
    if (b == nullptr || (count > 0 && worlds == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    for (uint32_t w = 0; w < count; ++w) {
        const NphGpuResult r = check_world(worlds[w]);
        if (r != NPH_GPU_OK) {
            return r;
        }
    }
    cudaSetDevice(b->device);
    // The slices, then the arrays sized to the batch.
    std::vector<WorldSlice> slices(count);
    uint64_t bodies = 0, slots = 0, fixed = 0, contacts = 0, joints = 0, max_slots = 0;
    for (uint32_t w = 0; w < count; ++w) {
        const NphGpuWorldView &v = worlds[w];
        WorldSlice &s = slices[w];
        std::memset(&s, 0, sizeof s);
        s.body_first = (uint32_t)bodies;
        s.slot_first = (uint32_t)slots;
        s.n = v.body_count;
        s.fixed_first = (uint32_t)fixed;
        s.nf = v.fixed_count;
        s.contact_first = (uint32_t)contacts;
        s.m = v.contact_count;
        s.joint_first = (uint32_t)joints;
        s.nj = v.joint_count;
        uint32_t cf = 0, jf = 0;
        for (uint32_t c = 0; c < NPH_GPU_COLOR_SLOTS; ++c) {
            s.cfirst[c] = cf;
            s.ccount[c] = v.contact_color_counts[c];
            s.jfirst[c] = jf;
            s.jcount[c] = v.joint_color_counts[c];
            cf += s.ccount[c];
            jf += s.jcount[c];
        }
        for (uint32_t j = 0; j < v.joint_count; ++j) {
            const NphGpuJoint &jr = v.joints[j];
            s.driven += (jr.type == NPH_GPU_JOINT_HINGE && jr.u.hinge.enable_motor != 0u &&
                         jr.u.hinge.motor_speed != 0.0f && jr.u.hinge.max_motor_torque > 0.0f)
                            ? 1u
                            : 0u;
        }
        bodies += v.body_count;
        slots += v.body_count + 1u;
        fixed += v.fixed_count;
        contacts += v.contact_count;
        joints += v.joint_count;
        max_slots = std::max<uint64_t>(max_slots, v.body_count + 1u);
    }
    if (slots >= 0xFFFFFFF0ull || contacts >= 0xFFFFFFF0ull || joints >= 0xFFFFFFF0ull) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    free_arrays(b);
    bool ok = balloc(b->d_bodies, bodies) && balloc(b->d_fixed, fixed) &&
              balloc(b->d_contacts, contacts) && balloc(b->d_joints, joints) &&
              balloc(b->vel, 2 * slots) && balloc(b->pos, 2 * slots) && balloc(b->prm, 3 * slots) &&
              balloc(b->itg, 6 * slots) && balloc(b->hdr, contacts) && balloc(b->nrm, contacts) &&
              balloc(b->rest, contacts) && balloc(b->pa, 4 * std::max<uint64_t>(contacts, 1)) &&
              balloc(b->pb, 4 * std::max<uint64_t>(contacts, 1)) &&
              balloc(b->pt, 4 * std::max<uint64_t>(contacts, 1)) &&
              balloc(b->pi, 4 * std::max<uint64_t>(contacts, 1)) &&
              balloc(b->jw, (uint64_t)kJointRows * std::max<uint64_t>(joints, 1)) &&
              balloc(b->d_worlds, count) && balloc(b->d_order, count);
    if (!ok) {
        free_arrays(b);
        cudaGetLastError();
        return NPH_GPU_OUT_OF_MEMORY;
    }
    b->world_count = count;
    b->bodies = bodies;
    b->slots = slots;
    b->fixed = fixed;
    b->contacts = contacts;
    b->joints = joints;
    b->max_world_slots = max_slots;
    b->worlds = slices;
    // Largest first: the work of a world grows with its manifolds, joints and bodies.
    std::vector<uint32_t> order(count);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        const uint64_t wx = 4ull * slices[x].m + 3ull * slices[x].nj + slices[x].n;
        const uint64_t wy = 4ull * slices[y].m + 3ull * slices[y].nj + slices[y].n;
        return wx > wy;
    });
    cudaMemcpyAsync(b->d_worlds, slices.data(), sizeof(WorldSlice) * count, cudaMemcpyHostToDevice, b->stream);
    cudaMemcpyAsync(b->d_order, order.data(), sizeof(uint32_t) * count, cudaMemcpyHostToDevice, b->stream);
    for (uint32_t w = 0; w < count; ++w) {
        const NphGpuWorldView &v = worlds[w];
        const WorldSlice &s = slices[w];
        if (v.body_count > 0) {
            cudaMemcpyAsync(b->d_bodies + s.body_first, v.bodies, sizeof(NphGpuBody) * v.body_count,
                            cudaMemcpyHostToDevice, b->stream);
        }
        if (v.fixed_count > 0) {
            cudaMemcpyAsync(b->d_fixed + s.fixed_first, v.fixed_bodies, sizeof(NphGpuBody) * v.fixed_count,
                            cudaMemcpyHostToDevice, b->stream);
        }
        if (v.contact_count > 0) {
            cudaMemcpyAsync(b->d_contacts + s.contact_first, v.contacts,
                            sizeof(NphGpuContact) * v.contact_count, cudaMemcpyHostToDevice, b->stream);
        }
        if (v.joint_count > 0) {
            cudaMemcpyAsync(b->d_joints + s.joint_first, v.joints, sizeof(NphGpuJoint) * v.joint_count,
                            cudaMemcpyHostToDevice, b->stream);
        }
    }
    cudaMemsetAsync(b->d_counters, 0, 4 * sizeof(uint32_t), b->stream);
    return cuda_result(cudaStreamSynchronize(b->stream));
}

NPH_GPU_API NphGpuResult nph_gpu_batch_step_async(NphGpuBatch *b, const NphGpuWorldParams *params,
                                                  float dt, uint32_t steps)
{
    if (b == nullptr || params == nullptr || !(dt > 0.0f) || params->substeps == 0u ||
        params->substeps > 64u) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if (params->solver != NPH_GPU_SOLVER_SOFT_STEP || params->enable_continuous != 0u) {
        return NPH_GPU_UNSUPPORTED;
    }
    if (b->world_count == 0) {
        return NPH_GPU_OK;
    }
    cudaSetDevice(b->device);
    const StepConsts K = make_step_consts(*params, dt);
    NphGpuResult r = NPH_GPU_OK;
    for (uint32_t i = 0; i < steps && r == NPH_GPU_OK; ++i) {
        r = launch_batch_step(b, K, params->substeps);
    }
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_batch_download(NphGpuBatch *b, NphGpuWorldView *worlds, uint32_t count)
{
    if (b == nullptr || count != b->world_count || (count > 0 && worlds == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(b->device);
    cudaMemcpyAsync(b->h_counters, b->d_counters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream);
    NphGpuResult r = cuda_result(cudaStreamSynchronize(b->stream));
    if (r != NPH_GPU_OK) {
        return r;
    }
    if (b->h_counters[1] != 0u) {
        return NPH_GPU_INVALID_ARGUMENT; // a malformed record: nothing written back
    }
    for (uint32_t w = 0; w < count; ++w) {
        NphGpuWorldView &v = worlds[w];
        const WorldSlice &s = b->worlds[w];
        if (v.body_count != s.n || v.contact_count != s.m || v.joint_count != s.nj) {
            return NPH_GPU_INVALID_STATE;
        }
    }
    for (uint32_t w = 0; w < count; ++w) {
        NphGpuWorldView &v = worlds[w];
        const WorldSlice &s = b->worlds[w];
        if (s.n > 0) {
            cudaMemcpyAsync(v.bodies, b->d_bodies + s.body_first, sizeof(NphGpuBody) * s.n,
                            cudaMemcpyDeviceToHost, b->stream);
        }
        if (s.m > 0) {
            cudaMemcpyAsync(v.contacts, b->d_contacts + s.contact_first, sizeof(NphGpuContact) * s.m,
                            cudaMemcpyDeviceToHost, b->stream);
        }
        if (s.nj > 0) {
            cudaMemcpyAsync(v.joints, b->d_joints + s.joint_first, sizeof(NphGpuJoint) * s.nj,
                            cudaMemcpyDeviceToHost, b->stream);
        }
    }
    return cuda_result(cudaStreamSynchronize(b->stream));
}

NPH_GPU_API NphGpuResult nph_gpu_phys_solve_worlds(NphGpuBatch *b, const NphGpuWorldParams *params,
                                                   float dt, NphGpuWorldView *worlds, uint32_t count)
{
    NphGpuResult r = nph_gpu_batch_upload(b, worlds, count);
    if (r == NPH_GPU_OK) {
        r = nph_gpu_batch_step_async(b, params, dt, 1);
    }
    if (r == NPH_GPU_OK) {
        r = nph_gpu_batch_download(b, worlds, count);
    }
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_batch_set_config(NphGpuBatch *b, uint32_t config,
                                                  uint32_t shared_velocities)
{
    if (b == nullptr || config >= kBatchConfigCount) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    b->config = config;
    b->shared_velocities = shared_velocities != 0u ? 1u : 0u;
    drop_batch_graph(b);
    return NPH_GPU_OK;
}

NPH_GPU_API uint32_t nph_gpu_batch_config_count(void) { return kBatchConfigCount; }

NPH_GPU_API NphGpuResult nph_gpu_batch_autotune(NphGpuBatch *b, const NphGpuWorldParams *params,
                                                float dt, uint32_t rounds, NphGpuBatchTuning *out)
{
    if (b == nullptr || params == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if (b->world_count == 0) {
        return NPH_GPU_INVALID_STATE;
    }
    cudaSetDevice(b->device);
    const StepConsts K = make_step_consts(*params, dt);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    uint32_t best_config = b->config, best_shared = b->shared_velocities;
    rounds = rounds == 0u ? 1u : rounds;
    NphGpuResult r = NPH_GPU_OK;
    for (uint32_t shared = 0; shared < 2u && r == NPH_GPU_OK; ++shared) {
        for (uint32_t c = 0; c < kBatchConfigCount && r == NPH_GPU_OK; ++c) {
            b->config = c;
            b->shared_velocities = shared;
            drop_batch_graph(b);
            r = launch_batch_step(b, K, params->substeps); // builds the graph, warms up
            cudaEventRecord(e0, b->stream);
            for (uint32_t i = 0; i < rounds && r == NPH_GPU_OK; ++i) {
                r = launch_batch_step(b, K, params->substeps);
            }
            cudaEventRecord(e1, b->stream);
            if (r == NPH_GPU_OK) {
                r = cuda_result(cudaEventSynchronize(e1));
            }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (r == NPH_GPU_OK && ms < best) {
                best = ms;
                best_config = c;
                best_shared = shared;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->config = best_config;
    b->shared_velocities = best_shared;
    drop_batch_graph(b);
    if (out != nullptr) {
        out->config = best_config;
        out->threads = kBatchConfigs[best_config].threads;
        out->shared_velocities = best_shared;
        out->ms_per_step = best / (float)rounds;
    }
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_batch_info(const NphGpuBatch *b, NphGpuBatchInfo *out)
{
    if (b == nullptr || out == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    std::memset(out, 0, sizeof *out);
    out->worlds = b->world_count;
    out->bodies = b->bodies;
    out->manifolds = b->contacts;
    out->joints = b->joints;
    out->config = b->config;
    out->threads = kBatchConfigs[b->config].threads;
    out->shared_velocities = b->shared_velocities;
    out->blocks_per_sm = b->blocks_per_sm;
    return NPH_GPU_OK;
}

} // extern "C"

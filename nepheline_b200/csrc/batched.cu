// SPDX-License-Identifier: Apache-2.0
//
// Many independent worlds of uneven size solved in one persistent launch. Worlds are taken
// whole from two queues sorted by size (largest first, so the last worlds taken are the
// smallest and the blocks finish together): first the large worlds, each by a whole block,
// then the small ones, each by a single warp. A team (the block or the warp) runs the
// world's entire solver stage (the stage list of phys_solve, solver.c:1032-1067): every
// stage and every colour is a loop over the world's items by the team's threads, with a team
// barrier between them. No team ever waits on another, so no device-wide barrier or spin
// exists. A warp team lets one SM overlap many small worlds, whose colours hold too few
// constraints to occupy a block.
//
// Each world's arithmetic is the single-world solver's (the same device functions of
// bodies.cuh, contacts.cuh and joints.cuh on the world's slice of the arrays), so a world in
// a batch gives the same bits as the world solved alone. Each item of a stage is a separate
// non-inlined function, so that the register allocation of one stage does not constrain
// another. With shared velocities, a world's body velocities (the only body rows the
// constraint passes write) live in the team's shared memory for the whole step when they fit.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <new>
#include <numeric>
#include <thread>
#include <vector>

#include "nepheline_b200.h"
#include "solver_link.h"

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
    uint32_t row_joints;    // slider, 6-DOF and distance joints
    uint32_t cfirst[NPH_GPU_COLOR_SLOTS]; // world-relative
    uint32_t ccount[NPH_GPU_COLOR_SLOTS];
    uint32_t jfirst[NPH_GPU_COLOR_SLOTS];
    uint32_t jcount[NPH_GPU_COLOR_SLOTS];
};

// Team sizes: a block of B warps runs its worlds in teams of B, B/2, ..., 1 warps (size
// class c: B >> c warps), each team on its own named barrier.
constexpr uint32_t kMaxClasses = 5; // 16, 8, 4, 2, 1 warps

struct BatchArgs {
    const WorldSlice *worlds;
    const uint32_t *order; // world indices: the worlds of size class 0, then class 1, ...
    uint32_t count;
    uint32_t class_first[kMaxClasses]; // where each class's worlds start in `order`
    uint32_t class_count[kMaxClasses];
    uint32_t classes;
    uint32_t *heads;       // one queue head per class
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
    uint32_t block_slots; // velocity slots (two rows each) in a block's shared memory
};

enum Pass : int { kWarm = 0, kSolve = 1, kRelax = 2, kRestitution = 3 };

// A team of threads that runs one world: a warp (synchronised by __syncwarp) or several
// warps on a named barrier of their own (barrier.sync id, threads), so teams of one block work
// on different worlds without waiting for each other.
struct Team {
    uint32_t rank, size, barrier; // barrier 0: the team is one warp

    __device__ void sync() const
    {
        if (barrier == 0u) {
            __syncwarp();
        } else {
            // The non-aligned form: a warp's threads may arrive after divergent item loops.
            asm volatile("barrier.sync %0, %1;" ::"r"(barrier), "r"(size) : "memory");
        }
    }
};

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
    S.cmask = nullptr;
    S.done = nullptr;
    S.jrank = nullptr;
    return S;
}

// ---- the items of each stage, one non-inlined function each ----

template <int P> __device__ __noinline__ void joint_item(const DevSolver &S, uint32_t j, const StepConsts &K)
{
    if (P == kWarm) {
        warm_joint(S, j);
    } else {
        solve_joint<P == kSolve>(S, j, K);
    }
}

template <int P>
__device__ __noinline__ void manifold_item(const DevSolver &S, uint32_t g, const StepConsts &K)
{
    if (P == kWarm) {
        warm_manifold(S, g);
    } else if (P == kRestitution) {
        restitution_manifold(S, g, K);
    } else {
        solve_manifold<P == kSolve>(S, g, K);
    }
}

__device__ __noinline__ void body_prepare_item(const BodyArrays &B, uint32_t i, uint32_t n,
                                               const NphGpuBody *bodies, const StepConsts &K)
{
    if (i < n) {
        prepare_body(B, i, bodies[i], K);
    } else {
        prepare_dummy(B, n);
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

// phys_joint_prepare for joint i of the world, or the neutral rows of a malformed one.
__device__ __noinline__ void joint_prepare_item(const DevSolver &S, const WorldSlice &W, uint32_t i,
                                                const NphGpuJoint *joints, const NphGpuBody *bodies,
                                                const NphGpuBody *fixed, float h, uint32_t *err)
{
    const uint32_t n = W.n, total = W.n + W.nf;
    const NphGpuJoint &jr = joints[i];
    if (jr.body_a >= total || jr.body_b >= total || nph_joint_check(&jr) != NPH_GPU_OK) {
        atomicOr(err, kErrBadJoint);
        for (uint32_t r = 0; r < kJointRows; ++r) {
            S.jw[r * S.jcap + i] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        S.jw[kJrFrameA * S.jcap + i] = make_float4(0.f, 0.f, 0.f, 1.f);
        S.jw[kJrFrameB * S.jcap + i] = make_float4(0.f, 0.f, 0.f, 1.f);
        S.jw[kJrHead * S.jcap + i] = make_float4(__uint_as_float(n), __uint_as_float(n), 0.f, 0.f);
        return;
    }
    const NphGpuBody &a = jr.body_a < n ? bodies[jr.body_a] : fixed[jr.body_a - n];
    const NphGpuBody &b = jr.body_b < n ? bodies[jr.body_b] : fixed[jr.body_b - n];
    prepare_joint(S, i, jr, a, b, jr.body_a < n ? jr.body_a : n, jr.body_b < n ? jr.body_b : n, h);
}

// prepare_group for manifold g of the world, or the neutral header of a malformed one.
__device__ __noinline__ void manifold_prepare_item(const DevSolver &S, const WorldSlice &W, uint32_t g,
                                                   const NphGpuContact *contacts, const NphGpuBody *bodies,
                                                   const NphGpuBody *fixed, uint32_t *err)
{
    const uint32_t n = W.n, total = W.n + W.nf;
    const NphGpuContact &c = contacts[g];
    if (c.body_a >= total || c.body_b >= total) {
        atomicOr(err, kErrBadIndex);
        S.hdr[g] = make_uint4(n, n, 0u, 0u);
        return;
    }
    if (c.point_count < 1u || c.point_count > NPH_GPU_MAX_POINTS) {
        atomicOr(err, kErrBadPoints);
        S.hdr[g] = make_uint4(n, n, 0u, 0u);
        return;
    }
    const NphGpuBody &ra = c.body_a < n ? bodies[c.body_a] : fixed[c.body_a - n];
    const NphGpuBody &rb = c.body_b < n ? bodies[c.body_b] : fixed[c.body_b - n];
    const bool dyn_a = ra.type == NPH_GPU_BODY_DYNAMIC;
    const bool dyn_b = rb.type == NPH_GPU_BODY_DYNAMIC;
    S.nrm[g] = make_float4(c.normal[0], c.normal[1], c.normal[2], c.friction);
    S.rest[g] = c.restitution;
    prepare_manifold(S, g, c, c.body_a < n ? c.body_a : n, c.body_b < n ? c.body_b : n, dyn_a, dyn_b,
                     dyn_a ? ra.inv_mass : 0.0f, dyn_b ? rb.inv_mass : 0.0f,
                     world_group_points(contacts, W, g));
}

__device__ __noinline__ void finalize_item(const BodyArrays &B, uint32_t i, NphGpuBody *bodies, float dt)
{
    finalize_body(B, i, bodies[i], dt);
}

__device__ __noinline__ void store_manifold_item(const DevSolver &S, uint32_t g, NphGpuContact *contacts)
{
    store_manifold(S, g, contacts[g]);
}

__device__ __noinline__ void store_joint_item(const DevSolver &S, uint32_t j, NphGpuJoint *joints)
{
    store_joint(S, j, joints[j]);
}

template <int P> __device__ void world_pass(const Team &T, const DevSolver &S, const WorldSlice &W, const StepConsts &K)
{
    const uint32_t o = NPH_GPU_OVERFLOW;
    // The overflow: one thread, its joints then its contacts in list order.
    const uint32_t oj = P == kRestitution ? 0u : W.jcount[o];
    if (W.ccount[o] > 0u || oj > 0u) {
        if (T.rank == 0u) {
            for (uint32_t j = 0; j < oj; ++j) {
                joint_item<P>(S, W.jfirst[o] + j, K);
            }
            for (uint32_t g = 0; g < W.ccount[o]; ++g) {
                manifold_item<P>(S, W.cfirst[o] + g, K);
            }
        }
        T.sync();
    }
    for (uint32_t c = 0; c < NPH_GPU_COLORS; ++c) {
        const uint32_t jc = P == kRestitution ? 0u : W.jcount[c];
        const uint32_t cc = W.ccount[c];
        if (jc + cc == 0u) {
            continue;
        }
        for (uint32_t i = T.rank; i < jc + cc; i += T.size) {
            if (i < jc) {
                joint_item<P>(S, W.jfirst[c] + i, K);
            } else {
                manifold_item<P>(S, W.cfirst[c] + (i - jc), K);
            }
        }
        T.sync();
    }
}

__device__ void world_step(const Team &T, const BatchArgs &A, const WorldSlice &W, const StepConsts &K,
                           uint32_t substeps, float4 *shared_vel, uint32_t shared_slots)
{
    const bool in_shared = W.n + 1u <= shared_slots;
    float4 *vel = in_shared ? shared_vel : A.vel + 2u * W.slot_first;
    const DevSolver S = world_solver(A, W, vel);
    const BodyArrays B{vel, A.pos + 2u * W.slot_first, A.prm + 3u * W.slot_first, A.itg + 6u * W.slot_first};
    NphGpuBody *bodies = A.bodies + W.body_first;
    const NphGpuBody *fixed = A.fixed + W.fixed_first;
    NphGpuContact *contacts = A.contacts + W.contact_first;
    NphGpuJoint *joints = A.joints + W.joint_first;
    const uint32_t n = W.n;
    // prepare_body (solver.c:131-168), the dummy last.
    for (uint32_t i = T.rank; i <= n; i += T.size) {
        body_prepare_item(B, i, n, bodies, K);
    }
    T.sync();
    // The joints and the manifolds (phys_joint_prepare, prepare_group).
    for (uint32_t i = T.rank; i < W.nj + W.m; i += T.size) {
        if (i < W.nj) {
            joint_prepare_item(S, W, i, joints, bodies, fixed, K.h, A.err);
        } else {
            manifold_prepare_item(S, W, i - W.nj, contacts, bodies, fixed, A.err);
        }
    }
    T.sync();
    for (uint32_t sub = 0; sub < substeps; ++sub) {
        for (uint32_t i = T.rank; i < n; i += T.size) {
            integrate_velocity(B, i, K.h);
        }
        T.sync();
        world_pass<kWarm>(T, S, W, K);
        world_pass<kSolve>(T, S, W, K);
        for (uint32_t i = T.rank; i < n; i += T.size) {
            integrate_position(B, i, K.h);
        }
        T.sync();
        if (K.solver == NPH_GPU_SOLVER_SOFT_STEP) {
            world_pass<kRelax>(T, S, W, K);
        }
    }
    if (K.solver == NPH_GPU_SOLVER_TGS) {
        world_pass<kRelax>(T, S, W, K);
    }
    world_pass<kRestitution>(T, S, W, K);
    // store_group, the joints' impulses, finalize_body.
    for (uint32_t g = T.rank; g < W.m; g += T.size) {
        store_manifold_item(S, g, contacts);
    }
    for (uint32_t j = T.rank; j < W.nj; j += T.size) {
        store_joint_item(S, j, joints);
    }
    for (uint32_t i = T.rank; i < n; i += T.size) {
        finalize_item(B, i, bodies, K.dt);
    }
    T.sync();
    // post_finalize's driven joints (solver.c:851-857).
    if (W.driven > 0u) {
        for (uint32_t j = T.rank; j < W.nj; j += T.size) {
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
    T.sync();
}

template <int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_worlds(BatchArgs A, StepConsts K, uint32_t substeps)
{
    extern __shared__ float4 shared_vel[];
    __shared__ uint32_t taken[16];
    const uint32_t warps = kThreads / 32u;
    const uint32_t warp = threadIdx.x >> 5;
    // Size class by size class, largest teams first: a team takes worlds from its class's queue
    // until it is empty, then splits into the next class's teams. Barrier ids are unique over
    // every (class, team): class c's teams use ids warps / tw .. 2 warps / tw - 1.
    for (uint32_t c = 0; c < A.classes; ++c) {
        const uint32_t tw = warps >> c; // warps per team
        const uint32_t team = warp / tw;
        const Team T{threadIdx.x - team * tw * 32u, tw * 32u, tw == 1u ? 0u : warps / tw + team};
        const uint32_t slots = A.block_slots / (warps / tw);
        float4 *mine = shared_vel + (size_t)team * 2u * slots;
        for (;;) {
            uint32_t q = 0;
            if (T.rank == 0u) {
                q = atomicAdd(&A.heads[c], 1u);
            }
            if (tw == 1u) {
                q = __shfl_sync(0xFFFFFFFFu, q, 0);
            } else {
                if (T.rank == 0u) {
                    taken[T.barrier] = q;
                }
                T.sync();
                q = taken[T.barrier];
                T.sync();
            }
            if (q >= A.class_count[c]) {
                break;
            }
            world_step(T, A, A.worlds[A.order[A.class_first[c] + q]], K, substeps, mine, slots);
        }
    }
}

// ---- the merged packing: the batch as one world --------------------------------------

// A world-local body index in the merged world: its awake bodies after the worlds before it,
// its fixed bodies after every awake body and the fixed bodies of the worlds before it. An
// index outside the world maps outside every world, where prepare marks the record inert and
// reports it.
__device__ __forceinline__ uint32_t merged_body(uint32_t x, const WorldSlice &w, uint32_t n_total)
{
    if (x < w.n) {
        return w.body_first + x;
    }
    if (x - w.n < w.nf) {
        return n_total + w.fixed_first + (x - w.n);
    }
    return 0xFFFFFFF0u;
}

// The merged contact list: each world's colour lists in turn, each padded to whole groups of
// eight with an inert manifold (its two sides the pad body, which is not dynamic: one point,
// apart, nothing written), so the eight-lane group decisions are each world's own.
__global__ void __launch_bounds__(256) k_merge_contacts(const NphGpuContact *packed, const uint32_t *map,
                                                        const uint32_t *mworld, const WorldSlice *worlds,
                                                        uint32_t n_total, uint32_t pad_body, NphGpuContact *out,
                                                        uint32_t count)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) {
        return;
    }
    const uint32_t src = map[p];
    NphGpuContact c;
    if (src == NPH_GPU_NULL) {
        memset(&c, 0, sizeof c);
        c.body_a = pad_body;
        c.body_b = pad_body;
        c.point_count = 1u;
        c.normal[1] = 1.0f;
        c.points[0].separation = 1.0f;
    } else {
        c = packed[src];
        const WorldSlice &w = worlds[mworld[p]];
        c.body_a = merged_body(c.body_a, w, n_total);
        c.body_b = merged_body(c.body_b, w, n_total);
    }
    out[p] = c;
}

// Back into each world's slice: the results, with the world's own body indices.
__global__ void __launch_bounds__(256) k_unmerge_contacts(const NphGpuContact *merged, const uint32_t *map,
                                                          NphGpuContact *packed, uint32_t count)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count || map[p] == NPH_GPU_NULL) {
        return;
    }
    NphGpuContact c = merged[p];
    NphGpuContact &dst = packed[map[p]];
    c.body_a = dst.body_a;
    c.body_b = dst.body_b;
    dst = c;
}

__global__ void __launch_bounds__(256) k_merge_joints(const NphGpuJoint *packed, const uint32_t *map,
                                                      const uint32_t *mworld, const WorldSlice *worlds,
                                                      uint32_t n_total, NphGpuJoint *out, uint32_t count)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) {
        return;
    }
    NphGpuJoint j = packed[map[p]];
    const WorldSlice &w = worlds[mworld[p]];
    j.body_a = merged_body(j.body_a, w, n_total);
    j.body_b = merged_body(j.body_b, w, n_total);
    out[p] = j;
}

__global__ void __launch_bounds__(256) k_unmerge_joints(const NphGpuJoint *merged, const uint32_t *map,
                                                        NphGpuJoint *packed, uint32_t count)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) {
        return;
    }
    NphGpuJoint j = merged[p];
    NphGpuJoint &dst = packed[map[p]];
    j.body_a = dst.body_a;
    j.body_b = dst.body_b;
    dst = j;
}

struct BatchConfig {
    uint32_t threads, min_blocks;
};
// Up to 16 warps a block: a block's named barriers (ids 1-15) cover every team of every
// size class.
constexpr BatchConfig kBatchConfigs[] = {{128, 4}, {256, 2}, {256, 1}, {512, 1}, {256, 4}, {512, 2}};
constexpr uint32_t kBatchConfigCount = sizeof(kBatchConfigs) / sizeof(kBatchConfigs[0]);

} // namespace

StepConsts make_step_consts(const NphGpuWorldParams &p, float dt);

} // namespace nph

using namespace nph;

constexpr uint32_t kNoPassConfig = 0xFFFFFFFFu; // the merged solver's own pass configuration

struct NphGpuBatch {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool use_graph = true;
    uint32_t config = 1;
    uint32_t shared_mode = NPH_GPU_BATCH_SHARED_SMALL;
    uint32_t items_per_thread = 2; // a world's team: the smallest whose threads cover its
                                   // largest colour at this many items a thread (0: a block)
    uint32_t blocks_per_sm = 0; // resident blocks of the chosen kernel (0: not yet known)
    uint32_t class_first[kMaxClasses] = {}, class_count[kMaxClasses] = {};
    uint32_t classes = 1;
    // The merged packing: a single-world solver on the batch's stream, the merged lists'
    // sources (packed index, or NPH_GPU_NULL for a pad) and worlds, and whether the current
    // state lives in the solver (true after a merged step, until the next upload).
    uint32_t packing = NPH_GPU_BATCH_PERSISTENT;
    NphGpuSolver *merged = nullptr;
    uint32_t merged_pass[4] = {kNoPassConfig, kNoPassConfig, kNoPassConfig, kNoPassConfig}; // set ones
    uint32_t *d_cmap = nullptr, *d_cworld = nullptr, *d_jmap = nullptr, *d_jworld = nullptr;
    uint64_t cap_cmap = 0, cap_jmap = 0;
    bool maps_valid = false;
    bool live_in_merged = false;
    NphGpuWorldView merged_shape{};
    uint32_t merged_driven = 0, merged_row_joints = 0;
    int sms = 148;
    // Device arrays and their capacities (grown, never shrunk, by uploads).
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
    uint32_t *d_counters = nullptr; // [0..4] the size classes' queue heads, [6] error bits
    uint32_t *h_counters = nullptr;
    uint64_t cap_bodies = 0, cap_slots = 0, cap_fixed = 0, cap_contacts = 0, cap_joints = 0, cap_worlds = 0;
    // Sizes of the uploaded batch.
    uint32_t world_count = 0;
    uint64_t bodies = 0, slots = 0, fixed = 0, contacts = 0, joints = 0;
    uint64_t max_world_slots = 0;
    std::vector<WorldSlice> worlds;
    std::vector<uint32_t> order;
    // The step graph.
    cudaGraphExec_t graph = nullptr;
    bool graph_valid = false;
    StepConsts graph_consts{};
    uint32_t graph_substeps = 0;
    // The drop-in call's pipeline: the worlds split into consecutive parts, each a batch on
    // its own stream, their uploads one after another, so that one part's records come back
    // while the next parts' go up and step.
    uint32_t pipeline_parts = 1;
    std::vector<NphGpuBatch *> parts;
    std::vector<cudaEvent_t> part_uploaded;
    // Where the last results live: the parts (after a split call, part p's worlds starting at
    // part_first[p]) or the batch itself.
    bool results_in_parts = false;
    std::vector<uint32_t> part_first;
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
    bfree(b->d_cmap);
    bfree(b->d_cworld);
    bfree(b->d_jmap);
    bfree(b->d_jworld);
    b->cap_cmap = b->cap_jmap = 0;
    b->maps_valid = false;
    b->live_in_merged = false;
    b->cap_bodies = b->cap_slots = b->cap_fixed = b->cap_contacts = b->cap_joints = b->cap_worlds = 0;
    b->world_count = 0;
}

NphGpuResult cuda_result(cudaError_t e)
{
    if (e == cudaSuccess) {
        return NPH_GPU_OK;
    }
    return e == cudaErrorMemoryAllocation ? NPH_GPU_OUT_OF_MEMORY : NPH_GPU_DEVICE_LOST;
}

// Dynamic shared memory of a block: two velocity rows per slot, for the largest world, within
// the mode's limit.
size_t shared_bytes(const NphGpuBatch *b)
{
    if (b->shared_mode == NPH_GPU_BATCH_SHARED_NONE) {
        return 0;
    }
    const uint64_t limit = b->shared_mode == NPH_GPU_BATCH_SHARED_SMALL ? (32ull << 10) : (160ull << 10);
    const uint64_t want = 2ull * b->max_world_slots * sizeof(float4);
    return (size_t)std::min<uint64_t>(want, limit);
}

// The largest colour (constraints of one colour slot other than the overflow) of a world.
uint32_t largest_color(const WorldSlice &s)
{
    uint32_t m = 0;
    for (uint32_t c = 0; c < NPH_GPU_COLORS; ++c) {
        m = std::max(m, s.ccount[c] + s.jcount[c]);
    }
    return m;
}

// The size classes of the configuration's block: teams of B, B/2, ..., 1 warps.
uint32_t class_count_of(uint32_t threads)
{
    uint32_t warps = threads / 32u, classes = 1;
    while (warps > 1u) {
        warps >>= 1;
        ++classes;
    }
    return classes;
}

// The queue order for the configuration: each world's size class (the smallest team whose
// threads cover its largest colour at items_per_thread items a thread; a whole block when
// items_per_thread is 0), the classes in order, each largest first (a world's work grows with
// its manifolds, joints and bodies). A world without awake bodies (every island asleep) is left
// out: its step does nothing (solver.c:963-966), so it costs the launch nothing.
void build_order(NphGpuBatch *b)
{
    const std::vector<WorldSlice> &w = b->worlds;
    const uint32_t warps = kBatchConfigs[b->config].threads / 32u;
    b->classes = class_count_of(kBatchConfigs[b->config].threads);
    std::vector<uint32_t> cls(w.size(), 0u);
    if (b->items_per_thread > 0u) {
        for (size_t i = 0; i < w.size(); ++i) {
            const uint64_t need = (largest_color(w[i]) + (uint64_t)b->items_per_thread - 1u) / b->items_per_thread;
            uint32_t tw = 1u;
            while (tw < warps && 32ull * tw < need) {
                tw <<= 1;
            }
            uint32_t c = 0;
            while ((warps >> c) > tw) {
                ++c;
            }
            cls[i] = c;
        }
    }
    std::vector<uint32_t> order;
    order.reserve(w.size());
    for (uint32_t i = 0; i < (uint32_t)w.size(); ++i) {
        if (w[i].n > 0u) {
            order.push_back(i);
        }
    }
    auto work = [&](uint32_t x) { return 4ull * w[x].m + 3ull * w[x].nj + w[x].n; };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        if (cls[x] != cls[y]) {
            return cls[x] < cls[y];
        }
        return work(x) > work(y);
    });
    for (uint32_t c = 0; c < kMaxClasses; ++c) {
        b->class_first[c] = 0;
        b->class_count[c] = 0;
    }
    for (size_t i = 0; i < order.size(); ++i) {
        const uint32_t c = cls[order[i]];
        if (b->class_count[c] == 0u) {
            b->class_first[c] = (uint32_t)i;
        }
        b->class_count[c]++;
    }
    b->order = order;
}

BatchArgs batch_args(const NphGpuBatch *b)
{
    BatchArgs A;
    A.worlds = b->d_worlds;
    A.order = b->d_order;
    A.count = (uint32_t)b->order.size();
    for (uint32_t c = 0; c < kMaxClasses; ++c) {
        A.class_first[c] = b->class_first[c];
        A.class_count[c] = b->class_count[c];
    }
    A.classes = b->classes;
    A.heads = b->d_counters;
    A.err = b->d_counters + 6;
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
    A.mcap = (uint32_t)std::max<uint64_t>(b->cap_contacts, 1);
    A.jw = b->jw;
    A.jcap = (uint32_t)std::max<uint64_t>(b->cap_joints, 1);
    A.block_slots = (uint32_t)(shared_bytes(b) / (2 * sizeof(float4)));
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
    case 4: configure_kernel<256, 4>(smem); per_sm = resident<256, 4>(smem); break;
    default: configure_kernel<512, 2>(smem); per_sm = resident<512, 2>(smem); break;
    }
    b->blocks_per_sm = per_sm;
}

void enqueue_batch_step(NphGpuBatch *b, const StepConsts &K, uint32_t substeps)
{
    const BatchArgs A = batch_args(b);
    const size_t smem = shared_bytes(b);
    cudaMemsetAsync(b->d_counters, 0, kMaxClasses * sizeof(uint32_t), b->stream);
    const uint32_t grid = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(b->world_count, (uint64_t)b->blocks_per_sm * (uint64_t)b->sms));
    switch (b->config) {
    case 0: k_worlds<128, 4><<<grid, 128, smem, b->stream>>>(A, K, substeps); break;
    case 1: k_worlds<256, 2><<<grid, 256, smem, b->stream>>>(A, K, substeps); break;
    case 2: k_worlds<256, 1><<<grid, 256, smem, b->stream>>>(A, K, substeps); break;
    case 3: k_worlds<512, 1><<<grid, 512, smem, b->stream>>>(A, K, substeps); break;
    case 4: k_worlds<256, 4><<<grid, 256, smem, b->stream>>>(A, K, substeps); break;
    default: k_worlds<512, 2><<<grid, 512, smem, b->stream>>>(A, K, substeps); break;
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

// Uploads the queue order for the current configuration.
NphGpuResult apply_order(NphGpuBatch *b)
{
    drop_batch_graph(b);
    if (b->world_count == 0) {
        return NPH_GPU_OK;
    }
    build_order(b);
    if (!b->order.empty()) {
        cudaMemcpyAsync(b->d_order, b->order.data(), sizeof(uint32_t) * b->order.size(), cudaMemcpyHostToDevice,
                        b->stream);
    }
    return cuda_result(cudaStreamSynchronize(b->stream));
}

// The merged lists of the uploaded batch (built on the host, once per upload): colour by
// colour, each world's list in turn, contact lists padded to whole groups of eight.
NphGpuResult build_merge_maps(NphGpuBatch *b)
{
    if (b->maps_valid) {
        return NPH_GPU_OK;
    }
    std::vector<uint32_t> cmap, cworld, jmap, jworld;
    cmap.reserve(b->contacts + 8ull * b->world_count);
    cworld.reserve(b->contacts + 8ull * b->world_count);
    jmap.reserve(b->joints);
    jworld.reserve(b->joints);
    NphGpuWorldView &shape = b->merged_shape;
    std::memset(&shape, 0, sizeof shape);
    uint32_t driven = 0;
    for (uint32_t c = 0; c < NPH_GPU_COLOR_SLOTS; ++c) {
        for (uint32_t w = 0; w < b->world_count; ++w) {
            const WorldSlice &ws = b->worlds[w];
            for (uint32_t i = 0; i < ws.ccount[c]; ++i) {
                cmap.push_back(ws.contact_first + ws.cfirst[c] + i);
                cworld.push_back(w);
            }
            const uint32_t pad = c < NPH_GPU_COLORS ? (8u - ws.ccount[c] % 8u) % 8u : 0u;
            for (uint32_t i = 0; i < pad; ++i) {
                cmap.push_back(NPH_GPU_NULL);
                cworld.push_back(w);
            }
            shape.contact_color_counts[c] += ws.ccount[c] + pad;
            for (uint32_t i = 0; i < ws.jcount[c]; ++i) {
                jmap.push_back(ws.joint_first + ws.jfirst[c] + i);
                jworld.push_back(w);
            }
            shape.joint_color_counts[c] += ws.jcount[c];
        }
    }
    uint32_t row_joints = 0;
    for (uint32_t w = 0; w < b->world_count; ++w) {
        driven += b->worlds[w].driven;
        row_joints += b->worlds[w].row_joints;
    }
    if (cmap.size() >= 0xFFFFFFF0ull || b->bodies + b->fixed + 1u >= 0xFFFFFFF0ull) {
        return NPH_GPU_TOO_LARGE;
    }
    if (cmap.size() > b->cap_cmap || b->d_cmap == nullptr) {
        const uint64_t cap = std::max<uint64_t>(cmap.size(), 1);
        b->cap_cmap = 0;
        if (!balloc(b->d_cmap, cap) || !balloc(b->d_cworld, cap)) {
            return NPH_GPU_OUT_OF_MEMORY;
        }
        b->cap_cmap = cap;
    }
    if (jmap.size() > b->cap_jmap || b->d_jmap == nullptr) {
        const uint64_t cap = std::max<uint64_t>(jmap.size(), 1);
        b->cap_jmap = 0;
        if (!balloc(b->d_jmap, cap) || !balloc(b->d_jworld, cap)) {
            return NPH_GPU_OUT_OF_MEMORY;
        }
        b->cap_jmap = cap;
    }
    cudaMemcpyAsync(b->d_cmap, cmap.data(), cmap.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream);
    cudaMemcpyAsync(b->d_cworld, cworld.data(), cworld.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                    b->stream);
    if (!jmap.empty()) {
        cudaMemcpyAsync(b->d_jmap, jmap.data(), jmap.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream);
        cudaMemcpyAsync(b->d_jworld, jworld.data(), jworld.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                        b->stream);
    }
    shape.body_count = (uint32_t)b->bodies;
    shape.fixed_count = (uint32_t)b->fixed + 1u; // and the pad body
    shape.contact_count = (uint32_t)cmap.size();
    shape.joint_count = (uint32_t)jmap.size();
    b->merged_driven = driven;
    b->merged_row_joints = row_joints;
    const NphGpuResult r = cuda_result(cudaStreamSynchronize(b->stream));
    b->maps_valid = r == NPH_GPU_OK;
    return r;
}

// Packed -> the merged solver (the state then lives there). Without `sync` the copies are only
// enqueued on the batch's stream.
NphGpuResult merged_setup(NphGpuBatch *b, bool sync = true)
{
    if (b->live_in_merged) {
        return NPH_GPU_OK;
    }
    NphGpuResult r = build_merge_maps(b);
    if (r != NPH_GPU_OK) {
        return r;
    }
    if (b->merged == nullptr) {
        NphGpuSolverDesc d{};
        d.device = b->device;
        d.stream = b->stream;
        d.use_graph = b->use_graph ? 1u : 0u;
        r = nph_gpu_solver_create(&d, &b->merged);
        if (r != NPH_GPU_OK) {
            b->merged = nullptr;
            return r;
        }
        for (uint32_t p = 0; p < 4u && r == NPH_GPU_OK; ++p) {
            if (b->merged_pass[p] != kNoPassConfig) {
                r = nph_gpu_solver_set_pass_config(b->merged, p, b->merged_pass[p]);
            }
        }
        if (r != NPH_GPU_OK) {
            return r;
        }
    }
    NphSolverRecords R;
    r = nph_solver_bind_device(b->merged, &b->merged_shape, b->merged_driven, b->merged_row_joints, &R);
    if (r != NPH_GPU_OK) {
        return r;
    }
    const uint32_t n_total = (uint32_t)b->bodies;
    if (b->bodies > 0) {
        cudaMemcpyAsync(R.bodies, b->d_bodies, sizeof(NphGpuBody) * b->bodies, cudaMemcpyDeviceToDevice, b->stream);
    }
    if (b->fixed > 0) {
        cudaMemcpyAsync(R.fixed, b->d_fixed, sizeof(NphGpuBody) * b->fixed, cudaMemcpyDeviceToDevice, b->stream);
    }
    NphGpuBody pad;
    std::memset(&pad, 0, sizeof pad);
    pad.rotation[3] = 1.0f;
    pad.type = NPH_GPU_BODY_STATIC;
    cudaMemcpyAsync(R.fixed + b->fixed, &pad, sizeof pad, cudaMemcpyHostToDevice, b->stream);
    const uint32_t mc = b->merged_shape.contact_count, mj = b->merged_shape.joint_count;
    if (mc > 0) {
        k_merge_contacts<<<(mc + 255u) / 256u, 256, 0, b->stream>>>(b->d_contacts, b->d_cmap, b->d_cworld, b->d_worlds,
                                                                  n_total, n_total + (uint32_t)b->fixed, R.contacts, mc);
    }
    if (mj > 0) {
        k_merge_joints<<<(mj + 255u) / 256u, 256, 0, b->stream>>>(b->d_joints, b->d_jmap, b->d_jworld, b->d_worlds,
                                                                n_total, R.joints, mj);
    }
    r = cuda_result(sync ? cudaStreamSynchronize(b->stream) : cudaGetLastError());
    b->live_in_merged = r == NPH_GPU_OK;
    return r;
}

// The merged solver's state -> packed (both then hold it).
NphGpuResult merged_to_packed(NphGpuBatch *b, bool sync = true)
{
    if (!b->live_in_merged) {
        return NPH_GPU_OK;
    }
    NphSolverRecords R;
    NphGpuResult r = nph_solver_records(b->merged, &R);
    if (r != NPH_GPU_OK) {
        return r;
    }
    if (b->bodies > 0) {
        cudaMemcpyAsync(b->d_bodies, R.bodies, sizeof(NphGpuBody) * b->bodies, cudaMemcpyDeviceToDevice, b->stream);
    }
    const uint32_t mc = b->merged_shape.contact_count, mj = b->merged_shape.joint_count;
    if (mc > 0) {
        k_unmerge_contacts<<<(mc + 255u) / 256u, 256, 0, b->stream>>>(R.contacts, b->d_cmap, b->d_contacts, mc);
    }
    if (mj > 0) {
        k_unmerge_joints<<<(mj + 255u) / 256u, 256, 0, b->stream>>>(R.joints, b->d_jmap, b->d_joints, mj);
    }
    return cuda_result(sync ? cudaStreamSynchronize(b->stream) : cudaGetLastError());
}

// Makes the packed arrays the live state (for the persistent packing).
NphGpuResult leave_merged(NphGpuBatch *b)
{
    const NphGpuResult r = merged_to_packed(b);
    b->live_in_merged = false;
    return r;
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
        const int bad = nph_joint_check(&v.joints[j]);
        if (bad != NPH_GPU_OK) {
            return (NphGpuResult)bad;
        }
    }
    return NPH_GPU_OK;
}

// Host<->device copies of many worlds' records, merged while both sides stay contiguous.
class CopyRun {
  public:
    CopyRun(cudaStream_t st, cudaMemcpyKind kind) : st_(st), kind_(kind) {}
    ~CopyRun() { flush(); }
    void add(void *dst, const void *src, size_t bytes)
    {
        if (bytes == 0) {
            return;
        }
        if (bytes_ > 0 && (char *)dst == dst_ + bytes_ && (const char *)src == src_ + bytes_) {
            bytes_ += bytes;
            return;
        }
        flush();
        dst_ = (char *)dst;
        src_ = (const char *)src;
        bytes_ = bytes;
    }
    void flush()
    {
        if (bytes_ > 0) {
            cudaMemcpyAsync(dst_, src_, bytes_, kind_, st_);
            ++copies;
        }
        bytes_ = 0;
    }
    uint32_t copies = 0;

  private:
    cudaStream_t st_;
    cudaMemcpyKind kind_;
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t bytes_ = 0;
};

template <typename T> bool grow(T *&p, uint64_t &cap, uint64_t want)
{
    if (want <= cap && p != nullptr) {
        return true;
    }
    const uint64_t c = std::max<uint64_t>(want, 1);
    if (!balloc(p, c)) {
        cap = 0;
        return false;
    }
    cap = c;
    return true;
}

// The body rows (velocities, positions, parameters, integration state) per solver slot.
bool grow_slots(NphGpuBatch *b, uint64_t slots)
{
    if (slots <= b->cap_slots && b->vel != nullptr) {
        return true;
    }
    const uint64_t c = std::max<uint64_t>(slots, 1);
    b->cap_slots = 0;
    if (!balloc(b->vel, 2 * c) || !balloc(b->pos, 2 * c) || !balloc(b->prm, 3 * c) || !balloc(b->itg, 6 * c)) {
        return false;
    }
    b->cap_slots = c;
    return true;
}

// The manifold records and rows; the point rows are strided by the capacity.
bool grow_contacts(NphGpuBatch *b, uint64_t m)
{
    if (m <= b->cap_contacts && b->d_contacts != nullptr) {
        return true;
    }
    const uint64_t c = std::max<uint64_t>(m, 1);
    b->cap_contacts = 0;
    if (!balloc(b->d_contacts, c) || !balloc(b->hdr, c) || !balloc(b->nrm, c) || !balloc(b->rest, c) ||
        !balloc(b->pa, 4 * c) || !balloc(b->pb, 4 * c) || !balloc(b->pt, 4 * c) || !balloc(b->pi, 4 * c)) {
        return false;
    }
    b->cap_contacts = c;
    return true;
}

// The joint records and rows; the rows are strided by the capacity.
bool grow_joints(NphGpuBatch *b, uint64_t nj)
{
    if (nj <= b->cap_joints && b->d_joints != nullptr) {
        return true;
    }
    const uint64_t c = std::max<uint64_t>(nj, 1);
    b->cap_joints = 0;
    if (!balloc(b->d_joints, c) || !balloc(b->jw, (uint64_t)kJointRows * c)) {
        return false;
    }
    b->cap_joints = c;
    return true;
}

bool grow_worlds(NphGpuBatch *b, uint64_t count)
{
    if (count <= b->cap_worlds && b->d_worlds != nullptr) {
        return true;
    }
    const uint64_t c = std::max<uint64_t>(count, 1);
    b->cap_worlds = 0;
    if (!balloc(b->d_worlds, c) || !balloc(b->d_order, c)) {
        return false;
    }
    b->cap_worlds = c;
    return true;
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
    if (!balloc(b->d_counters, 8) ||
        cudaMallocHost((void **)&b->h_counters, 8 * sizeof(uint32_t)) != cudaSuccess) {
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
    for (NphGpuBatch *q : b->parts) {
        nph_gpu_batch_destroy(q);
    }
    for (cudaEvent_t e : b->part_uploaded) {
        cudaEventDestroy(e);
    }
    if (b->merged != nullptr) {
        nph_gpu_solver_destroy(b->merged);
        b->merged = nullptr;
    }
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

} // extern "C"

namespace {

// The upload of worlds that check_world accepted, enqueued on the batch's stream.
NphGpuResult upload_begin(NphGpuBatch *b, const NphGpuWorldView *worlds, uint32_t count)
{
    cudaSetDevice(b->device);
    // The slices, then the arrays grown to the batch.
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
        bodies += v.body_count;
        slots += v.body_count + 1u;
        fixed += v.fixed_count;
        contacts += v.contact_count;
        joints += v.joint_count;
        max_slots = std::max<uint64_t>(max_slots, v.body_count + 1u);
    }
    // Each world's driven and row-type joints: a read of every joint record, on host threads.
    {
        const uint32_t threads = std::max(1u, std::min({16u, std::thread::hardware_concurrency(), count / 64u}));
        auto scan = [&](uint32_t first, uint32_t end) {
            for (uint32_t w = first; w < end; ++w) {
                const NphGpuWorldView &v = worlds[w];
                uint32_t driven = 0, rows = 0;
                for (uint32_t j = 0; j < v.joint_count; ++j) {
                    const NphGpuJoint &jr = v.joints[j];
                    driven += nph_joint_is_driven(&jr) ? 1u : 0u;
                    rows += (nph_joint_has_axes(jr.type) || jr.type == NPH_GPU_JOINT_DISTANCE) ? 1u : 0u;
                }
                slices[w].driven = driven;
                slices[w].row_joints = rows;
            }
        };
        std::vector<std::thread> pool;
        for (uint32_t t = 1; t < threads; ++t) {
            const uint32_t first = (uint32_t)((uint64_t)count * t / threads);
            const uint32_t end = (uint32_t)((uint64_t)count * (t + 1) / threads);
            try {
                pool.emplace_back(scan, first, end);
            } catch (...) { // no thread to be had: this one scans the run
                scan(first, end);
            }
        }
        scan(0u, (uint32_t)((uint64_t)count / threads));
        for (std::thread &th : pool) {
            th.join();
        }
    }
    if (slots >= 0xFFFFFFF0ull || contacts >= 0xFFFFFFF0ull || joints >= 0xFFFFFFF0ull ||
        4ull * contacts >= 0xFFFFFFF0ull || (uint64_t)kJointRows * joints >= 0xFFFFFFF0ull) {
        return NPH_GPU_TOO_LARGE;
    }
    // The same worlds' shapes as the last upload (every count and offset): the arrays keep
    // their size, so the captured step and the merged lists stay valid; only records move.
    const bool same_batch = count == b->world_count && b->worlds.size() == count &&
                            (count == 0 ||
                             std::memcmp(b->worlds.data(), slices.data(), sizeof(WorldSlice) * count) == 0);
    if (!same_batch) {
        drop_batch_graph(b);
    }
    // The point and joint rows are strided by their capacity: a capacity change reallocates
    // them with the new stride.
    const bool ok = grow(b->d_bodies, b->cap_bodies, bodies) && grow(b->d_fixed, b->cap_fixed, fixed) &&
                    grow_slots(b, slots) && grow_contacts(b, contacts) && grow_joints(b, joints) &&
                    grow_worlds(b, count);
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
    b->maps_valid = b->maps_valid && same_batch;
    b->live_in_merged = false;
    build_order(b);
    cudaMemcpyAsync(b->d_worlds, slices.data(), sizeof(WorldSlice) * count, cudaMemcpyHostToDevice, b->stream);
    if (!b->order.empty()) {
        cudaMemcpyAsync(b->d_order, b->order.data(), sizeof(uint32_t) * b->order.size(), cudaMemcpyHostToDevice,
                        b->stream);
    }
    {
        CopyRun cb(b->stream, cudaMemcpyHostToDevice), cf(b->stream, cudaMemcpyHostToDevice),
            cc(b->stream, cudaMemcpyHostToDevice), cj(b->stream, cudaMemcpyHostToDevice);
        for (uint32_t w = 0; w < count; ++w) {
            const NphGpuWorldView &v = worlds[w];
            const WorldSlice &s = slices[w];
            cb.add(b->d_bodies + s.body_first, v.bodies, sizeof(NphGpuBody) * v.body_count);
            cf.add(b->d_fixed + s.fixed_first, v.fixed_bodies, sizeof(NphGpuBody) * v.fixed_count);
            cc.add(b->d_contacts + s.contact_first, v.contacts, sizeof(NphGpuContact) * v.contact_count);
            cj.add(b->d_joints + s.joint_first, v.joints, sizeof(NphGpuJoint) * v.joint_count);
        }
    }
    cudaMemsetAsync(b->d_counters, 0, 8 * sizeof(uint32_t), b->stream);
    return cuda_result(cudaGetLastError());
}

NphGpuResult step_begin(NphGpuBatch *b, const NphGpuWorldParams *params, float dt, uint32_t steps,
                        bool sync_setup)
{
    if (b->world_count == 0) {
        return NPH_GPU_OK;
    }
    cudaSetDevice(b->device);
    if (b->packing == NPH_GPU_BATCH_MERGED) {
        const NphGpuResult r = merged_setup(b, sync_setup);
        return r != NPH_GPU_OK ? r : nph_gpu_world_step_async(b->merged, params, dt, steps);
    }
    NphGpuResult r = leave_merged(b);
    const StepConsts K = make_step_consts(*params, dt);
    for (uint32_t i = 0; i < steps && r == NPH_GPU_OK; ++i) {
        r = launch_batch_step(b, K, params->substeps);
    }
    return r;
}

// The packed results' copies into the worlds' records, enqueued on the batch's stream.
NphGpuResult enqueue_downloads(NphGpuBatch *b, NphGpuWorldView *worlds, uint32_t count)
{
    for (uint32_t w = 0; w < count; ++w) {
        const NphGpuWorldView &v = worlds[w];
        const WorldSlice &s = b->worlds[w];
        if (v.body_count != s.n || v.contact_count != s.m || v.joint_count != s.nj ||
            (s.n > 0 && v.bodies == nullptr) || (s.m > 0 && v.contacts == nullptr) ||
            (s.nj > 0 && v.joints == nullptr)) {
            return NPH_GPU_INVALID_STATE;
        }
    }
    CopyRun cb(b->stream, cudaMemcpyDeviceToHost), cc(b->stream, cudaMemcpyDeviceToHost),
        cj(b->stream, cudaMemcpyDeviceToHost);
    for (uint32_t w = 0; w < count; ++w) {
        NphGpuWorldView &v = worlds[w];
        const WorldSlice &s = b->worlds[w];
        cb.add(v.bodies, b->d_bodies + s.body_first, sizeof(NphGpuBody) * s.n);
        cc.add(v.contacts, b->d_contacts + s.contact_first, sizeof(NphGpuContact) * s.m);
        cj.add(v.joints, b->d_joints + s.joint_first, sizeof(NphGpuJoint) * s.nj);
    }
    cb.flush();
    cc.flush();
    cj.flush();
    return cuda_result(cudaGetLastError());
}

// Waits for the batch's stream and reports a record the device refused.
NphGpuResult batch_finish(NphGpuBatch *b)
{
    cudaSetDevice(b->device);
    NphGpuResult r = NPH_GPU_OK;
    if (b->live_in_merged) {
        r = nph_solver_check(b->merged);
    }
    cudaMemcpyAsync(b->h_counters, b->d_counters, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream);
    const NphGpuResult e = cuda_result(cudaStreamSynchronize(b->stream));
    if (r == NPH_GPU_OK) {
        r = e;
    }
    if (r == NPH_GPU_OK && b->h_counters[6] != 0u) {
        r = NPH_GPU_INVALID_ARGUMENT;
    }
    return r;
}

// Every record the device would refuse (check_world's and prepare's checks: a joint's or a
// manifold's body outside its world, a manifold without points or with more than four), on
// the host, so that a pipelined call refuses a batch before any of it is written back.
// check_world over every world, on up to 16 host threads; the result of the first world (in
// order) that fails, as a loop over the worlds would return it.
NphGpuResult check_worlds(const NphGpuWorldView *worlds, uint32_t count)
{
    const uint32_t threads = std::max(1u, std::min({16u, std::thread::hardware_concurrency(), count / 64u}));
    std::vector<uint32_t> first_bad(threads, count);
    std::vector<NphGpuResult> code(threads, NPH_GPU_OK);
    auto scan = [&](uint32_t t, uint32_t first, uint32_t end) {
        for (uint32_t w = first; w < end; ++w) {
            const NphGpuResult r = check_world(worlds[w]);
            if (r != NPH_GPU_OK) {
                first_bad[t] = w;
                code[t] = r;
                return;
            }
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) {
        const uint32_t first = (uint32_t)((uint64_t)count * t / threads);
        const uint32_t end = (uint32_t)((uint64_t)count * (t + 1) / threads);
        try {
            pool.emplace_back(scan, t, first, end);
        } catch (...) { // no thread to be had: this one scans the run
            scan(t, first, end);
        }
    }
    scan(0u, 0u, (uint32_t)((uint64_t)count / threads));
    for (std::thread &th : pool) {
        th.join();
    }
    for (uint32_t t = 0; t < threads; ++t) { // the runs are in world order
        if (first_bad[t] < count) {
            return code[t];
        }
    }
    return NPH_GPU_OK;
}

NphGpuResult check_records(const NphGpuWorldView *worlds, uint32_t count)
{
    std::atomic<uint32_t> bad{0};
    auto scan = [&](uint32_t first, uint32_t end) {
        for (uint32_t w = first; w < end && bad.load(std::memory_order_relaxed) == 0u; ++w) {
            const NphGpuWorldView &v = worlds[w];
            const uint64_t total = (uint64_t)v.body_count + v.fixed_count;
            uint32_t worst = 0u;
            for (uint32_t i = 0; i < v.contact_count; ++i) {
                const NphGpuContact &c = v.contacts[i];
                worst |= (c.body_a >= total) | (c.body_b >= total) | (c.point_count < 1u) |
                         (c.point_count > NPH_GPU_MAX_POINTS);
            }
            for (uint32_t j = 0; j < v.joint_count; ++j) {
                worst |= (v.joints[j].body_a >= total) | (v.joints[j].body_b >= total);
            }
            if (worst != 0u) {
                bad.store(1u, std::memory_order_relaxed);
            }
        }
    };
    const uint32_t threads = std::max(1u, std::min({16u, std::thread::hardware_concurrency(), count / 64u}));
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) {
        const uint32_t first = (uint32_t)((uint64_t)count * t / threads);
        const uint32_t end = (uint32_t)((uint64_t)count * (t + 1) / threads);
        try {
            pool.emplace_back(scan, first, end);
        } catch (...) { // no thread to be had: this one scans the run
            scan(first, end);
        }
    }
    scan(0u, (uint32_t)((uint64_t)count / threads));
    for (std::thread &t : pool) {
        t.join();
    }
    return bad.load() != 0u ? NPH_GPU_INVALID_ARGUMENT : NPH_GPU_OK;
}

// The parts' batches and their events, created or released to match the requested count, each
// part on the parent's launch configuration.
NphGpuResult ensure_parts(NphGpuBatch *b, uint32_t parts)
{
    while (b->parts.size() > parts) {
        nph_gpu_batch_destroy(b->parts.back());
        b->parts.pop_back();
        cudaEventDestroy(b->part_uploaded.back());
        b->part_uploaded.pop_back();
    }
    while (b->parts.size() < parts) {
        NphGpuSolverDesc d{};
        d.device = b->device;
        d.use_graph = b->use_graph ? 1u : 0u;
        NphGpuBatch *q = nullptr;
        NphGpuResult r = nph_gpu_batch_create(&d, &q);
        if (r != NPH_GPU_OK) {
            return r;
        }
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            nph_gpu_batch_destroy(q);
            return cuda_result(cudaGetLastError());
        }
        b->parts.push_back(q);
        b->part_uploaded.push_back(e);
    }
    for (NphGpuBatch *q : b->parts) {
        if (q->packing != b->packing || q->config != b->config || q->shared_mode != b->shared_mode ||
            q->items_per_thread != b->items_per_thread) {
            NphGpuBatchTuning t{};
            t.config = b->config;
            t.shared_velocities = b->shared_mode;
            t.items_per_thread = b->items_per_thread;
            t.packing = b->packing;
            const NphGpuResult r = nph_gpu_batch_set_config(q, &t);
            if (r != NPH_GPU_OK) {
                return r;
            }
        }
    }
    return NPH_GPU_OK;
}

uint64_t record_bytes(const NphGpuWorldView &v)
{
    return sizeof(NphGpuBody) * ((uint64_t)v.body_count + v.fixed_count) + sizeof(NphGpuContact) * (uint64_t)v.contact_count +
           sizeof(NphGpuJoint) * (uint64_t)v.joint_count;
}

// nph_gpu_phys_solve_worlds in parts: consecutive runs of worlds of about equal record bytes,
// after the host has checked every record (a refused batch has nothing written back). Each
// part's stream holds its upload, step and download in turn, and its upload waits for the
// previous part's, so a part's results come back while the later parts still go up.
NphGpuResult solve_in_parts(NphGpuBatch *b, const NphGpuWorldParams *params, float dt, NphGpuWorldView *worlds,
                            uint32_t count)
{
    NphGpuResult r = check_records(worlds, count);
    if (r != NPH_GPU_OK) {
        return r;
    }
    const uint32_t parts = std::min(b->pipeline_parts, count);
    r = ensure_parts(b, parts);
    if (r != NPH_GPU_OK) {
        return r;
    }
    std::vector<uint32_t> first(parts + 1u, count);
    {
        uint64_t total = 0;
        for (uint32_t w = 0; w < count; ++w) {
            total += record_bytes(worlds[w]);
        }
        uint64_t sum = 0;
        uint32_t p = 1;
        first[0] = 0;
        for (uint32_t w = 0; w < count && p < parts; ++w) {
            sum += record_bytes(worlds[w]);
            while (p < parts && sum * parts >= total * p) {
                first[p++] = w + 1u;
            }
        }
    }
    uint32_t started = 0;
    for (uint32_t p = 0; p < parts && r == NPH_GPU_OK; ++p) {
        NphGpuBatch *q = b->parts[p];
        const uint32_t n = first[p + 1u] - first[p];
        cudaSetDevice(q->device);
        if (p > 0) {
            cudaStreamWaitEvent(q->stream, b->part_uploaded[p - 1u], 0);
        }
        started = p + 1u;
        r = upload_begin(q, worlds + first[p], n);
        cudaEventRecord(b->part_uploaded[p], q->stream);
        if (r == NPH_GPU_OK) {
            r = step_begin(q, params, dt, 1u, false);
        }
        if (r == NPH_GPU_OK) {
            r = merged_to_packed(q, false);
        }
        if (r == NPH_GPU_OK) {
            r = enqueue_downloads(q, worlds + first[p], n);
        }
    }
    for (uint32_t p = 0; p < started; ++p) {
        const NphGpuResult e = batch_finish(b->parts[p]);
        if (r == NPH_GPU_OK) {
            r = e;
        }
    }
    b->results_in_parts = r == NPH_GPU_OK;
    b->part_first.assign(first.begin(), first.begin() + parts);
    return r;
}

} // namespace

extern "C" {

NPH_GPU_API NphGpuResult nph_gpu_batch_upload(NphGpuBatch *b, const NphGpuWorldView *worlds,
                                              uint32_t count)
{
    if (b == nullptr || (count > 0 && worlds == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    {
        const NphGpuResult r = check_worlds(worlds, count);
        if (r != NPH_GPU_OK) {
            return r;
        }
    }
    b->results_in_parts = false;
    const NphGpuResult r = upload_begin(b, worlds, count);
    return r != NPH_GPU_OK ? r : cuda_result(cudaStreamSynchronize(b->stream));
}

NPH_GPU_API NphGpuResult nph_gpu_batch_step_async(NphGpuBatch *b, const NphGpuWorldParams *params,
                                                  float dt, uint32_t steps)
{
    if (b == nullptr || params == nullptr || !(dt > 0.0f) || params->substeps == 0u ||
        params->substeps > 64u) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if ((params->solver != NPH_GPU_SOLVER_SOFT_STEP && params->solver != NPH_GPU_SOLVER_TGS) ||
        params->enable_continuous != 0u) {
        return NPH_GPU_UNSUPPORTED;
    }
    return step_begin(b, params, dt, steps, true);
}

NPH_GPU_API NphGpuResult nph_gpu_batch_download(NphGpuBatch *b, NphGpuWorldView *worlds, uint32_t count)
{
    if (b == nullptr || count != b->world_count || (count > 0 && worlds == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(b->device);
    NphGpuResult r = NPH_GPU_OK;
    if (b->live_in_merged) {
        r = nph_solver_check(b->merged);
        if (r == NPH_GPU_OK) {
            r = merged_to_packed(b);
        }
        if (r != NPH_GPU_OK) {
            return r;
        }
    }
    cudaMemcpyAsync(b->h_counters, b->d_counters, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream);
    r = cuda_result(cudaStreamSynchronize(b->stream));
    if (r != NPH_GPU_OK) {
        return r;
    }
    if (b->h_counters[6] != 0u) {
        return NPH_GPU_INVALID_ARGUMENT; // a malformed record: nothing written back
    }
    r = enqueue_downloads(b, worlds, count);
    return r != NPH_GPU_OK ? r : cuda_result(cudaStreamSynchronize(b->stream));
}

NPH_GPU_API NphGpuResult nph_gpu_phys_solve_worlds(NphGpuBatch *b, const NphGpuWorldParams *params,
                                                   float dt, NphGpuWorldView *worlds, uint32_t count)
{
    if (b != nullptr && b->pipeline_parts > 1u && count > 1u) {
        if (worlds == nullptr || params == nullptr || !(dt > 0.0f) || params->substeps == 0u ||
            params->substeps > 64u) {
            return NPH_GPU_INVALID_ARGUMENT;
        }
        if ((params->solver != NPH_GPU_SOLVER_SOFT_STEP && params->solver != NPH_GPU_SOLVER_TGS) ||
            params->enable_continuous != 0u) {
            return NPH_GPU_UNSUPPORTED;
        }
        const NphGpuResult r = check_worlds(worlds, count);
        if (r != NPH_GPU_OK) {
            return r;
        }
        return solve_in_parts(b, params, dt, worlds, count);
    }
    NphGpuResult r = nph_gpu_batch_upload(b, worlds, count);
    if (r == NPH_GPU_OK) {
        r = nph_gpu_batch_step_async(b, params, dt, 1);
    }
    if (r == NPH_GPU_OK) {
        r = nph_gpu_batch_download(b, worlds, count);
    }
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_batch_set_config(NphGpuBatch *b, const NphGpuBatchTuning *t)
{
    if (b == nullptr || t == nullptr || t->config >= kBatchConfigCount ||
        t->shared_velocities > NPH_GPU_BATCH_SHARED_LARGE || t->packing > NPH_GPU_BATCH_MERGED) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    cudaSetDevice(b->device);
    if (t->packing != b->packing) {
        const NphGpuResult r = leave_merged(b);
        if (r != NPH_GPU_OK) {
            return r;
        }
    }
    b->packing = t->packing;
    b->config = t->config;
    b->shared_mode = t->shared_velocities;
    b->items_per_thread = t->items_per_thread;
    return apply_order(b);
}

NPH_GPU_API NphGpuResult nph_gpu_batch_hit_events(NphGpuBatch *b, float threshold, NphGpuHitEvent *events,
                                                 uint32_t capacity, uint32_t *count)
{
    if (b == nullptr || count == nullptr || (capacity > 0u && events == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    *count = 0u;
    std::vector<std::pair<NphGpuBatch *, uint32_t>> sources; // a batch, its first world
    if (b->results_in_parts) {
        for (size_t p = 0; p < b->part_first.size() && p < b->parts.size(); ++p) {
            sources.emplace_back(b->parts[p], b->part_first[p]);
        }
    } else {
        sources.emplace_back(b, 0u);
    }
    uint32_t total = 0u;
    for (const auto &src : sources) {
        NphGpuBatch *q = src.first;
        if (q->world_count == 0u) {
            continue;
        }
        cudaSetDevice(q->device);
        NphGpuResult r = merged_to_packed(q);
        if (r != NPH_GPU_OK) {
            return r;
        }
        const uint32_t room = total < capacity ? capacity - total : 0u;
        uint32_t n = 0u;
        r = nph_hits_scan(q->d_contacts, (uint32_t)q->contacts, threshold, q->stream,
                          room > 0u ? events + total : nullptr, room, &n);
        if (r != NPH_GPU_OK) {
            return r;
        }
        // A packed index into its world: the last world starting at or before it.
        for (uint32_t i = 0; i < std::min(n, room); ++i) {
            NphGpuHitEvent &e = events[total + i];
            const auto it = std::upper_bound(q->worlds.begin(), q->worlds.end(), e.contact,
                                             [](uint32_t x, const WorldSlice &w) { return x < w.contact_first; });
            const uint32_t w = (uint32_t)(it - q->worlds.begin()) - 1u;
            e.contact -= q->worlds[w].contact_first;
            e.world = src.second + w;
        }
        total += n;
    }
    *count = total;
    return NPH_GPU_OK;
}

NPH_GPU_API NphGpuResult nph_gpu_batch_set_pipeline(NphGpuBatch *b, uint32_t parts)
{
    if (b == nullptr || parts < 1u || parts > NPH_GPU_BATCH_MAX_PARTS) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    b->pipeline_parts = parts;
    if (parts == 1u) {
        return ensure_parts(b, 0u); // the parts' arrays released
    }
    return NPH_GPU_OK;
}

NPH_GPU_API NphGpuResult nph_gpu_batch_set_pass_config(NphGpuBatch *b, uint32_t pass, uint32_t config)
{
    if (b == nullptr || pass >= 4u || config >= nph_gpu_pass_config_count()) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    b->merged_pass[pass] = config;
    if (b->merged != nullptr) {
        return nph_gpu_solver_set_pass_config(b->merged, pass, config);
    }
    return NPH_GPU_OK;
}

NPH_GPU_API uint32_t nph_gpu_batch_config_count(void) { return kBatchConfigCount; }

NPH_GPU_API NphGpuResult nph_gpu_batch_autotune(NphGpuBatch *b, const NphGpuWorldParams *params,
                                                float dt, uint32_t rounds, NphGpuBatchTuning *out)
{
    if (b == nullptr || params == nullptr || !(dt > 0.0f) || params->substeps == 0u || params->substeps > 64u) {
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
    static const uint32_t kSplits[] = {0u, 1u, 2u, 4u, 8u};
    float best = 1e30f;
    NphGpuBatchTuning chosen{b->config, kBatchConfigs[b->config].threads, b->shared_mode, b->items_per_thread,
                             b->packing, 0.0f, 0.0f, 0.0f};
    float best_persistent = 0.0f, merged_ms = 0.0f;
    rounds = rounds == 0u ? 1u : rounds;
    auto timed = [&](auto &&step) -> float {
        cudaEventRecord(e0, b->stream);
        NphGpuResult q = NPH_GPU_OK;
        for (uint32_t i = 0; i < rounds && q == NPH_GPU_OK; ++i) {
            q = step();
        }
        cudaEventRecord(e1, b->stream);
        if (q == NPH_GPU_OK) {
            q = cuda_result(cudaEventSynchronize(e1));
        }
        float ms = 1e30f;
        if (q == NPH_GPU_OK) {
            cudaEventElapsedTime(&ms, e0, e1);
        }
        return ms;
    };
    // The persistent packing: every launch shape, shared-memory mode and team sizing.
    NphGpuResult r = leave_merged(b);
    for (uint32_t shared = 0; shared <= NPH_GPU_BATCH_SHARED_LARGE && r == NPH_GPU_OK; ++shared) {
        for (uint32_t c = 0; c < kBatchConfigCount && r == NPH_GPU_OK; ++c) {
            for (uint32_t split : kSplits) {
                if (r != NPH_GPU_OK) {
                    break;
                }
                b->packing = NPH_GPU_BATCH_PERSISTENT;
                b->config = c;
                b->shared_mode = shared;
                b->items_per_thread = split;
                r = apply_order(b);
                if (r == NPH_GPU_OK) {
                    r = launch_batch_step(b, K, params->substeps); // builds the graph, warms up
                }
                if (r != NPH_GPU_OK) {
                    break;
                }
                const float ms = timed([&] { return launch_batch_step(b, K, params->substeps); });
                if (ms < best) {
                    best = ms;
                    best_persistent = ms / (float)rounds;
                    chosen = NphGpuBatchTuning{c, kBatchConfigs[c].threads, shared, split, NPH_GPU_BATCH_PERSISTENT,
                                               ms / (float)rounds, 0.0f, 0.0f};
                }
            }
        }
    }
    // The merged packing, its passes tuned by the single-world autotuner.
    if (r == NPH_GPU_OK) {
        b->packing = NPH_GPU_BATCH_MERGED;
        r = merged_setup(b);
        uint32_t pass[4];
        if (r == NPH_GPU_OK) {
            r = nph_gpu_solver_autotune(b->merged, params, dt, rounds, pass);
        }
        if (r == NPH_GPU_OK) {
            r = nph_gpu_world_step_async(b->merged, params, dt, 1); // builds the graph, warms up
        }
        if (r == NPH_GPU_OK) {
            const float ms = timed([&] { return nph_gpu_world_step_async(b->merged, params, dt, 1); });
            merged_ms = ms / (float)rounds;
            if (ms < best) {
                best = ms;
                chosen = NphGpuBatchTuning{b->config, kBatchConfigs[b->config].threads, b->shared_mode,
                                           b->items_per_thread, NPH_GPU_BATCH_MERGED, ms / (float)rounds, 0.0f,
                                           0.0f};
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    NphGpuResult ro = NPH_GPU_OK;
    if (chosen.packing == NPH_GPU_BATCH_PERSISTENT) {
        ro = leave_merged(b);
    }
    b->packing = chosen.packing;
    b->config = chosen.config;
    b->shared_mode = chosen.shared_velocities;
    b->items_per_thread = chosen.items_per_thread;
    if (ro == NPH_GPU_OK) {
        ro = apply_order(b);
    }
    chosen.persistent_ms_per_step = best_persistent;
    chosen.merged_ms_per_step = merged_ms;
    if (out != nullptr) {
        *out = chosen;
    }
    return r != NPH_GPU_OK ? r : ro;
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
    out->shared_velocities = b->shared_mode;
    out->blocks_per_sm = b->blocks_per_sm;
    out->items_per_thread = b->items_per_thread;
    out->packing = b->packing;
    out->launches_per_step = 1u;
    if (b->packing == NPH_GPU_BATCH_MERGED && b->merged != nullptr) {
        NphGpuStepStats st;
        if (nph_gpu_solver_stats(b->merged, &st) == NPH_GPU_OK) {
            out->launches_per_step = st.launches;
        }
    }
    out->warp_worlds = b->class_count[b->classes - 1u];
    out->block_worlds = b->class_count[0];
    return NPH_GPU_OK;
}

} // extern "C"

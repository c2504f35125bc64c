// SPDX-License-Identifier: Apache-2.0
//
// The narrow phase's closed-form pairs (collide.cuh), one thread per pair.

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <new>
#include <vector>

#include "nepheline_b200.h"

#include "collide.cuh"

namespace {

// One pair's manifold into out[i]: the cleared manifold and a count in `bad` for an unknown type.
__device__ __forceinline__ void collide_pair(const NphGpuShape *a, const NphGpuPose *pa, const NphGpuShape *b,
                                             const NphGpuPose *pb, const float *spec, uint32_t i,
                                             NphGpuManifold *out, uint32_t *bad)
{
    NphGpuManifold m;
    for (uint32_t k = 0; k < NPH_GPU_MAX_POINTS; ++k) {
        m.points[k] = NphGpuManifoldPoint{{0.0f, 0.0f, 0.0f}, 0.0f, 0u};
    }
    if (a[i].type > NPH_GPU_SHAPE_BOX || b[i].type > NPH_GPU_SHAPE_BOX) {
        m.normal[0] = 0.0f;
        m.normal[1] = 1.0f;
        m.normal[2] = 0.0f;
        m.point_count = 0u;
        if (bad != nullptr) {
            atomicAdd(bad, 1u);
        }
    } else {
        nph_nc::collide(a[i], pa[i], b[i], pb[i], spec[i], m);
    }
    out[i] = m;
}

__global__ void __launch_bounds__(256) k_collide(const NphGpuShape *a, const NphGpuPose *pa, const NphGpuShape *b,
                                                 const NphGpuPose *pb, const float *spec, uint32_t count,
                                                 NphGpuManifold *out, uint32_t *bad)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        collide_pair(a, pa, b, pb, spec, i, out, bad);
    }
}

// The pair kinds, (type a, type b) in 0..15 (unknown types share kind 15), counted and each pair
// given its place among its kind's: the warps of the sorted launch then run one kind's code.
constexpr uint32_t kKinds = 16u;

__device__ __forceinline__ uint32_t pair_kind(const NphGpuShape &a, const NphGpuShape &b)
{
    return a.type <= NPH_GPU_SHAPE_BOX && b.type <= NPH_GPU_SHAPE_BOX ? a.type * 3u + b.type : kKinds - 1u;
}

// Box pairs apart along a face axis by more than the slop take the GJK path (or none), the rest
// the face clip: an estimate from the six face axes gives the apart ones a kind of their own
// (kind 9), so that a warp runs one of the two paths. Only the order of the pairs depends on it.
constexpr uint32_t kKindBoxesApart = 9u;

__device__ __forceinline__ bool boxes_apart(const NphGpuShape &a, const NphGpuPose &pa, const NphGpuShape &b,
                                            const NphGpuPose &pb)
{
    using namespace nph_nc;
    const Q qa{pa.rotation[0], pa.rotation[1], pa.rotation[2], pa.rotation[3]};
    const Q qb{pb.rotation[0], pb.rotation[1], pb.rotation[2], pb.rotation[3]};
    const V t = rotate_inverse(qa, V{pb.position[0] - pa.position[0], pb.position[1] - pa.position[1],
                                     pb.position[2] - pa.position[2]});
    const Q rq = q_mul(Q{-qa.x, -qa.y, -qa.z, qa.w}, qb);
    const V c[3] = {axis_x(rq), axis_y(rq), axis_z(rq)}; // B's axes in A's frame
    float worst = -3.4e38f;
#pragma unroll
    for (uint32_t i = 0; i < 3u; ++i) {
        const float ra = a.dims[i];
        const float rb = b.dims[0] * fabsf(at(c[0], i)) + b.dims[1] * fabsf(at(c[1], i)) + b.dims[2] * fabsf(at(c[2], i));
        worst = fmaxf(worst, fabsf(at(t, i)) - (ra + rb));
    }
#pragma unroll
    for (uint32_t j = 0; j < 3u; ++j) {
        const float ra = a.dims[0] * fabsf(c[j].x) + a.dims[1] * fabsf(c[j].y) + a.dims[2] * fabsf(c[j].z);
        worst = fmaxf(worst, fabsf(dot(t, c[j])) - (ra + b.dims[j]));
    }
    return worst > 0.005f;
}

__global__ void __launch_bounds__(256) k_classify(const NphGpuShape *a, const NphGpuPose *pa, const NphGpuShape *b,
                                                  const NphGpuPose *pb, uint32_t count, uint32_t *counts,
                                                  uint32_t *place)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        // One atomic per kind and warp: the lanes of a kind take consecutive places.
        uint32_t k = pair_kind(a[i], b[i]);
        if (k == NPH_GPU_SHAPE_BOX * 4u && boxes_apart(a[i], pa[i], b[i], pb[i])) {
            k = kKindBoxesApart;
        }
        const uint32_t lane = threadIdx.x & 31u;
        const uint32_t group = __match_any_sync(__activemask(), k);
        const uint32_t leader = __ffs(group) - 1u;
        uint32_t base = 0u;
        if (lane == leader) {
            base = atomicAdd(&counts[k], (uint32_t)__popc(group));
        }
        base = __shfl_sync(group, base, leader);
        place[i] = (k << 28u) | (base + (uint32_t)__popc(group & ((1u << lane) - 1u)));
    }
}

__global__ void k_kind_offsets(uint32_t *counts)
{
    if (threadIdx.x == 0u) {
        uint32_t sum = 0u;
        for (uint32_t k = 0; k < kKinds; ++k) {
            const uint32_t c = counts[k];
            counts[kKinds + k] = sum;
            sum += c;
        }
    }
}

__global__ void __launch_bounds__(256) k_scatter(const uint32_t *counts, const uint32_t *place, uint32_t count,
                                                 uint32_t *order)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        const uint32_t p = place[i];
        order[counts[kKinds + (p >> 28u)] + (p & 0x0FFFFFFFu)] = i;
    }
}

// Three blocks an SM (80 registers): on the 4,194,304 mixed pairs 3.72 ms against 3.70 for four
// (64 registers) and 3.91 for two (109); DRAM bytes a launch 24 % fewer than with four, 39 %
// more than with two: each thread's clip polygons, candidates and corners live in local
// memory, and fewer resident threads keep more of those lines in L2.
#ifndef NPH_COLLIDE_BLOCKS_PER_SM
#define NPH_COLLIDE_BLOCKS_PER_SM 3
#endif
__global__ void __launch_bounds__(256, NPH_COLLIDE_BLOCKS_PER_SM) k_collide_sorted(const NphGpuShape *a, const NphGpuPose *pa,
                                                        const NphGpuShape *b, const NphGpuPose *pb,
                                                        const float *spec, uint32_t count, const uint32_t *order,
                                                        NphGpuManifold *out, uint32_t *bad)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) {
        collide_pair(a, pa, b, pb, spec, order[t], out, bad);
    }
}

// The host-buffer call's pipeline: the pairs in chunks over three slots, each slot a stream
// and one chunk's device arrays. A chunk's upload waits for the previous chunk's (uploads go in
// order over the host link), its sort, collision and download follow on its slot's stream, so
// one chunk's manifolds come back while later chunks go up and collide. The slots' arrays stay
// allocated between calls (one set per device, grown to the largest chunk).
constexpr uint32_t kSlots = 3u;
constexpr uint32_t kChunkMin = 65536u;
constexpr uint32_t kChunksWanted = 16u;

struct Slot {
    NphGpuShape *a = nullptr, *b = nullptr;
    NphGpuPose *pa = nullptr, *pb = nullptr;
    float *spec = nullptr;
    NphGpuManifold *out = nullptr;
    uint32_t *ws = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t up = nullptr;
};

struct Pipe {
    uint32_t chunk_cap = 0;
    Slot slot[kSlots];
    uint32_t *d_bad = nullptr; // pairs of unknown types in the call
};

std::mutex g_pipe_mutex;
std::vector<Pipe> *g_pipes = nullptr; // per device; kept to the process's end

void free_slot_arrays(Slot &s)
{
    cudaFree(s.a);
    cudaFree(s.b);
    cudaFree(s.pa);
    cudaFree(s.pb);
    cudaFree(s.spec);
    cudaFree(s.out);
    cudaFree(s.ws);
    s.a = s.b = nullptr;
    s.pa = s.pb = nullptr;
    s.spec = nullptr;
    s.out = nullptr;
    s.ws = nullptr;
}

template <typename T> bool alloc(T *&p, uint64_t count)
{
    return cudaMalloc((void **)&p, sizeof(T) * count) == cudaSuccess;
}

NphGpuResult ensure_pipe(Pipe &pipe, uint32_t chunk)
{
    if (pipe.d_bad == nullptr && !alloc(pipe.d_bad, 1)) {
        cudaGetLastError();
        return NPH_GPU_OUT_OF_MEMORY;
    }
    for (Slot &s : pipe.slot) {
        if (s.st == nullptr && (cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking) != cudaSuccess ||
                                cudaEventCreateWithFlags(&s.up, cudaEventDisableTiming) != cudaSuccess)) {
            cudaGetLastError();
            return NPH_GPU_DEVICE_LOST;
        }
    }
    if (chunk <= pipe.chunk_cap) {
        return NPH_GPU_OK;
    }
    for (Slot &s : pipe.slot) {
        cudaStreamSynchronize(s.st);
        free_slot_arrays(s);
    }
    pipe.chunk_cap = 0;
    const uint64_t ws_words = nph_gpu_collide_workspace_bytes(chunk) / sizeof(uint32_t);
    for (Slot &s : pipe.slot) {
        if (!alloc(s.a, chunk) || !alloc(s.b, chunk) || !alloc(s.pa, chunk) || !alloc(s.pb, chunk) ||
            !alloc(s.spec, chunk) || !alloc(s.out, chunk) || !alloc(s.ws, ws_words)) {
            cudaGetLastError();
            for (Slot &t : pipe.slot) {
                free_slot_arrays(t);
            }
            return NPH_GPU_OUT_OF_MEMORY;
        }
    }
    pipe.chunk_cap = chunk;
    return NPH_GPU_OK;
}

} // namespace

extern "C" {

NPH_GPU_API NphGpuResult nph_gpu_collide(const NphGpuShape *a, const NphGpuPose *pose_a, const NphGpuShape *b,
                                         const NphGpuPose *pose_b, const float *speculative, uint32_t count,
                                         NphGpuManifold *out)
{
    if (count == 0) {
        return NPH_GPU_OK;
    }
    if (a == nullptr || pose_a == nullptr || b == nullptr || pose_b == nullptr || speculative == nullptr ||
        out == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return NPH_GPU_DEVICE_LOST;
    }
    std::lock_guard<std::mutex> lock(g_pipe_mutex);
    if (g_pipes == nullptr) {
        g_pipes = new (std::nothrow) std::vector<Pipe>();
        if (g_pipes == nullptr) {
            return NPH_GPU_OUT_OF_MEMORY;
        }
    }
    if (g_pipes->size() <= (size_t)device) {
        try {
            g_pipes->resize((size_t)device + 1u);
        } catch (...) {
            return NPH_GPU_OUT_OF_MEMORY;
        }
    }
    Pipe &pipe = (*g_pipes)[(size_t)device];
    const uint32_t chunk = std::min(count, std::max(kChunkMin, (count + kChunksWanted - 1u) / kChunksWanted));
    NphGpuResult r = ensure_pipe(pipe, chunk);
    if (r != NPH_GPU_OK) {
        return r;
    }
    const uint64_t ws_bytes = nph_gpu_collide_workspace_bytes(chunk);
    const uint32_t chunks = (count + chunk - 1u) / chunk;
    // Every later chunk's stream waits for the first chunk's upload, so for this too.
    cudaMemsetAsync(pipe.d_bad, 0, sizeof(uint32_t), pipe.slot[0].st);
    for (uint32_t c = 0; c < chunks && r == NPH_GPU_OK; ++c) {
        Slot &s = pipe.slot[c % kSlots];
        const uint32_t first = c * chunk;
        const uint32_t n = std::min(chunk, count - first);
        if (c > 0) {
            cudaStreamWaitEvent(s.st, pipe.slot[(c - 1u) % kSlots].up, 0);
        }
        cudaMemcpyAsync(s.a, a + first, sizeof(NphGpuShape) * n, cudaMemcpyHostToDevice, s.st);
        cudaMemcpyAsync(s.pa, pose_a + first, sizeof(NphGpuPose) * n, cudaMemcpyHostToDevice, s.st);
        cudaMemcpyAsync(s.b, b + first, sizeof(NphGpuShape) * n, cudaMemcpyHostToDevice, s.st);
        cudaMemcpyAsync(s.pb, pose_b + first, sizeof(NphGpuPose) * n, cudaMemcpyHostToDevice, s.st);
        cudaMemcpyAsync(s.spec, speculative + first, sizeof(float) * n, cudaMemcpyHostToDevice, s.st);
        cudaEventRecord(s.up, s.st);
        r = nph_gpu_collide_async(s.a, s.pa, s.b, s.pb, s.spec, n, s.out, pipe.d_bad, s.ws, ws_bytes, s.st);
        cudaMemcpyAsync(out + first, s.out, sizeof(NphGpuManifold) * n, cudaMemcpyDeviceToHost, s.st);
    }
    for (Slot &s : pipe.slot) {
        if (cudaStreamSynchronize(s.st) != cudaSuccess && r == NPH_GPU_OK) {
            r = NPH_GPU_DEVICE_LOST;
        }
    }
    if (r == NPH_GPU_OK && cudaGetLastError() != cudaSuccess) {
        r = NPH_GPU_DEVICE_LOST;
    }
    uint32_t bad = 0;
    if (r == NPH_GPU_OK && cudaMemcpy(&bad, pipe.d_bad, sizeof bad, cudaMemcpyDeviceToHost) != cudaSuccess) {
        r = NPH_GPU_DEVICE_LOST;
    }
    return r == NPH_GPU_OK && bad != 0u ? NPH_GPU_UNSUPPORTED : r;
}

NPH_GPU_API void nph_gpu_collide_release(void)
{
    std::lock_guard<std::mutex> lock(g_pipe_mutex);
    if (g_pipes == nullptr) {
        return;
    }
    int current = 0;
    cudaGetDevice(&current);
    for (size_t d = 0; d < g_pipes->size(); ++d) {
        Pipe &pipe = (*g_pipes)[d];
        if (pipe.d_bad == nullptr && pipe.slot[0].st == nullptr) {
            continue;
        }
        cudaSetDevice((int)d);
        for (Slot &s : pipe.slot) {
            if (s.st != nullptr) {
                cudaStreamSynchronize(s.st);
                cudaStreamDestroy(s.st);
            }
            if (s.up != nullptr) {
                cudaEventDestroy(s.up);
            }
            free_slot_arrays(s);
            s.st = nullptr;
            s.up = nullptr;
        }
        cudaFree(pipe.d_bad);
        pipe.d_bad = nullptr;
        pipe.chunk_cap = 0;
    }
    cudaSetDevice(current);
}

NPH_GPU_API uint64_t nph_gpu_collide_workspace_bytes(uint32_t count)
{
    return 2ull * kKinds * sizeof(uint32_t) + 2ull * count * sizeof(uint32_t);
}

NPH_GPU_API NphGpuResult nph_gpu_collide_async(const NphGpuShape *a, const NphGpuPose *pose_a, const NphGpuShape *b,
                                               const NphGpuPose *pose_b, const float *speculative, uint32_t count,
                                               NphGpuManifold *out, uint32_t *bad_pairs, void *workspace,
                                               uint64_t workspace_bytes, void *stream)
{
    if (count == 0) {
        return NPH_GPU_OK;
    }
    if (a == nullptr || pose_a == nullptr || b == nullptr || pose_b == nullptr || speculative == nullptr ||
        out == nullptr || count >= (1u << 28)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    const cudaStream_t st = (cudaStream_t)stream;
    const uint32_t blocks = (count + 255u) / 256u;
    if (workspace == nullptr) {
        k_collide<<<blocks, 256, 0, st>>>(a, pose_a, b, pose_b, speculative, count, out, bad_pairs);
    } else {
        if (workspace_bytes < nph_gpu_collide_workspace_bytes(count) || ((uintptr_t)workspace & 3u) != 0u) {
            return NPH_GPU_INVALID_ARGUMENT;
        }
        uint32_t *counts = (uint32_t *)workspace;
        uint32_t *place = counts + 2u * kKinds;
        uint32_t *order = place + count;
        cudaMemsetAsync(counts, 0, kKinds * sizeof(uint32_t), st);
        k_classify<<<blocks, 256, 0, st>>>(a, pose_a, b, pose_b, count, counts, place);
        k_kind_offsets<<<1, 32, 0, st>>>(counts);
        k_scatter<<<blocks, 256, 0, st>>>(counts, place, count, order);
        k_collide_sorted<<<blocks, 256, 0, st>>>(a, pose_a, b, pose_b, speculative, count, order, out, bad_pairs);
    }
    return cudaGetLastError() == cudaSuccess ? NPH_GPU_OK : NPH_GPU_DEVICE_LOST;
}

} // extern "C"

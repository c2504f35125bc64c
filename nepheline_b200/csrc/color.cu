// SPDX-License-Identifier: Apache-2.0
//
// The constraint graph's colouring on the device, equal bit for bit to the reference's
// sequential first-fit (graph_pick_color, engine/physics/src/island.c:34-56, applied by
// phys_graph_add / phys_graph_add_joint, island.c:77-118, one constraint at a time in
// insertion order).
//
// Sequentially, constraint i takes the first colour in its range that none of its dynamic
// bodies already holds, a body holding colour k when an earlier constraint of colour k has
// it as a dynamic body. So i's colour is a function of the colours of its lower-index
// neighbours (earlier constraints sharing a dynamic body) alone, and the sequential result
// is the unique fixpoint of
//
//     c_i = first_fit(range_i, { c_j : j < i, j shares a dynamic body with i }).
//
// The device iterates that map over all constraints at once (Jacobi rounds, double
// buffered) from all-overflow: after round r every constraint whose longest chain of
// lower-index neighbours is shorter than r holds its final colour, so the rounds stop, at
// the latest after that chain's length plus one, on the first round that changes nothing.
// Each colour's list is then the insertion order of its constraints of one kind (a colour
// keeps a contact list and a joint list, world_internal.h:363-367): a stable radix sort by
// (colour, kind) gives every constraint its slot.

#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <new>

#include "nepheline_b200.h"

namespace {

constexpr uint32_t kBlock = 256;
constexpr uint8_t kOverflow = (uint8_t)NPH_GPU_OVERFLOW;
constexpr uint32_t kRoundsPerCheck = 8;

struct Scratch {
    void *base = nullptr;
    size_t size = 0;
};

__global__ void k_check_and_count(const uint32_t *a, const uint32_t *b, const uint8_t *dyn,
                                  uint32_t count, uint32_t slots, uint32_t *degree, uint32_t *err)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) {
        return;
    }
    if (a[i] >= slots || b[i] >= slots || ((dyn[i] & 3u) == 3u && a[i] == b[i])) {
        atomicOr(err, 1u);
        return;
    }
    if ((dyn[i] & NPH_GPU_CONSTRAINT_A_DYNAMIC) != 0u) {
        atomicAdd(&degree[a[i]], 1u);
    }
    if ((dyn[i] & NPH_GPU_CONSTRAINT_B_DYNAMIC) != 0u) {
        atomicAdd(&degree[b[i]], 1u);
    }
}

__global__ void k_fill(const uint32_t *a, const uint32_t *b, const uint8_t *dyn, uint32_t count,
                       uint32_t *cursor, uint32_t *incident)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) {
        return;
    }
    if ((dyn[i] & NPH_GPU_CONSTRAINT_A_DYNAMIC) != 0u) {
        incident[atomicAdd(&cursor[a[i]], 1u)] = i;
    }
    if ((dyn[i] & NPH_GPU_CONSTRAINT_B_DYNAMIC) != 0u) {
        incident[atomicAdd(&cursor[b[i]], 1u)] = i;
    }
}

// The colours body `x` holds among constraints before i.
__device__ __forceinline__ uint32_t used_before(uint32_t x, uint32_t i, const uint32_t *offsets,
                                                const uint32_t *incident, const uint8_t *cur)
{
    uint32_t used = 0;
    const uint32_t end = offsets[x + 1];
    for (uint32_t p = offsets[x]; p < end; ++p) {
        const uint32_t j = incident[p];
        if (j < i) {
            const uint32_t c = cur[j];
            used |= c < kOverflow ? (1u << c) : 0u;
        }
    }
    return used;
}

__global__ void k_round(const uint32_t *a, const uint32_t *b, const uint8_t *dyn, uint32_t count,
                        const uint32_t *offsets, const uint32_t *incident, const uint8_t *cur,
                        uint8_t *next, uint32_t *changed)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool diff = false;
    if (i < count) {
        const uint32_t d = dyn[i];
        const bool da = (d & NPH_GPU_CONSTRAINT_A_DYNAMIC) != 0u;
        const bool db = (d & NPH_GPU_CONSTRAINT_B_DYNAMIC) != 0u;
        uint32_t color = kOverflow;
        if (da && db) {
            const uint32_t used = used_before(a[i], i, offsets, incident, cur) |
                                  used_before(b[i], i, offsets, incident, cur);
            const uint32_t free = ~used & ((1u << NPH_GPU_DYNAMIC_COLORS) - 1u);
            color = free != 0u ? (uint32_t)(__ffs(free) - 1) : kOverflow;
        } else if (da || db) {
            const uint32_t used = used_before(da ? a[i] : b[i], i, offsets, incident, cur);
            const uint32_t free = ~used & (((1u << NPH_GPU_COLORS) - 1u) & ~1u);
            color = free != 0u ? (uint32_t)(__ffs(free) - 1) : kOverflow;
        }
        next[i] = (uint8_t)color;
        diff = color != cur[i];
    }
    const uint32_t votes = __ballot_sync(0xFFFFFFFFu, diff);
    if ((threadIdx.x & 31u) == 0u && votes != 0u) {
        atomicAdd(changed, (uint32_t)__popc(votes));
    }
}

__global__ void k_keys(const uint8_t *color, const uint8_t *dyn, uint32_t count, uint8_t *keys,
                       uint32_t *index, uint32_t *bucket_count)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) {
        return;
    }
    const uint32_t key = color[i] * 2u + ((dyn[i] & NPH_GPU_CONSTRAINT_JOINT) != 0u ? 1u : 0u);
    keys[i] = (uint8_t)key;
    index[i] = i;
    atomicAdd(&bucket_count[key], 1u);
}

__global__ void k_slots(const uint8_t *sorted_keys, const uint32_t *sorted_index, uint32_t count,
                        const uint32_t *bucket_count, const uint8_t *color, uint32_t *out_color,
                        uint32_t *out_slot)
{
    __shared__ uint32_t first[2 * NPH_GPU_COLOR_SLOTS];
    if (threadIdx.x == 0) {
        uint32_t f = 0;
        for (uint32_t k = 0; k < 2u * NPH_GPU_COLOR_SLOTS; ++k) {
            first[k] = f;
            f += bucket_count[k];
        }
    }
    __syncthreads();
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) {
        return;
    }
    const uint32_t i = sorted_index[p];
    out_slot[i] = p - first[sorted_keys[p]];
    out_color[i] = color[i];
}

uint32_t blocks_for(uint64_t n) { return (uint32_t)((n + kBlock - 1) / kBlock); }

template <typename T> T *carve(char *&cursor, size_t count)
{
    const size_t bytes = ((count * sizeof(T)) + 255u) & ~(size_t)255u;
    T *p = reinterpret_cast<T *>(cursor);
    cursor += bytes;
    return p;
}

} // namespace

extern "C" {

// The solver object only lends its device and stream.
struct NphGpuSolver;
NPH_GPU_API void *nph_gpu_solver_stream(const NphGpuSolver *s);

NPH_GPU_API NphGpuResult nph_gpu_graph_color(NphGpuSolver *solver, const uint32_t *body_a,
                                             const uint32_t *body_b, const uint8_t *dynamic_bits,
                                             uint32_t count, uint32_t body_slots,
                                             uint32_t *out_color, uint32_t *out_slot)
{
    if (solver == nullptr || (count > 0 && (body_a == nullptr || body_b == nullptr ||
                                            dynamic_bits == nullptr || out_color == nullptr ||
                                            out_slot == nullptr))) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if (count == 0) {
        return NPH_GPU_OK;
    }
    cudaStream_t st = (cudaStream_t)nph_gpu_solver_stream(solver);
    // Scratch: inputs, the body adjacency, two colour buffers, the sort's keys and payload.
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint8_t *)nullptr, (uint8_t *)nullptr,
                                    (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)count, 0, 6);
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                  (int)body_slots + 1);
    const size_t n = count;
    const size_t slots = (size_t)body_slots + 1u;
    // Two passes over the same carving: the first measures, the second places.
    char *base = nullptr;
    uint32_t *d_a, *d_b, *d_color, *d_slot, *index, *index_sorted, *degree, *offsets, *cursor,
        *incident, *counters;
    uint8_t *d_dyn, *c0, *c1, *keys, *keys_sorted;
    void *sort_tmp, *scan_tmp;
    size_t total = 0;
    for (int pass = 0; pass < 2; ++pass) {
        char *cur = base;
        d_a = carve<uint32_t>(cur, n);
        d_b = carve<uint32_t>(cur, n);
        d_color = carve<uint32_t>(cur, n);
        d_slot = carve<uint32_t>(cur, n);
        d_dyn = carve<uint8_t>(cur, n);
        c0 = carve<uint8_t>(cur, n);
        c1 = carve<uint8_t>(cur, n);
        keys = carve<uint8_t>(cur, n);
        keys_sorted = carve<uint8_t>(cur, n);
        index = carve<uint32_t>(cur, n);
        index_sorted = carve<uint32_t>(cur, n);
        degree = carve<uint32_t>(cur, slots);
        offsets = carve<uint32_t>(cur, slots);
        cursor = carve<uint32_t>(cur, slots);
        incident = carve<uint32_t>(cur, 2 * n);
        counters = carve<uint32_t>(cur, 64); // [0] error, [1] changed, [2..51] buckets
        sort_tmp = carve<char>(cur, sort_bytes);
        scan_tmp = carve<char>(cur, scan_bytes);
        if (pass == 0) {
            total = (size_t)(cur - base);
            if (cudaMalloc((void **)&base, total) != cudaSuccess) {
                cudaGetLastError();
                return NPH_GPU_OUT_OF_MEMORY;
            }
        }
    }

    NphGpuResult result = NPH_GPU_OK;
    uint32_t host_counters[2] = {0, 0};
    cudaMemcpyAsync(d_a, body_a, n * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_b, body_b, n * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_dyn, dynamic_bits, n, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(degree, 0, slots * 4, st);
    cudaMemsetAsync(counters, 0, 64 * 4, st);
    k_check_and_count<<<blocks_for(n), kBlock, 0, st>>>(d_a, d_b, d_dyn, count, body_slots, degree,
                                                        counters);
    cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, degree, offsets, (int)body_slots + 1, st);
    cudaMemcpyAsync(cursor, offsets, slots * 4, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(&host_counters[0], counters, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        result = NPH_GPU_DEVICE_LOST;
    } else if (host_counters[0] != 0u) {
        result = NPH_GPU_INVALID_ARGUMENT;
    }
    if (result == NPH_GPU_OK) {
        k_fill<<<blocks_for(n), kBlock, 0, st>>>(d_a, d_b, d_dyn, count, cursor, incident);
        cudaMemsetAsync(c0, kOverflow, n, st);
        // At most count + 1 rounds: the longest chain of lower-index neighbours is shorter.
        uint8_t *in = c0;
        uint8_t *out = c1;
        uint64_t rounds = 0;
        for (;;) {
            cudaMemsetAsync(counters + 1, 0, 4, st);
            for (uint32_t r = 0; r < kRoundsPerCheck; ++r) {
                k_round<<<blocks_for(n), kBlock, 0, st>>>(d_a, d_b, d_dyn, count, offsets, incident, in,
                                                         out, counters + 1);
                uint8_t *t = in;
                in = out;
                out = t;
            }
            rounds += kRoundsPerCheck;
            cudaMemcpyAsync(&host_counters[1], counters + 1, 4, cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) {
                result = NPH_GPU_DEVICE_LOST;
                break;
            }
            // The last round of the batch changed nothing only if the counter saw no change
            // in all of them: a batch with zero changes ends the iteration.
            if (host_counters[1] == 0u) {
                break;
            }
            if (rounds > (uint64_t)count + 2u * kRoundsPerCheck) {
                result = NPH_GPU_UNKNOWN; // cannot happen: the map converges within count + 1
                break;
            }
        }
        if (result == NPH_GPU_OK) {
            uint32_t *buckets = counters + 2;
            k_keys<<<blocks_for(n), kBlock, 0, st>>>(in, d_dyn, count, keys, index, buckets);
            cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, keys, keys_sorted, index, index_sorted,
                                            (int)count, 0, 6, st);
            k_slots<<<blocks_for(n), kBlock, 0, st>>>(keys_sorted, index_sorted, count, buckets, in,
                                                      d_color, d_slot);
            cudaMemcpyAsync(out_color, d_color, n * 4, cudaMemcpyDeviceToHost, st);
            cudaMemcpyAsync(out_slot, d_slot, n * 4, cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) {
                result = NPH_GPU_DEVICE_LOST;
            }
        }
    }
    cudaFree(base);
    return result;
}

} // extern "C"

// ------------------------------------------------------------------------------------
// The colouring without allocation
//
// For callers that may not allocate device memory once they run: an engine that reserves
// all of its device memory up front, a frame loop with a fixed memory budget, a process
// whose allocator is owned by another runtime, code recorded into work that must not
// allocate. The scratch the colouring needs lives in one file-scope device array of fixed
// size, which every GPU that loads this library holds until the process exits. The host
// cannot use the array's name as a device address (in host code it names a host-side
// stand-in), so the first call on each device asks the runtime for the address once, with
// that device current, and keeps it.
// ------------------------------------------------------------------------------------

namespace {

constexpr uint32_t kStaticMaxConstraints = NPH_GPU_GRAPH_COLOR_STATIC_MAX_CONSTRAINTS;
constexpr uint32_t kStaticMaxBodySlots = NPH_GPU_GRAPH_COLOR_STATIC_MAX_BODY_SLOTS;
constexpr size_t kStaticScratchBytes = (size_t)NPH_GPU_GRAPH_COLOR_STATIC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_color_scratch[kStaticScratchBytes];

struct StaticScratch {
    std::atomic<int> state[kMaxDevices]; // 0 unset, 1 being set, 2 set
    void *ptr[kMaxDevices];
};
StaticScratch g_static;

// The device address of g_color_scratch on the current device (first call: looked up).
NphGpuResult static_scratch(int device, unsigned char **out)
{
    if (device < 0 || device >= kMaxDevices) {
        return NPH_GPU_UNSUPPORTED;
    }
    int expected = 0;
    if (g_static.state[device].compare_exchange_strong(expected, 1)) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_color_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            g_static.state[device].store(0);
            return NPH_GPU_DEVICE_LOST;
        }
        g_static.ptr[device] = p;
        g_static.state[device].store(2);
    }
    while (g_static.state[device].load() != 2) {
        if (g_static.state[device].load() == 0) {
            return NPH_GPU_DEVICE_LOST; // another thread's lookup failed
        }
    }
    *out = (unsigned char *)g_static.ptr[device];
    return NPH_GPU_OK;
}

} // namespace

extern "C" {

NPH_GPU_API NphGpuResult nph_gpu_graph_color_static(void *stream, const uint32_t *body_a,
                                                    const uint32_t *body_b,
                                                    const uint8_t *dynamic_bits, uint32_t count,
                                                    uint32_t body_slots, uint32_t *out_color,
                                                    uint32_t *out_slot)
{
    if (count > 0 && (body_a == nullptr || body_b == nullptr || dynamic_bits == nullptr ||
                      out_color == nullptr || out_slot == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if (count > kStaticMaxConstraints || body_slots > kStaticMaxBodySlots) {
        return NPH_GPU_TOO_LARGE;
    }
    if (count == 0) {
        return NPH_GPU_OK;
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return NPH_GPU_DEVICE_LOST;
    }
    unsigned char *base = nullptr;
    NphGpuResult result = static_scratch(device, &base);
    if (result != NPH_GPU_OK) {
        return result;
    }
    cudaStream_t st = (cudaStream_t)stream;
    // The sort's and the scan's temporary storage, for these sizes, must fit what is left.
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint8_t *)nullptr, (uint8_t *)nullptr,
                                    (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)count, 0, 6);
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                  (int)body_slots + 1);
    const size_t n = count;
    const size_t slots = (size_t)body_slots + 1u;
    char *cur = (char *)base;
    uint32_t *d_a = carve<uint32_t>(cur, n);
    uint32_t *d_b = carve<uint32_t>(cur, n);
    uint32_t *d_color = carve<uint32_t>(cur, n);
    uint32_t *d_slot = carve<uint32_t>(cur, n);
    uint8_t *d_dyn = carve<uint8_t>(cur, n);
    uint8_t *c0 = carve<uint8_t>(cur, n);
    uint8_t *c1 = carve<uint8_t>(cur, n);
    uint8_t *keys = carve<uint8_t>(cur, n);
    uint8_t *keys_sorted = carve<uint8_t>(cur, n);
    uint32_t *index = carve<uint32_t>(cur, n);
    uint32_t *index_sorted = carve<uint32_t>(cur, n);
    uint32_t *degree = carve<uint32_t>(cur, slots);
    uint32_t *offsets = carve<uint32_t>(cur, slots);
    uint32_t *cursor = carve<uint32_t>(cur, slots);
    uint32_t *incident = carve<uint32_t>(cur, 2 * n);
    uint32_t *counters = carve<uint32_t>(cur, 64);
    void *sort_tmp = carve<char>(cur, sort_bytes);
    void *scan_tmp = carve<char>(cur, scan_bytes);
    if ((size_t)(cur - (char *)base) > kStaticScratchBytes) {
        return NPH_GPU_TOO_LARGE;
    }

    // The array keeps the last call's contents: what must start at zero is cleared here.
    uint32_t host_counters[2] = {0, 0};
    cudaMemcpyAsync(d_a, body_a, n * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_b, body_b, n * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_dyn, dynamic_bits, n, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(degree, 0, slots * 4, st);
    cudaMemsetAsync(counters, 0, 64 * 4, st);
    k_check_and_count<<<blocks_for(n), kBlock, 0, st>>>(d_a, d_b, d_dyn, count, body_slots, degree,
                                                        counters);
    cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, degree, offsets, (int)body_slots + 1, st);
    cudaMemcpyAsync(cursor, offsets, slots * 4, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(&host_counters[0], counters, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return NPH_GPU_DEVICE_LOST;
    }
    if (host_counters[0] != 0u) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    k_fill<<<blocks_for(n), kBlock, 0, st>>>(d_a, d_b, d_dyn, count, cursor, incident);
    cudaMemsetAsync(c0, kOverflow, n, st);
    uint8_t *in = c0;
    uint8_t *out = c1;
    uint64_t rounds = 0;
    for (;;) {
        cudaMemsetAsync(counters + 1, 0, 4, st);
        for (uint32_t r = 0; r < kRoundsPerCheck; ++r) {
            k_round<<<blocks_for(n), kBlock, 0, st>>>(d_a, d_b, d_dyn, count, offsets, incident, in, out,
                                                     counters + 1);
            uint8_t *t = in;
            in = out;
            out = t;
        }
        rounds += kRoundsPerCheck;
        cudaMemcpyAsync(&host_counters[1], counters + 1, 4, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            return NPH_GPU_DEVICE_LOST;
        }
        if (host_counters[1] == 0u) {
            break;
        }
        if (rounds > (uint64_t)count + 2u * kRoundsPerCheck) {
            return NPH_GPU_UNKNOWN;
        }
    }
    uint32_t *buckets = counters + 2;
    k_keys<<<blocks_for(n), kBlock, 0, st>>>(in, d_dyn, count, keys, index, buckets);
    cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, keys, keys_sorted, index, index_sorted,
                                    (int)count, 0, 6, st);
    k_slots<<<blocks_for(n), kBlock, 0, st>>>(keys_sorted, index_sorted, count, buckets, in, d_color,
                                              d_slot);
    cudaMemcpyAsync(out_color, d_color, n * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(out_slot, d_slot, n * 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return NPH_GPU_DEVICE_LOST;
    }
    return NPH_GPU_OK;
}

} // extern "C"

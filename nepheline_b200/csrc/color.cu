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

#include <climits>
#include <cstdint>
#include <cstring>
#include <new>

#include "nepheline_b200.h"
#include "solver_link.h"

namespace {

constexpr uint32_t kBlock = 256;
constexpr uint8_t kOverflow = (uint8_t)NPH_GPU_OVERFLOW;
constexpr uint32_t kRoundsPerCheck = 8;

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

// The first-fit rule itself, in insertion order, over a colour mask per body slot (bit k: the
// body is a dynamic body of a constraint of colour k). This is the reference's sequential
// algorithm (graph_pick_color over per-colour body sets, island.c:34-56) and gives the fixpoint
// the rounds converge to; it finishes the colouring when the rounds would take too many
// launches (a long chain of constraints, each sharing a body with the one before it: a rope or
// a stack inserted in order). One warp takes 32 constraints at a time: each lane loads its
// constraint and its bodies' masks as they were before the batch, then the lanes decide one
// after another, each choice broadcast so later lanes on the same body add its colour.
__global__ void k_sequential_first_fit(const uint32_t *a, const uint32_t *b, const uint8_t *dyn,
                                       uint32_t count, uint32_t *mask, uint8_t *color)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32u) {
        return;
    }
    const uint32_t lane = threadIdx.x;
    for (uint32_t base = 0; base < count; base += 32u) {
        const uint32_t i = base + lane;
        const bool valid = i < count;
        const uint32_t ai = valid ? a[i] : 0u;
        const uint32_t bi = valid ? b[i] : 0u;
        const uint32_t d = valid ? (uint32_t)dyn[i] : 0u;
        const bool da = (d & NPH_GPU_CONSTRAINT_A_DYNAMIC) != 0u;
        const bool db = (d & NPH_GPU_CONSTRAINT_B_DYNAMIC) != 0u;
        // L2 reads: the masks were changed by atomics of earlier batches.
        uint32_t ma = da ? __ldcg(&mask[ai]) : 0u;
        uint32_t mb = db ? __ldcg(&mask[bi]) : 0u;
        uint32_t mine = kOverflow;
        for (uint32_t k = 0; k < 32u; ++k) {
            if (lane == k) {
                if (da && db) {
                    const uint32_t free = ~(ma | mb) & ((1u << NPH_GPU_DYNAMIC_COLORS) - 1u);
                    mine = free != 0u ? (uint32_t)(__ffs(free) - 1) : kOverflow;
                } else if (da || db) {
                    const uint32_t free = ~(da ? ma : mb) & (((1u << NPH_GPU_COLORS) - 1u) & ~1u);
                    mine = free != 0u ? (uint32_t)(__ffs(free) - 1) : kOverflow;
                }
            }
            const uint32_t ck = __shfl_sync(0xFFFFFFFFu, mine, (int)k);
            const uint32_t ak = __shfl_sync(0xFFFFFFFFu, ai, (int)k);
            const uint32_t bk = __shfl_sync(0xFFFFFFFFu, bi, (int)k);
            const uint32_t dk = __shfl_sync(0xFFFFFFFFu, d, (int)k);
            if (lane > k && ck < kOverflow) {
                const bool ka = (dk & NPH_GPU_CONSTRAINT_A_DYNAMIC) != 0u;
                const bool kb = (dk & NPH_GPU_CONSTRAINT_B_DYNAMIC) != 0u;
                const uint32_t bit = 1u << ck;
                if (da && ((ka && ak == ai) || (kb && bk == ai))) {
                    ma |= bit;
                }
                if (db && ((ka && ak == bi) || (kb && bk == bi))) {
                    mb |= bit;
                }
            }
        }
        if (valid) {
            color[i] = (uint8_t)mine;
            if (mine < kOverflow) {
                if (da) {
                    atomicOr(&mask[ai], 1u << mine);
                }
                if (db) {
                    atomicOr(&mask[bi], 1u << mine);
                }
            }
        }
        __threadfence();
        __syncwarp();
    }
}

template <typename T> T *carve(char *&cursor, size_t count)
{
    const size_t bytes = ((count * sizeof(T)) + 255u) & ~(size_t)255u;
    T *p = reinterpret_cast<T *>(cursor);
    cursor += bytes;
    return p;
}

// Every scratch array of one colouring, carved in order from one base address.
struct Carving {
    uint32_t *a, *b, *color, *slot, *index, *index_sorted, *degree, *offsets, *cursor, *incident,
        *counters; // counters: [0] error, [1] changed, [2..51] the (colour, kind) buckets
    uint8_t *dyn, *c0, *c1, *keys, *keys_sorted;
    void *sort_tmp, *scan_tmp;
    size_t sort_bytes, scan_bytes;
};

// Places the arrays from `base` (nullptr: measures only) and returns the bytes they span.
size_t carve_all(char *base, size_t n, size_t slots, size_t sort_bytes, size_t scan_bytes,
                 Carving *c)
{
    char *cur = base;
    c->a = carve<uint32_t>(cur, n);
    c->b = carve<uint32_t>(cur, n);
    c->color = carve<uint32_t>(cur, n);
    c->slot = carve<uint32_t>(cur, n);
    c->dyn = carve<uint8_t>(cur, n);
    c->c0 = carve<uint8_t>(cur, n);
    c->c1 = carve<uint8_t>(cur, n);
    c->keys = carve<uint8_t>(cur, n);
    c->keys_sorted = carve<uint8_t>(cur, n);
    c->index = carve<uint32_t>(cur, n);
    c->index_sorted = carve<uint32_t>(cur, n);
    c->degree = carve<uint32_t>(cur, slots);
    c->offsets = carve<uint32_t>(cur, slots);
    c->cursor = carve<uint32_t>(cur, slots);
    c->incident = carve<uint32_t>(cur, 2 * n);
    c->counters = carve<uint32_t>(cur, 64);
    c->sort_tmp = carve<char>(cur, sort_bytes);
    c->scan_tmp = carve<char>(cur, scan_bytes);
    c->sort_bytes = sort_bytes;
    c->scan_bytes = scan_bytes;
    return (size_t)(cur - base);
}

// The temporary storage the library's sort and scan need for these sizes.
void temp_bytes(uint32_t count, uint32_t body_slots, size_t *sort_bytes, size_t *scan_bytes)
{
    *sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, *sort_bytes, (const uint8_t *)nullptr, (uint8_t *)nullptr,
                                    (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)count, 0, 6);
    *scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, *scan_bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                  (int)body_slots + 1);
}

// A launch that failed to start leaves no error on the stream: it is read here, before any
// result is trusted.
NphGpuResult launch_status()
{
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        return NPH_GPU_OK;
    }
    return e == cudaErrorInvalidResourceHandle || e == cudaErrorInvalidValue ||
                   e == cudaErrorInvalidDevice
               ? NPH_GPU_INVALID_ARGUMENT
               : NPH_GPU_DEVICE_LOST;
}

NphGpuResult sync_status(cudaStream_t st)
{
    const NphGpuResult launched = launch_status();
    const cudaError_t e = cudaStreamSynchronize(st);
    if (launched != NPH_GPU_OK) {
        return launched;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e == cudaErrorInvalidResourceHandle ? NPH_GPU_INVALID_ARGUMENT : NPH_GPU_DEVICE_LOST;
    }
    return NPH_GPU_OK;
}

// Rounds of the fixpoint before the sequential rule takes over: a round costs a launch (a few
// microseconds) or, on large graphs, about a pass over the incidence lists in L2, while the
// warp's sequential pass costs about 60 ns a constraint; so the rounds get at least 512 and
// one for every 512 constraints. The 1,048,576-body lattice (3.4 M constraints) needs at
// most 320 rounds, a rope of n links n.
uint64_t max_rounds(uint32_t count) { return count / 512u > 512u ? count / 512u : 512u; }

// The colouring on scratch already carved: both entry points run this. Inputs are host arrays;
// every array that must start at zero is cleared here (the allocation-free entry's scratch
// keeps the previous call's contents).
NphGpuResult colour_graph(const Carving &c, cudaStream_t st, const uint32_t *body_a,
                          const uint32_t *body_b, const uint8_t *dynamic_bits, uint32_t count,
                          uint32_t body_slots, uint32_t *out_color, uint32_t *out_slot)
{
    const size_t n = count;
    const size_t slots = (size_t)body_slots + 1u;
    uint32_t host_counters[2] = {0, 0};
    cudaMemcpyAsync(c.a, body_a, n * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(c.b, body_b, n * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(c.dyn, dynamic_bits, n, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(c.degree, 0, slots * 4, st);
    cudaMemsetAsync(c.counters, 0, 64 * 4, st);
    k_check_and_count<<<blocks_for(n), kBlock, 0, st>>>(c.a, c.b, c.dyn, count, body_slots, c.degree,
                                                        c.counters);
    size_t scan_bytes = c.scan_bytes;
    cub::DeviceScan::ExclusiveSum(c.scan_tmp, scan_bytes, c.degree, c.offsets, (int)body_slots + 1, st);
    cudaMemcpyAsync(c.cursor, c.offsets, slots * 4, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(&host_counters[0], c.counters, 4, cudaMemcpyDeviceToHost, st);
    NphGpuResult result = sync_status(st);
    if (result != NPH_GPU_OK) {
        return result;
    }
    if (host_counters[0] != 0u) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    k_fill<<<blocks_for(n), kBlock, 0, st>>>(c.a, c.b, c.dyn, count, c.cursor, c.incident);
    cudaMemsetAsync(c.c0, kOverflow, n, st);
    // After round r every constraint whose longest chain of lower-index neighbours is shorter
    // than r holds its final colour, so a batch of rounds that changes nothing ends the
    // iteration. A longer chain (one launch per round) goes to the sequential rule instead.
    uint8_t *in = c.c0;
    uint8_t *out = c.c1;
    uint64_t rounds = 0;
    for (;;) {
        cudaMemsetAsync(c.counters + 1, 0, 4, st);
        for (uint32_t r = 0; r < kRoundsPerCheck; ++r) {
            k_round<<<blocks_for(n), kBlock, 0, st>>>(c.a, c.b, c.dyn, count, c.offsets, c.incident, in,
                                                     out, c.counters + 1);
            uint8_t *t = in;
            in = out;
            out = t;
        }
        rounds += kRoundsPerCheck;
        cudaMemcpyAsync(&host_counters[1], c.counters + 1, 4, cudaMemcpyDeviceToHost, st);
        result = sync_status(st);
        if (result != NPH_GPU_OK) {
            return result;
        }
        if (host_counters[1] == 0u) {
            break;
        }
        if (rounds >= max_rounds(count)) {
            // cursor is free once the incidence lists are filled: it holds the body masks.
            cudaMemsetAsync(c.cursor, 0, slots * 4, st);
            k_sequential_first_fit<<<1, 32, 0, st>>>(c.a, c.b, c.dyn, count, c.cursor, in);
            break;
        }
    }
    uint32_t *buckets = c.counters + 2;
    k_keys<<<blocks_for(n), kBlock, 0, st>>>(in, c.dyn, count, c.keys, c.index, buckets);
    size_t sort_bytes = c.sort_bytes;
    cub::DeviceRadixSort::SortPairs(c.sort_tmp, sort_bytes, c.keys, c.keys_sorted, c.index,
                                    c.index_sorted, (int)count, 0, 6, st);
    k_slots<<<blocks_for(n), kBlock, 0, st>>>(c.keys_sorted, c.index_sorted, count, buckets, in,
                                              c.color, c.slot);
    cudaMemcpyAsync(out_color, c.color, n * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(out_slot, c.slot, n * 4, cudaMemcpyDeviceToHost, st);
    return sync_status(st);
}

} // namespace

extern "C" {

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
    // The library's sort and scan count items in int; the incidence lists hold 2 count.
    if (count > (uint32_t)(INT32_MAX / 2) || body_slots >= (uint32_t)INT32_MAX) {
        return NPH_GPU_TOO_LARGE;
    }
    if (count == 0) {
        return NPH_GPU_OK;
    }
    if (cudaSetDevice(nph_solver_device(solver)) != cudaSuccess) {
        cudaGetLastError();
        return NPH_GPU_DEVICE_LOST;
    }
    cudaStream_t st = (cudaStream_t)nph_gpu_solver_stream(solver);
    size_t sort_bytes = 0, scan_bytes = 0;
    temp_bytes(count, body_slots, &sort_bytes, &scan_bytes);
    Carving c{};
    const size_t total = carve_all(nullptr, count, (size_t)body_slots + 1u, sort_bytes, scan_bytes, &c);
    char *base = nullptr;
    if (cudaMalloc((void **)&base, total) != cudaSuccess) {
        cudaGetLastError();
        return NPH_GPU_OUT_OF_MEMORY;
    }
    carve_all(base, count, (size_t)body_slots + 1u, sort_bytes, scan_bytes, &c);
    const NphGpuResult result =
        colour_graph(c, st, body_a, body_b, dynamic_bits, count, body_slots, out_color, out_slot);
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
// stand-in), so each call asks the runtime for the array's address in the current context,
// with the caller's device current: an address kept from an earlier call could belong to a
// context that has since been destroyed (cudaDeviceReset) or to another context the caller
// made current. After the first call in a context, which loads the module, the lookup is cheap.
// ------------------------------------------------------------------------------------

namespace {

constexpr uint32_t kStaticMaxConstraints = NPH_GPU_GRAPH_COLOR_STATIC_MAX_CONSTRAINTS;
constexpr uint32_t kStaticMaxBodySlots = NPH_GPU_GRAPH_COLOR_STATIC_MAX_BODY_SLOTS;
constexpr size_t kStaticScratchBytes = (size_t)NPH_GPU_GRAPH_COLOR_STATIC_SCRATCH_BYTES;

__device__ __align__(256) unsigned char g_color_scratch[kStaticScratchBytes];

// The device address of g_color_scratch in the current context.
NphGpuResult static_scratch(unsigned char **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_color_scratch);
    if (e != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        return NPH_GPU_DEVICE_LOST;
    }
    *out = (unsigned char *)p;
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
    unsigned char *base = nullptr;
    NphGpuResult result = static_scratch(&base);
    if (result != NPH_GPU_OK) {
        return result;
    }
    size_t sort_bytes = 0, scan_bytes = 0;
    temp_bytes(count, body_slots, &sort_bytes, &scan_bytes);
    Carving c{};
    if (carve_all(nullptr, count, (size_t)body_slots + 1u, sort_bytes, scan_bytes, &c) >
        kStaticScratchBytes) {
        return NPH_GPU_TOO_LARGE;
    }
    carve_all((char *)base, count, (size_t)body_slots + 1u, sort_bytes, scan_bytes, &c);
    return colour_graph(c, (cudaStream_t)stream, body_a, body_b, dynamic_bits, count, body_slots,
                        out_color, out_slot);
}

} // extern "C"

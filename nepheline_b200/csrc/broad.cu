// SPDX-License-Identifier: Apache-2.0
//
// The stages either side of the narrow phase for worlds the library steps itself, on the device:
//
//   nph_gpu_broad_phase          the pairs of boxes whose bounding boxes overlap, within each
//                                group (world): the reference keeps them in AABB trees and pairs
//                                fattened boxes (phys_update_pairs, contact.c:811; boxes_overlap,
//                                contact.c:286-290); here a uniform grid of cells at least as
//                                large as any box, a radix sort of the boxes by cell, and one
//                                thread per box scanning the 27 cells around its own;
//   nph_gpu_warm_start_contacts  phys_contact_update's warm start (contact.c:516-565) over host
//                                arrays of last step's records and this step's narrow-phase
//                                records, pair by pair (warm_match.h).
//
// Both allocate their device arrays per call: they serve scene generation and tests, not the
// solver stage's steady state.

#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <cmath>
#include <cstdint>

#include "nepheline_b200.h"
#include "warm_match.h"

namespace {

constexpr uint32_t kBlock = 256;
constexpr int kCoordBias = 1 << 15;

uint32_t blocks_for(uint64_t n) { return (uint32_t)((n + kBlock - 1) / kBlock); }

// A cell's key: the group in the top 16 bits, then the cell's coordinates biased by 2^15.
__device__ __forceinline__ uint64_t cell_key(uint32_t group, int x, int y, int z)
{
    return ((uint64_t)(group & 0xFFFFu) << 48) | ((uint64_t)(uint32_t)(x + kCoordBias) & 0xFFFFu) << 32 |
           ((uint64_t)(uint32_t)(y + kCoordBias) & 0xFFFFu) << 16 | ((uint64_t)(uint32_t)(z + kCoordBias) & 0xFFFFu);
}

__device__ __forceinline__ int cell_of(float v, float inv_cell) { return (int)floorf(v * inv_cell); }

__global__ void k_keys(const float3 *lo, const uint32_t *group, uint32_t n, float inv_cell, uint64_t *keys,
                       uint32_t *index)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const float3 p = lo[i];
    keys[i] = cell_key(group[i], cell_of(p.x, inv_cell), cell_of(p.y, inv_cell), cell_of(p.z, inv_cell));
    index[i] = i;
}

// The first position in sorted[0..n) whose key is not below k.
__device__ uint32_t lower_bound(const uint64_t *sorted, uint32_t n, uint64_t k)
{
    uint32_t a = 0, b = n;
    while (a < b) {
        const uint32_t m = (a + b) >> 1;
        if (sorted[m] < k) {
            a = m + 1;
        } else {
            b = m;
        }
    }
    return a;
}

// Box i against the boxes of the 27 cells around its own, each pair once (from its lower index).
__global__ void k_pairs(const float3 *lo, const float3 *hi, const uint32_t *group, uint32_t n, float inv_cell,
                        const uint64_t *sorted_keys, const uint32_t *sorted_index, uint64_t *pairs,
                        uint32_t capacity, uint32_t *counter)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const float3 a0 = lo[i], a1 = hi[i];
    const uint32_t g = group[i];
    const int cx = cell_of(a0.x, inv_cell), cy = cell_of(a0.y, inv_cell), cz = cell_of(a0.z, inv_cell);
    for (int dx = -1; dx <= 1; ++dx) {
        for (int dy = -1; dy <= 1; ++dy) {
            for (int dz = -1; dz <= 1; ++dz) {
                const uint64_t k = cell_key(g, cx + dx, cy + dy, cz + dz);
                for (uint32_t p = lower_bound(sorted_keys, n, k); p < n && sorted_keys[p] == k; ++p) {
                    const uint32_t j = sorted_index[p];
                    if (j <= i || group[j] != g) { // keys hold 16 bits of the group
                        continue;
                    }
                    const float3 b0 = lo[j], b1 = hi[j];
                    if (a0.x <= b1.x && b0.x <= a1.x && a0.y <= b1.y && b0.y <= a1.y && a0.z <= b1.z &&
                        b0.z <= a1.z) {
                        const uint32_t at = atomicAdd(counter, 1u);
                        if (at < capacity) {
                            pairs[at] = ((uint64_t)i << 32) | j;
                        }
                    }
                }
            }
        }
    }
}

__global__ void k_split(const uint64_t *pairs, uint32_t count, uint32_t *a, uint32_t *b)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        a[i] = (uint32_t)(pairs[i] >> 32);
        b[i] = (uint32_t)pairs[i];
    }
}

__global__ void k_warm(const NphGpuContact *old, const NphGpuContact *fresh, uint32_t count, NphGpuContact *out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        NphGpuContact c;
        nph_warm_update(&old[i], &fresh[i], &c);
        out[i] = c;
    }
}

NphGpuResult status(cudaError_t e)
{
    if (e == cudaSuccess) {
        return NPH_GPU_OK;
    }
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? NPH_GPU_OUT_OF_MEMORY : NPH_GPU_DEVICE_LOST;
}

} // namespace

extern "C" {

NPH_GPU_API NphGpuResult nph_gpu_broad_phase(const float *lo, const float *hi, const uint32_t *group,
                                             uint32_t count, float cell, uint32_t *pair_a, uint32_t *pair_b,
                                             uint32_t capacity, uint32_t *pair_count)
{
    if (pair_count == nullptr || (count > 0 && (lo == nullptr || hi == nullptr || group == nullptr)) ||
        (capacity > 0 && (pair_a == nullptr || pair_b == nullptr)) || !(cell > 0.0f) || !std::isfinite(cell)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    *pair_count = 0;
    if (count < 2) {
        return NPH_GPU_OK;
    }
    if (count > (1u << 30)) {
        return NPH_GPU_TOO_LARGE;
    }
    const size_t n = count;
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                    (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)count);
    size_t pair_sort_bytes = 0;
    const uint32_t cap = capacity;
    cub::DeviceRadixSort::SortKeys(nullptr, pair_sort_bytes, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                   (int)(cap > 0 ? cap : 1));
    float3 *d_lo = nullptr, *d_hi = nullptr;
    uint32_t *d_group = nullptr, *d_index = nullptr, *d_sorted_index = nullptr, *d_counter = nullptr, *d_a = nullptr,
             *d_b = nullptr;
    uint64_t *d_keys = nullptr, *d_sorted_keys = nullptr, *d_pairs = nullptr, *d_pairs_sorted = nullptr;
    void *d_tmp = nullptr;
    const size_t tmp_bytes = sort_bytes > pair_sort_bytes ? sort_bytes : pair_sort_bytes;
    cudaStream_t st = nullptr;
    NphGpuResult r = status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const size_t pcap = cap > 0 ? cap : 1;
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_lo, n * sizeof(float3)));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_hi, n * sizeof(float3)));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_group, n * 4));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_index, n * 4));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_sorted_index, n * 4));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_keys, n * 8));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_sorted_keys, n * 8));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_counter, 4));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_pairs, pcap * 8));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_pairs_sorted, pcap * 8));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_a, pcap * 4));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_b, pcap * 4));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc(&d_tmp, tmp_bytes > 0 ? tmp_bytes : 1));
    }
    uint32_t found = 0;
    if (r == NPH_GPU_OK) {
        cudaMemcpyAsync(d_lo, lo, n * sizeof(float3), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_hi, hi, n * sizeof(float3), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_group, group, n * 4, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(d_counter, 0, 4, st);
        const float inv_cell = 1.0f / cell;
        k_keys<<<blocks_for(n), kBlock, 0, st>>>(d_lo, d_group, count, inv_cell, d_keys, d_index);
        size_t bytes = sort_bytes;
        cub::DeviceRadixSort::SortPairs(d_tmp, bytes, d_keys, d_sorted_keys, d_index, d_sorted_index, (int)count, 0,
                                        64, st);
        k_pairs<<<blocks_for(n), kBlock, 0, st>>>(d_lo, d_hi, d_group, count, inv_cell, d_sorted_keys,
                                                  d_sorted_index, d_pairs, cap, d_counter);
        cudaMemcpyAsync(&found, d_counter, 4, cudaMemcpyDeviceToHost, st);
        r = status(cudaStreamSynchronize(st));
        if (r == NPH_GPU_OK) {
            r = status(cudaGetLastError());
        }
    }
    if (r == NPH_GPU_OK) {
        *pair_count = found;
        const uint32_t kept = found < cap ? found : cap;
        if (kept > 0) {
            // In index order, so the caller's constraint order does not depend on thread timing.
            size_t bytes = pair_sort_bytes;
            cub::DeviceRadixSort::SortKeys(d_tmp, bytes, d_pairs, d_pairs_sorted, (int)kept, 0, 64, st);
            k_split<<<blocks_for(kept), kBlock, 0, st>>>(d_pairs_sorted, kept, d_a, d_b);
            cudaMemcpyAsync(pair_a, d_a, (size_t)kept * 4, cudaMemcpyDeviceToHost, st);
            cudaMemcpyAsync(pair_b, d_b, (size_t)kept * 4, cudaMemcpyDeviceToHost, st);
            r = status(cudaStreamSynchronize(st));
        }
    }
    cudaFree(d_lo);
    cudaFree(d_hi);
    cudaFree(d_group);
    cudaFree(d_index);
    cudaFree(d_sorted_index);
    cudaFree(d_keys);
    cudaFree(d_sorted_keys);
    cudaFree(d_counter);
    cudaFree(d_pairs);
    cudaFree(d_pairs_sorted);
    cudaFree(d_a);
    cudaFree(d_b);
    cudaFree(d_tmp);
    if (st != nullptr) {
        cudaStreamDestroy(st);
    }
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_warm_start_contacts(const NphGpuContact *old, const NphGpuContact *fresh,
                                                     uint32_t count, NphGpuContact *out)
{
    if (count > 0 && (old == nullptr || fresh == nullptr || out == nullptr)) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    if (count == 0) {
        return NPH_GPU_OK;
    }
    const size_t bytes = (size_t)count * sizeof(NphGpuContact);
    NphGpuContact *d_old = nullptr, *d_fresh = nullptr, *d_out = nullptr;
    cudaStream_t st = nullptr;
    NphGpuResult r = status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_old, bytes));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_fresh, bytes));
    }
    if (r == NPH_GPU_OK) {
        r = status(cudaMalloc((void **)&d_out, bytes));
    }
    if (r == NPH_GPU_OK) {
        cudaMemcpyAsync(d_old, old, bytes, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_fresh, fresh, bytes, cudaMemcpyHostToDevice, st);
        k_warm<<<blocks_for(count), kBlock, 0, st>>>(d_old, d_fresh, count, d_out);
        cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, st);
        r = status(cudaStreamSynchronize(st));
        if (r == NPH_GPU_OK) {
            r = status(cudaGetLastError());
        }
    }
    cudaFree(d_old);
    cudaFree(d_fresh);
    cudaFree(d_out);
    if (st != nullptr) {
        cudaStreamDestroy(st);
    }
    return r;
}

} // extern "C"

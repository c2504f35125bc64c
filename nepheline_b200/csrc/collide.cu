// SPDX-License-Identifier: Apache-2.0
//
// The narrow phase's closed-form pairs (collide.cuh), one thread per pair.

#include <cuda_runtime.h>

#include "nepheline_b200.h"

#include "collide.cuh"

namespace {

__global__ void __launch_bounds__(256) k_collide(const NphGpuShape *a, const NphGpuPose *pa, const NphGpuShape *b,
                                                 const NphGpuPose *pb, const float *spec, uint32_t count,
                                                 NphGpuManifold *out, uint32_t *bad)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) {
        return;
    }
    if (a[i].type > NPH_GPU_SHAPE_BOX || b[i].type > NPH_GPU_SHAPE_BOX) {
        // An unknown type: the cleared manifold, and the pair counted.
        NphGpuManifold m;
        m.normal[0] = 0.0f;
        m.normal[1] = 1.0f;
        m.normal[2] = 0.0f;
        m.point_count = 0u;
        for (uint32_t k = 0; k < NPH_GPU_MAX_POINTS; ++k) {
            m.points[k] = NphGpuManifoldPoint{{0.0f, 0.0f, 0.0f}, 0.0f, 0u};
        }
        out[i] = m;
        if (bad != nullptr) {
            atomicAdd(bad, 1u);
        }
        return;
    }
    NphGpuManifold m;
    for (uint32_t k = 0; k < NPH_GPU_MAX_POINTS; ++k) {
        m.points[k] = NphGpuManifoldPoint{{0.0f, 0.0f, 0.0f}, 0.0f, 0u};
    }
    nph_nc::collide(a[i], pa[i], b[i], pb[i], spec[i], m);
    out[i] = m;
}

// Spheres, capsules and boxes, every pair of them.
bool supported(uint32_t ta, uint32_t tb) { return ta <= NPH_GPU_SHAPE_BOX && tb <= NPH_GPU_SHAPE_BOX; }

template <typename T> NphGpuResult stage(T *&dst, const T *src, uint32_t count, cudaStream_t st)
{
    if (cudaMalloc((void **)&dst, sizeof(T) * count) != cudaSuccess) {
        cudaGetLastError();
        return NPH_GPU_OUT_OF_MEMORY;
    }
    if (src != nullptr) {
        cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyHostToDevice, st);
    }
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
    for (uint32_t i = 0; i < count; ++i) {
        if (!supported(a[i].type, b[i].type)) {
            return NPH_GPU_UNSUPPORTED;
        }
    }
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return NPH_GPU_DEVICE_LOST;
    }
    NphGpuShape *da = nullptr, *db = nullptr;
    NphGpuPose *dpa = nullptr, *dpb = nullptr;
    float *ds = nullptr;
    NphGpuManifold *dout = nullptr;
    NphGpuResult r = stage(da, a, count, st);
    if (r == NPH_GPU_OK) r = stage(db, b, count, st);
    if (r == NPH_GPU_OK) r = stage(dpa, pose_a, count, st);
    if (r == NPH_GPU_OK) r = stage(dpb, pose_b, count, st);
    if (r == NPH_GPU_OK) r = stage(ds, speculative, count, st);
    if (r == NPH_GPU_OK) r = stage(dout, (const NphGpuManifold *)nullptr, count, st);
    if (r == NPH_GPU_OK) {
        k_collide<<<(count + 255u) / 256u, 256, 0, st>>>(da, dpa, db, dpb, ds, count, dout, nullptr);
        cudaMemcpyAsync(out, dout, sizeof(NphGpuManifold) * count, cudaMemcpyDeviceToHost, st);
        const cudaError_t e = cudaStreamSynchronize(st);
        r = e == cudaSuccess ? NPH_GPU_OK : NPH_GPU_DEVICE_LOST;
    }
    cudaFree(da);
    cudaFree(db);
    cudaFree(dpa);
    cudaFree(dpb);
    cudaFree(ds);
    cudaFree(dout);
    cudaStreamDestroy(st);
    return r;
}

NPH_GPU_API NphGpuResult nph_gpu_collide_async(const NphGpuShape *a, const NphGpuPose *pose_a, const NphGpuShape *b,
                                               const NphGpuPose *pose_b, const float *speculative, uint32_t count,
                                               NphGpuManifold *out, uint32_t *bad_pairs, void *stream)
{
    if (count == 0) {
        return NPH_GPU_OK;
    }
    if (a == nullptr || pose_a == nullptr || b == nullptr || pose_b == nullptr || speculative == nullptr ||
        out == nullptr) {
        return NPH_GPU_INVALID_ARGUMENT;
    }
    k_collide<<<(count + 255u) / 256u, 256, 0, (cudaStream_t)stream>>>(a, pose_a, b, pose_b, speculative, count,
                                                                     out, bad_pairs);
    return cudaGetLastError() == cudaSuccess ? NPH_GPU_OK : NPH_GPU_DEVICE_LOST;
}

} // extern "C"

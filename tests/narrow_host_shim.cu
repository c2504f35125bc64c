// The device narrow phase's pair code (nepheline_b200/csrc/collide.cuh, __host__ __device__)
// compiled for the host with the device's floating-point contract (no contraction, correctly
// rounded division and square root), for the CPU tests: the same operations in the same order
// give the same bits as on the device, so the reference can check the code without a GPU.
#include "collide.cuh"

extern "C" void nph_host_collide(const NphGpuShape *a, const NphGpuPose *pa, const NphGpuShape *b,
                                 const NphGpuPose *pb, const float *spec, unsigned n, NphGpuManifold *out)
{
    for (unsigned i = 0; i < n; ++i) {
        NphGpuManifold m;
        for (unsigned k = 0; k < NPH_GPU_MAX_POINTS; ++k) {
            m.points[k] = NphGpuManifoldPoint{{0.0f, 0.0f, 0.0f}, 0.0f, 0u};
        }
        nph_nc::collide(a[i], pa[i], b[i], pb[i], spec[i], m);
        out[i] = m;
    }
}

// SPDX-License-Identifier: Apache-2.0
//
// Internal links between the library's translation units (not part of the C ABI): a batch
// packed as one world hands its records to a single-world solver on the device.
#pragma once

#include <cuda_runtime.h>

#include "nepheline_b200.h"

struct NphSolverRecords {
    NphGpuBody *bodies;
    NphGpuBody *fixed;
    NphGpuContact *contacts;
    NphGpuJoint *joints;
};

// Sizes the solver for a world of `shape`'s counts and colour tables (its record pointers are
// not read), marks it uploaded, and gives its device record arrays for the caller to fill on
// the solver's stream before the next step. `driven`: the view's motor-driven joints;
// `row_joints`: its slider, 6-DOF and distance joints.
NphGpuResult nph_solver_bind_device(NphGpuSolver *s, const NphGpuWorldView *shape, uint32_t driven,
                                    uint32_t row_joints, NphSolverRecords *out);
// The device record arrays of the bound world.
NphGpuResult nph_solver_records(NphGpuSolver *s, NphSolverRecords *out);
// The prepare kernels' error word as a result code (NPH_GPU_INVALID_ARGUMENT on a bad record).
NphGpuResult nph_solver_check(NphGpuSolver *s);
// hit_events over `m` device-resident contact records on stream `st` (nph_gpu_world_hit_events'
// scan): the first min(total, capacity) events to the host array `events`, in record order, with
// `contact` the record's index and `world` 0; the total to `*count`.
NphGpuResult nph_hits_scan(const NphGpuContact *contacts, uint32_t m, float threshold, cudaStream_t st,
                           NphGpuHitEvent *events, uint32_t capacity, uint32_t *count);
// The CUDA device a solver was created on.
int nph_solver_device(const NphGpuSolver *s);

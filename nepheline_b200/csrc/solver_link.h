// SPDX-License-Identifier: Apache-2.0
//
// Internal links between the library's translation units (not part of the C ABI): a batch
// packed as one world hands its records to a single-world solver on the device.
#pragma once

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

// The reference engine's world step with the device solver as its solver stage, through the
// binding (nepheline_b200/binding/phys_solve_dispatch.c) linked into the engine with world.c
// compiled as -Dphys_solve=phys_solve_dispatch (oracle/Makefile, target `binding`).
//
// Builds the reference build's determinism scene through the engine's public API: a 20-row
// box pyramid (row r holds 20 - r unit boxes at x = (j - (n - 1) / 2) 1.05, y = 0.5 + r,
// benchmarks/physics/bench_physics.c:1233-1252) on a static ground slab, sleep off, dt 1/60,
// 4 substeps; steps it with nph_physics_world_step and prints the world hash
// (nph_physics_world_hash) and the step's result code.
//
//   binding_world_step cpu  STEPS   the engine's own stage (no device solver attached)
//   binding_world_step gpu  STEPS   the device solver attached
//   binding_world_step xpbd STEPS   the device solver attached to an XPBD world (refused)
#include <nepheline/core/alloc.h>
#include <nepheline/physics/body.h>
#include <nepheline/physics/shape.h>
#include <nepheline/physics/world.h>

#include "nepheline_b200.h"

#include <inttypes.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void nph_gpu_binding_attach(NphGpuSolver *solver);
void nph_gpu_binding_release(void);

static int add_box(NphPhysicsWorld *w, NphPhysicsBodyType type, double x, double y, double z, float hx,
                   float hy, float hz)
{
    NphPhysicsBodyDesc bd = nph_physics_body_desc_default();
    bd.type = type;
    bd.position = nph_dvec3(x, y, z);
    bd.gyroscopic = 1;
    bd.enable_sleep = 1;
    NphPhysicsBody b;
    if (nph_physics_body_create(w, &bd, &b) != NPH_RESULT_OK) {
        return 1;
    }
    NphPhysicsShapeDesc sd = nph_physics_shape_desc_default(nph_physics_geometry_box(nph_vec3(hx, hy, hz)));
    sd.density = 1000.0F;
    sd.friction = 0.6F;
    sd.restitution = 0.0F;
    NphPhysicsShape s;
    return nph_physics_shape_create(w, b, &sd, &s) != NPH_RESULT_OK;
}

int main(int argc, char **argv)
{
    const char *mode = argc > 1 ? argv[1] : "cpu";
    const int steps = argc > 2 ? atoi(argv[2]) : 600;
    NphPhysicsWorldDesc d = nph_physics_world_desc_default();
    d.alloc = nph_allocator_system();
    d.enable_sleep = 0;
    d.enable_continuous = 0;
    if (strcmp(mode, "xpbd") == 0) {
        d.solver = NPH_PHYSICS_SOLVER_XPBD;
    }
    NphPhysicsWorld *w = NULL;
    if (nph_physics_world_create(&d, &w) != NPH_RESULT_OK) {
        return 2;
    }
    int bad = add_box(w, NPH_PHYSICS_BODY_STATIC, 0.0, -1.0, 0.0, 50.0F, 1.0F, 50.0F);
    for (int row = 0; row < 20; ++row) {
        const int n = 20 - row;
        for (int j = 0; j < n; ++j) {
            bad |= add_box(w, NPH_PHYSICS_BODY_DYNAMIC, ((double)j - (double)(n - 1) / 2.0) * 1.05,
                           0.5 + (double)row, 0.0, 0.5F, 0.5F, 0.5F);
        }
    }
    if (bad) {
        return 3;
    }
    NphGpuSolver *solver = NULL;
    if (strcmp(mode, "cpu") != 0) {
        NphGpuSolverDesc sd;
        memset(&sd, 0, sizeof sd);
        sd.device = 0;
        sd.use_graph = 1;
        if (nph_gpu_solver_create(&sd, &solver) != NPH_GPU_OK) {
            return 4;
        }
        nph_gpu_binding_attach(solver);
    }
    NphResult r = NPH_RESULT_OK;
    int done = 0;
    for (; done < steps && r == NPH_RESULT_OK; ++done) {
        r = nph_physics_world_step(w, 1.0F / 60.0F, NULL);
    }
    printf("mode %s steps %d result %d hash %016" PRIx64 "\n", mode, done, (int)r, nph_physics_world_hash(w));
    nph_gpu_binding_attach(NULL);
    nph_gpu_binding_release();
    if (solver != NULL) {
        nph_gpu_solver_destroy(solver);
    }
    nph_physics_world_destroy(w);
    return 0;
}

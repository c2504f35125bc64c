/* SPDX-License-Identifier: Apache-2.0
 *
 * nepheline_b200: the physics world step's solver stage (the graph-coloured
 * soft-step contact and joint solver) on one NVIDIA B200, behind a plain C ABI.
 *
 * The entry points replace the reference engine's
 *
 *     NphResult phys_solve(NphPhysicsWorld *w, f32 dt, NphJobSystem *js);
 *
 * (engine/physics/src/world_internal.h:791, defined at engine/physics/src/solver.c:961,
 * called once per step from nph_physics_world_step at engine/physics/src/world.c:346).
 * The reference passes its whole world; this ABI passes the part of it the solver
 * stage reads and writes, as flat arrays of plain records (the "world view"):
 *
 *   - the awake bodies, in the world's awake-list order (world_internal.h:600), which is
 *     the solver-body order of solver.c:967-973;
 *   - the bodies a constraint names that have no solver slot (static bodies, sleeping
 *     kinematic ones), read-only;
 *   - the touching contacts of the constraint graph, in colour order (colours 0..23, then
 *     the overflow: the order build_groups lays out, solver.c:810-843), each colour's
 *     contacts in its list order (world_internal.h:363-367);
 *   - the graph's joints, in the same colour order (build_step_joints, solver.c:793-806).
 *
 * Every record is updated in place with what phys_solve writes back into the world:
 * body velocities, rotation, centre, origin, sleep time, cleared force and torque
 * (finalize_body, solver.c:304-349); contact points' impulses, approach speeds and the
 * HIT flag (store_group, solver.c:475-499); joints' accumulated impulses.
 *
 * Result codes have the values of the reference's NphResult (engine/core/include/
 * nepheline/core/result.h:16-36), so a caller can return them as they are.
 *
 * Threading: one thread owns a solver object. Calls are synchronous (they return after
 * the device-to-host copy), as phys_solve returns after its stages, except the
 * *_async device-resident calls, which enqueue on the solver's stream.
 */
#ifndef NEPHELINE_B200_H
#define NEPHELINE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define NPH_GPU_API __attribute__((visibility("default")))
#else
#define NPH_GPU_API
#endif

/* ------------------------------------------------------------------------------------
 * Constants (the reference's values)
 * ---------------------------------------------------------------------------------- */

#define NPH_GPU_NULL 0xFFFFFFFFu
#define NPH_GPU_MAX_POINTS 4u        /* NPH_PHYSICS_MANIFOLD_MAX_POINTS, collide.h:64 */
#define NPH_GPU_COLORS 24u           /* PHYS_GRAPH_COLORS, world_internal.h:359 */
#define NPH_GPU_DYNAMIC_COLORS 20u   /* PHYS_GRAPH_DYNAMIC_COLORS, world_internal.h:360 */
#define NPH_GPU_OVERFLOW 24u         /* PHYS_GRAPH_OVERFLOW, world_internal.h:361 */
#define NPH_GPU_COLOR_SLOTS 25u      /* colours 0..23 and the overflow */

/* Result codes: the values of NphResult (core/result.h:16-36). */
typedef int32_t NphGpuResult;
#define NPH_GPU_OK 0
#define NPH_GPU_OUT_OF_MEMORY 1
#define NPH_GPU_INVALID_ARGUMENT 2
#define NPH_GPU_TOO_LARGE 7 /* NPH_RESULT_OVERFLOW: beyond a fixed capacity */
#define NPH_GPU_UNSUPPORTED 8
#define NPH_GPU_DEVICE_LOST 17
#define NPH_GPU_INVALID_STATE 18
#define NPH_GPU_UNKNOWN 19

/* Body types (NphPhysicsBodyType, body.h). */
#define NPH_GPU_BODY_STATIC 0u
#define NPH_GPU_BODY_KINEMATIC 1u
#define NPH_GPU_BODY_DYNAMIC 2u

/* Body flag bits the solver stage reads (PHYS_BODY_*, world_internal.h:59-69). */
#define NPH_GPU_BODY_ENABLE_SLEEP (1u << 1)
#define NPH_GPU_BODY_GYROSCOPIC (1u << 2)
#define NPH_GPU_BODY_BULLET (1u << 5)

/* Lock bits (NPH_PHYSICS_LOCK_*, body.h). */
#define NPH_GPU_LOCK_LINEAR_X (1u << 0)
#define NPH_GPU_LOCK_LINEAR_Y (1u << 1)
#define NPH_GPU_LOCK_LINEAR_Z (1u << 2)
#define NPH_GPU_LOCK_ANGULAR_X (1u << 3)
#define NPH_GPU_LOCK_ANGULAR_Y (1u << 4)
#define NPH_GPU_LOCK_ANGULAR_Z (1u << 5)

/* Contact flag bits the solver stage reads and writes (PHYS_CONTACT_*,
 * world_internal.h:207-213): HIT in and out; HIT_EVENTS (either shape reports hits) read by
 * nph_gpu_world_hit_events; the solver keeps every other bit as it came. */
#define NPH_GPU_CONTACT_HIT_EVENTS (1u << 2)
#define NPH_GPU_CONTACT_HIT (1u << 4)

/* Constraint bits of nph_gpu_graph_color. */
#define NPH_GPU_CONSTRAINT_A_DYNAMIC 1u
#define NPH_GPU_CONSTRAINT_B_DYNAMIC 2u
#define NPH_GPU_CONSTRAINT_JOINT 4u

/* Joint types (NphPhysicsJointType, joint.h:60-68): the device solver runs all six. */
#define NPH_GPU_JOINT_BALL 0u
#define NPH_GPU_JOINT_HINGE 1u
#define NPH_GPU_JOINT_FIXED 2u
#define NPH_GPU_JOINT_SLIDER 3u
#define NPH_GPU_JOINT_DISTANCE 4u
#define NPH_GPU_JOINT_D6 5u

/* How a 6-DOF joint's axis moves (NphPhysicsAxisMotion, joint.h:144-148), and its axes in A's
 * frame: translation along X, Y, Z, then twist about X and swing about Y and Z. */
#define NPH_GPU_AXIS_LOCKED 0u
#define NPH_GPU_AXIS_LIMITED 1u
#define NPH_GPU_AXIS_FREE 2u
#define NPH_GPU_D6_AXES 6u

/* A slider's, 6-DOF joint's or distance joint's rows per axis (PHYS_ROW_*,
 * world_internal.h:273-278): the lock or lower limit, the upper limit, the motor, the spring. */
#define NPH_GPU_ROW_LOCK 0u
#define NPH_GPU_ROW_UPPER 1u
#define NPH_GPU_ROW_MOTOR 2u
#define NPH_GPU_ROW_SPRING 3u

/* Joint flags, in and out: the blocks a slider or 6-DOF joint solved its rows as last step
 * (PHYS_JOINT_BLOCK_*, joint_solver.c:103-112). A change of block zeroes the block's
 * accumulated impulse, whose meaning changes with it. */
#define NPH_GPU_JOINT_BLOCK_ROTATION (1u << 11)
#define NPH_GPU_JOINT_BLOCK_SWING (1u << 12)
#define NPH_GPU_JOINT_BLOCK_POINT (1u << 13)

/* Solvers (NphPhysicsSolver, world.h:86-101). The device solver runs the soft step and TGS;
 * XPBD is refused with NPH_GPU_UNSUPPORTED. The learned warm start is the soft step's: a
 * TGS step does not apply it, and its feature and convergence calls refuse TGS. */
#define NPH_GPU_SOLVER_SOFT_STEP 0u
#define NPH_GPU_SOLVER_TGS 1u

/* ------------------------------------------------------------------------------------
 * Records
 * ---------------------------------------------------------------------------------- */

/* The world settings the solver stage reads: NphPhysicsWorldDesc (world.h:104-143),
 * defaults at world.c:85-104. */
typedef struct NphGpuWorldParams {
    float gravity[3];
    uint32_t solver; /* NPH_GPU_SOLVER_SOFT_STEP or NPH_GPU_SOLVER_TGS */
    uint32_t substeps;
    float contact_hertz; /* 0: an eighth of the substep rate (solver.c:996-997) */
    float contact_damping_ratio;
    float contact_push_max_velocity;
    float restitution_threshold;
    float max_linear_speed;
    float joint_hertz; /* 0: a quarter of the substep rate (solver.c:998) */
    float joint_damping_ratio;
    uint32_t enable_continuous; /* must be 0: continuous collision stays on the host */
} NphGpuWorldParams;

/* A body, as PhysBody (world_internal.h:71-107) holds what the solver stage reads.
 * Matrices are column-major, as NphMat3 (m[col * 3 + row]). Quaternions are x, y, z, w. */
typedef struct NphGpuBody {
    double center[3];           /* centre of mass, world; in and out */
    double origin[3];           /* the body frame's origin; out */
    float rotation[4];          /* in and out */
    float local_center[3];      /* centre of mass in the body frame */
    float linear_velocity[3];   /* in and out */
    float angular_velocity[3];  /* in and out */
    float force[3];             /* in; zero after the step */
    float torque[3];            /* in; zero after the step */
    float inertia[9];           /* about the centre of mass, body axes */
    float inv_inertia[9];
    float inv_mass;
    float linear_damping;
    float angular_damping;
    float gravity_scale;
    float sleep_threshold;
    float sleep_time;           /* in and out */
    float max_extent;
    uint32_t type;              /* NPH_GPU_BODY_* */
    uint32_t flags;             /* NPH_GPU_BODY_* bits */
    uint32_t locks;             /* NPH_GPU_LOCK_* bits */
    uint32_t pad;
} NphGpuBody;

/* A manifold point, as PhysContactPoint (world_internal.h:196-205). */
typedef struct NphGpuContactPoint {
    float anchor_a[3];          /* from A's centre of mass, world axes */
    float anchor_b[3];          /* from B's */
    float separation;
    float normal_impulse;       /* in (warm start) and out */
    float max_normal_impulse;   /* out: the largest this step */
    float tangent_impulse[3];   /* in and out: world vector */
    float relative_velocity;    /* out: normal approach speed at the step's start */
    uint32_t id;                /* the narrow phase's feature id: passed through */
} NphGpuContactPoint;

/* A touching contact (one manifold), as PhysContact (world_internal.h:229-253).
 * `body_a` and `body_b` index the view's bodies: below `body_count` an awake body,
 * from `body_count` on the fixed body `index - body_count`. */
typedef struct NphGpuContact {
    uint32_t body_a;
    uint32_t body_b;
    uint32_t flags;             /* NPH_GPU_CONTACT_HIT: in and out; NPH_GPU_CONTACT_HIT_EVENTS */
    uint32_t point_count;       /* 1..4 */
    float normal[3];            /* from A to B */
    float friction;
    float restitution;
    uint32_t pad[3];
    NphGpuContactPoint points[NPH_GPU_MAX_POINTS];
} NphGpuContact;

/* Ball joint settings (NphPhysicsBallJoint, joint.h). */
typedef struct NphGpuBallJoint {
    uint32_t enable_swing_limit;
    float swing_y;
    float swing_z;
    uint32_t enable_twist_limit;
    float twist_lower;
    float twist_upper;
    float friction_torque;
    float pad[3];
} NphGpuBallJoint;

/* Hinge joint settings (NphPhysicsHingeJoint, joint.h). */
typedef struct NphGpuHingeJoint {
    uint32_t enable_limit;
    float lower;
    float upper;
    uint32_t enable_motor;
    float motor_speed;
    float max_motor_torque;
    uint32_t enable_spring;
    float spring_hertz;
    float spring_damping_ratio;
    float spring_target;
} NphGpuHingeJoint;

/* Slider joint settings (NphPhysicsSliderJoint, joint.h:107-121): along A's X axis. */
typedef struct NphGpuSliderJoint {
    uint32_t enable_limit;
    float lower;
    float upper;
    uint32_t enable_motor;
    float motor_speed;
    float max_motor_force;
    uint32_t enable_spring;
    float spring_hertz;
    float spring_damping_ratio;
    float spring_target;
} NphGpuSliderJoint;

/* Distance joint settings (NphPhysicsDistanceJoint, joint.h:128-140). */
typedef struct NphGpuDistanceJoint {
    float length;
    uint32_t enable_limit;
    float min_length;
    float max_length;
    uint32_t enable_spring;
    float spring_hertz;
    float spring_damping_ratio;
    uint32_t enable_motor;
    float motor_speed;
    float max_motor_force;
} NphGpuDistanceJoint;

/* One axis of a 6-DOF joint (NphPhysicsD6Axis, joint.h:152-163). */
typedef struct NphGpuD6Axis {
    uint32_t motion; /* NPH_GPU_AXIS_* */
    float lower;
    float upper;
    uint32_t enable_motor;
    float motor_speed;
    float max_motor_force;
    uint32_t enable_spring;
    float spring_hertz;
    float spring_damping_ratio;
    float spring_target;
} NphGpuD6Axis;

/* A joint of the constraint graph, as PhysJoint (world_internal.h:280-330): its frames
 * in the bodies' frames, its settings, and its accumulated impulses (in and out). */
typedef struct NphGpuJoint {
    uint32_t type;              /* NPH_GPU_JOINT_* */
    uint32_t body_a;            /* as NphGpuContact */
    uint32_t body_b;
    uint32_t flags;             /* NPH_GPU_JOINT_BLOCK_*: in and out */
    float frame_a_position[3];  /* in body A's frame (its origin) */
    float frame_a_rotation[4];
    float frame_b_position[3];
    float frame_b_rotation[4];
    union {
        NphGpuBallJoint ball;
        NphGpuHingeJoint hinge;
        NphGpuSliderJoint slider;
        NphGpuDistanceJoint distance;
        NphGpuD6Axis d6[NPH_GPU_D6_AXES];
    } u;
    float linear_impulse[3];    /* the anchors as one block, world */
    float angular_impulse[3];   /* the hinge's or swing block's two rows, or a world vector */
    float friction_impulse[3];
    float lower_impulse;
    float upper_impulse;
    float swing_impulse;
    float motor_impulse;
    float spring_impulse;
    float axis_impulse[NPH_GPU_D6_AXES][4]; /* NPH_GPU_ROW_* per axis (distance: axis 0) */
} NphGpuJoint;

/* The solver stage's part of a world. The arrays are the caller's; a solve updates
 * `bodies`, `contacts` and `joints` in place. */
typedef struct NphGpuWorldView {
    NphGpuBody *bodies;                 /* awake bodies, awake-list order */
    uint32_t body_count;
    uint32_t fixed_count;
    const NphGpuBody *fixed_bodies;     /* bodies without a solver slot, read only */
    NphGpuContact *contacts;            /* colour order */
    uint32_t contact_count;
    uint32_t joint_count;
    NphGpuJoint *joints;                /* colour order */
    uint32_t contact_color_counts[NPH_GPU_COLOR_SLOTS]; /* colours 0..23, then the overflow */
    uint32_t joint_color_counts[NPH_GPU_COLOR_SLOTS];
} NphGpuWorldView;

/* The packed records of nph_gpu_phys_solve_packed: the fields the solver stage reads of a
 * body and of a contact (NphGpuBody and NphGpuContact without what the stage only writes or
 * never reads), and the fields it writes of a body, a contact and a joint. */
typedef struct NphGpuBodyInput {
    double center[3];
    float rotation[4];
    float local_center[3];
    float linear_velocity[3];
    float angular_velocity[3];
    float force[3];
    float torque[3];
    float inertia[9];
    float inv_inertia[9];
    float inv_mass;
    float linear_damping;
    float angular_damping;
    float gravity_scale;
    float sleep_threshold;
    float sleep_time;
    float max_extent;
    uint32_t type;
    uint32_t flags;
    uint32_t locks;
    uint32_t pad;
} NphGpuBodyInput;

typedef struct NphGpuContactPointInput {
    float anchor_a[3];
    float anchor_b[3];
    float separation;
    float normal_impulse;      /* the warm start */
    float tangent_impulse[3];  /* the warm start: world vector */
    uint32_t id;               /* kept on the device for a later nph_gpu_world_update_contacts */
} NphGpuContactPointInput;

typedef struct NphGpuContactInput {
    uint32_t body_a;
    uint32_t body_b;
    uint32_t flags;
    uint32_t point_count;
    float normal[3];
    float friction;
    float restitution;
    NphGpuContactPointInput points[NPH_GPU_MAX_POINTS];
} NphGpuContactInput;

/* After the step: force and torque are zero, as phys_solve leaves them (the caller clears its
 * own; they are not sent back). */
typedef struct NphGpuBodyOutput {
    double center[3];
    double origin[3];
    float rotation[4];
    float linear_velocity[3];
    float angular_velocity[3];
    float sleep_time;
    uint32_t pad;
} NphGpuBodyOutput;

typedef struct NphGpuContactPointOutput {
    float normal_impulse;
    float max_normal_impulse;
    float tangent_impulse[3];
    float relative_velocity;
} NphGpuContactPointOutput;

typedef struct NphGpuContactOutput {
    uint32_t flags; /* the input's flags with NPH_GPU_CONTACT_HIT as the step leaves it */
    NphGpuContactPointOutput points[NPH_GPU_MAX_POINTS]; /* the first point_count are live */
} NphGpuContactOutput;

typedef struct NphGpuJointOutput {
    float linear_impulse[3];
    float angular_impulse[3];
    float friction_impulse[3];
    float lower_impulse;
    float upper_impulse;
    float swing_impulse;
    float motor_impulse;
    float spring_impulse;
    float axis_impulse[NPH_GPU_D6_AXES][4];
    uint32_t flags; /* NPH_GPU_JOINT_BLOCK_* as the step leaves them */
} NphGpuJointOutput;

typedef struct NphGpuPackedInput {
    const NphGpuBodyInput *bodies;      /* awake bodies, awake-list order */
    uint32_t body_count;
    uint32_t fixed_count;
    const NphGpuBody *fixed_bodies;     /* bodies without a solver slot, read only */
    const NphGpuContactInput *contacts; /* colour order */
    uint32_t contact_count;
    uint32_t joint_count;
    const NphGpuJoint *joints;          /* colour order, whole records (settings and impulses) */
    uint32_t contact_color_counts[NPH_GPU_COLOR_SLOTS];
    uint32_t joint_color_counts[NPH_GPU_COLOR_SLOTS];
} NphGpuPackedInput;

typedef struct NphGpuPackedOutput {
    NphGpuBodyOutput *bodies;       /* body_count records */
    NphGpuContactOutput *contacts;  /* contact_count records */
    NphGpuJointOutput *joints;      /* joint_count records */
} NphGpuPackedOutput;

/* What a step reports (a subset of NphPhysicsStats, world.h:250-278). */
typedef struct NphGpuStepStats {
    uint32_t colors_used;           /* colours holding contacts or joints */
    uint32_t overflow_contacts;
    uint32_t overflow_joints;
    uint32_t launches;              /* device kernels launched per step */
    float device_ms;                /* device time of the last step (CUDA events) */
    float upload_ms;                /* host->device of the last phys_solve call */
    float download_ms;              /* device->host of the last phys_solve call */
    uint32_t error_word;            /* device error flags of the last step (0: none) */
} NphGpuStepStats;

/* ------------------------------------------------------------------------------------
 * The solver object
 * ---------------------------------------------------------------------------------- */

typedef struct NphGpuSolver NphGpuSolver;

typedef struct NphGpuSolverDesc {
    int32_t device;            /* CUDA ordinal */
    void *stream;              /* a cudaStream_t to launch on, or NULL for the solver's own */
    uint32_t use_graph;        /* 1: replay each step's launches as one CUDA graph */
    uint32_t body_capacity;    /* initial device capacities (grown between steps) */
    uint32_t contact_capacity;
    uint32_t joint_capacity;
} NphGpuSolverDesc;

/* Creates a solver on `desc->device`. Device buffers are sized to the capacities and grow
 * only between steps, so a steady state allocates nothing (as the world's arrays,
 * world.h:37-43). */
NPH_GPU_API NphGpuResult nph_gpu_solver_create(const NphGpuSolverDesc *desc, NphGpuSolver **out);
NPH_GPU_API void nph_gpu_solver_destroy(NphGpuSolver *solver);

/* The drop-in for phys_solve (solver.c:961-1105): uploads the view, runs the stage list
 * (prepare bodies, prepare contacts and joints; per substep integrate velocities, warm
 * start, solve, integrate positions, relax, each constraint pass colour by colour with the
 * overflow first; then restitution, store, finalize) and writes the results back into the
 * view's arrays. Returns NPH_GPU_INVALID_ARGUMENT for a malformed view (an index out of
 * range, a point count outside 1..4, colour counts that do not add up, an axis motion other
 * than NPH_GPU_AXIS_*, a body record with a value the stage reads that is not finite: NaN or
 * infinite), NPH_GPU_UNSUPPORTED for a setting the device solver does not run
 * (XPBD, continuous collision, an unknown joint type), NPH_GPU_OUT_OF_MEMORY when the device buffers
 * cannot grow (the view is then untouched: the step did not happen), and
 * NPH_GPU_DEVICE_LOST when a device wait gave up or the device reported an error. */
NPH_GPU_API NphGpuResult nph_gpu_phys_solve(NphGpuSolver *solver, const NphGpuWorldParams *params,
                                            float dt, NphGpuWorldView *view);

/* nph_gpu_phys_solve on packed records: the host arrays hold only the fields the stage reads
 * (in) and writes (out), so each step moves about 1.5 GB over PCIe for the 1,048,576-body
 * lattice instead of 2.5 GB of whole records. The records are expanded and packed on the
 * device; the results equal nph_gpu_phys_solve's field for field. The same refusals, with the
 * outputs untouched. A caller that keeps its world in other records (the engine's own) gathers
 * the inputs from them and scatters the outputs back, as it would for the whole records. */
NPH_GPU_API NphGpuResult nph_gpu_phys_solve_packed(NphGpuSolver *solver,
                                                   const NphGpuWorldParams *params, float dt,
                                                   const NphGpuPackedInput *in,
                                                   NphGpuPackedOutput *out);

/* Device-resident stepping: the view's records are uploaded once, stepped `steps` times on
 * the device (each step the whole solver stage over the resident records: the manifolds'
 * geometry stays as uploaded, the bodies and impulses carry over), and read back when the
 * caller asks. upload/download are synchronous; step_async enqueues on the solver's stream. */
NPH_GPU_API NphGpuResult nph_gpu_world_upload(NphGpuSolver *solver, const NphGpuWorldView *view);
NPH_GPU_API NphGpuResult nph_gpu_world_step_async(NphGpuSolver *solver,
                                                  const NphGpuWorldParams *params, float dt,
                                                  uint32_t steps);
NPH_GPU_API NphGpuResult nph_gpu_world_download(NphGpuSolver *solver, NphGpuWorldView *view);
NPH_GPU_API NphGpuResult nph_gpu_solver_synchronize(NphGpuSolver *solver);
NPH_GPU_API NphGpuResult nph_gpu_solver_stats(const NphGpuSolver *solver, NphGpuStepStats *out);
/* The stream the solver launches on (a cudaStream_t). */
NPH_GPU_API void *nph_gpu_solver_stream(const NphGpuSolver *solver);

/* A budget for the solver's record and row arrays, in bytes (0, the default: none). A call
 * whose view would grow them beyond it returns NPH_GPU_OUT_OF_MEMORY before any array or the
 * view is touched, as an allocation failure does (world.h:163-165: the step did not happen;
 * the reference's failing-allocator test, test_sensor.c:342-392, fails its steps this way).
 * An engine that gives the solver a fixed share of device memory sets it. */
NPH_GPU_API NphGpuResult nph_gpu_solver_set_memory_limit(NphGpuSolver *solver, uint64_t bytes);
/* The bytes the solver's record and row arrays hold now (the figure the budget limits). */
NPH_GPU_API uint64_t nph_gpu_solver_memory(const NphGpuSolver *solver);
/* Failure injection for the dependency-driven passes (a test hook; 0, the default: off). Every
 * constraint then waits for `extra` more finished constraints on its bodies than will come, so
 * its waits give up after about a second: the call returns NPH_GPU_DEVICE_LOST with nothing
 * written back, and the solver (and its device context) takes the next call as usual. */
NPH_GPU_API NphGpuResult nph_gpu_solver_set_wait_injection(NphGpuSolver *solver, uint32_t extra);

/* One kind of kernel in a profiled step. */
typedef struct NphGpuKernelTime {
    char name[32];
    uint32_t launches;
    uint32_t pad;
    uint64_t units;              /* manifolds, joints or bodies processed over the launches */
    double total_ms;             /* summed device time of the launches (CUDA events) */
    double algorithmic_bytes;    /* the reference data model's live bytes over the launches */
} NphGpuKernelTime;

/* One step of the uploaded world with every launch issued directly and bracketed by CUDA
 * events on the solver's stream, reported per kind of kernel (at most `capacity` kinds;
 * `*count` receives how many). The step is a real step: the world advances. The
 * algorithmic bytes use the reference data model's per-unit figures (a manifold solve pass
 * 224 + 148 per point bytes, relax 212 + 148 per point, warm start 120 per point, prepare 936,
 * store 160, restitution check 40; a body's prepare 368, each integration 84, finalize 200;
 * a joint pass 330). */
NPH_GPU_API NphGpuResult nph_gpu_world_profile_step(NphGpuSolver *solver,
                                                    const NphGpuWorldParams *params, float dt,
                                                    NphGpuKernelTime *out, uint32_t capacity,
                                                    uint32_t *count);

/* The constraint passes' launch configuration (threads per block and register budget), per
 * pass kind: 0 warm start, 1 solve, 2 relax, 3 restitution; `config` below
 * nph_gpu_pass_config_count(). Results do not depend on it. */
NPH_GPU_API NphGpuResult nph_gpu_solver_set_pass_config(NphGpuSolver *solver, uint32_t pass,
                                                        uint32_t config);
NPH_GPU_API uint32_t nph_gpu_pass_config_count(void);

/* The autotuner: times every pass configuration on the uploaded world (`rounds` timed steps
 * each, after one untimed step, launch by launch) and keeps the fastest per pass kind, written
 * to chosen[4] when not NULL. With a step graph, the solve and relax passes' best
 * dependency-driven configuration is then weighed against the choice over whole graph steps
 * (rounds + 1 each), where a colour's joints run beside its contacts. Each timed step is a
 * real step: the world advances. */
NPH_GPU_API NphGpuResult nph_gpu_solver_autotune(NphGpuSolver *solver,
                                                 const NphGpuWorldParams *params, float dt,
                                                 uint32_t rounds, uint32_t *chosen);

/* ------------------------------------------------------------------------------------
 * Batched worlds: many independent worlds of uneven size in one persistent launch
 * ---------------------------------------------------------------------------------------
 * The reference steps one world per nph_physics_world_step; this steps a batch of worlds
 * with the same settings, each as phys_solve would, in one kernel launch per step. Worlds are
 * taken whole from queues sorted by size, one queue per team size: a team of a whole block,
 * half a block, ... down to one warp runs a world, with barriers of its own between stages
 * and colours, so one SM works on several worlds at once. A world solved in a batch gives the
 * same bits as the world solved alone by nph_gpu_phys_solve. */

typedef struct NphGpuBatch NphGpuBatch;

/* Packings of a batch. */
#define NPH_GPU_BATCH_PERSISTENT 0u /* one persistent launch a step: teams take whole worlds */
#define NPH_GPU_BATCH_MERGED 1u     /* the batch as one world: a launch per stage and colour over
                                       every world at once (each world's colour lists padded to
                                       whole eight-lane groups, so each world's results stay
                                       the same bits), replayed as a CUDA graph */

/* Shared-memory modes for a world's body velocities. */
#define NPH_GPU_BATCH_SHARED_NONE 0u  /* in global memory */
#define NPH_GPU_BATCH_SHARED_SMALL 1u /* up to 32 KiB per block */
#define NPH_GPU_BATCH_SHARED_LARGE 2u /* up to 160 KiB per block (the largest world) */

/* A batch launch configuration (results do not depend on it). */
typedef struct NphGpuBatchTuning {
    uint32_t config;            /* launch shape, below nph_gpu_batch_config_count() */
    uint32_t threads;           /* threads per block of that shape (filled in) */
    uint32_t shared_velocities; /* NPH_GPU_BATCH_SHARED_* */
    uint32_t items_per_thread;  /* a world runs on the smallest team (1, 2, 4, ... warps, up
                                   to the block) whose threads cover its largest colour at
                                   this many constraints a thread; 0: every world on a block */
    uint32_t packing;           /* NPH_GPU_BATCH_PERSISTENT or NPH_GPU_BATCH_MERGED; the fields
                                   above apply to the persistent packing */
    float ms_per_step;          /* the autotuner's time for it (filled in) */
    float persistent_ms_per_step; /* the autotuner's best persistent configuration's time */
    float merged_ms_per_step;     /* the autotuner's time for the merged packing */
} NphGpuBatchTuning;

typedef struct NphGpuBatchInfo {
    uint32_t worlds;
    uint32_t config;
    uint64_t bodies;
    uint64_t manifolds;
    uint64_t joints;
    uint32_t threads;
    uint32_t shared_velocities;
    uint32_t blocks_per_sm;
    uint32_t items_per_thread;
    uint32_t warp_worlds;  /* worlds the current configuration runs on one warp */
    uint32_t block_worlds; /* worlds it runs on a whole block */
    uint32_t packing;
    uint32_t launches_per_step; /* kernel launches a step makes (1 for the persistent packing) */
} NphGpuBatchInfo;

NPH_GPU_API NphGpuResult nph_gpu_batch_create(const NphGpuSolverDesc *desc, NphGpuBatch **out);
NPH_GPU_API void nph_gpu_batch_destroy(NphGpuBatch *batch);
NPH_GPU_API void *nph_gpu_batch_stream(const NphGpuBatch *batch);
/* Uploads `count` world views (device arrays grown to the batch when needed). Refuses as
 * nph_gpu_phys_solve does. Worlds whose records lie back to back in host memory (consecutive
 * slices of one array) are copied with one transfer per array. */
NPH_GPU_API NphGpuResult nph_gpu_batch_upload(NphGpuBatch *batch, const NphGpuWorldView *worlds,
                                              uint32_t count);
/* `steps` steps of every uploaded world, enqueued on the batch's stream (one CUDA graph launch
 * per step). */
NPH_GPU_API NphGpuResult nph_gpu_batch_step_async(NphGpuBatch *batch,
                                                  const NphGpuWorldParams *params, float dt,
                                                  uint32_t steps);
/* Writes every world's results back into its view (the same views, in the same order). */
NPH_GPU_API NphGpuResult nph_gpu_batch_download(NphGpuBatch *batch, NphGpuWorldView *worlds,
                                                uint32_t count);
/* Upload, one step, download: phys_solve for each of `count` worlds. */
NPH_GPU_API NphGpuResult nph_gpu_phys_solve_worlds(NphGpuBatch *batch,
                                                   const NphGpuWorldParams *params, float dt,
                                                   NphGpuWorldView *worlds, uint32_t count);
/* Sets the launch configuration (tuning->ms_per_step and ->threads are ignored). */
NPH_GPU_API NphGpuResult nph_gpu_batch_set_config(NphGpuBatch *batch,
                                                  const NphGpuBatchTuning *tuning);
/* Splits nph_gpu_phys_solve_worlds into `parts` (1..NPH_GPU_BATCH_MAX_PARTS; 1, the default,
 * does not split): consecutive runs of worlds of about equal record bytes, each solved by a
 * batch of its own on its own stream with this batch's launch configuration. A part's upload
 * follows the previous part's, its step and its download follow its upload, so the host link
 * carries one part's results back while later parts' records go up. Results are the same bits
 * as unsplit (the worlds are independent). Every record the device would refuse is checked on
 * the host before anything is copied, so a refused batch still has nothing written back. The
 * parts hold device arrays of their own (released by setting 1 part); the batch's own upload,
 * step and download calls do not use them. */
#define NPH_GPU_BATCH_MAX_PARTS 16u
NPH_GPU_API NphGpuResult nph_gpu_batch_set_pipeline(NphGpuBatch *batch, uint32_t parts);
/* The merged packing's pass configuration per pass kind, as nph_gpu_solver_set_pass_config
 * (the autotuner sets them too). Results do not depend on it. */
NPH_GPU_API NphGpuResult nph_gpu_batch_set_pass_config(NphGpuBatch *batch, uint32_t pass, uint32_t config);
NPH_GPU_API uint32_t nph_gpu_batch_config_count(void);
/* The batch autotuner: times every configuration on the uploaded worlds (`rounds` timed steps
 * each after an untimed one; the worlds advance) and keeps the fastest. */
NPH_GPU_API NphGpuResult nph_gpu_batch_autotune(NphGpuBatch *batch,
                                                const NphGpuWorldParams *params, float dt,
                                                uint32_t rounds, NphGpuBatchTuning *out);
NPH_GPU_API NphGpuResult nph_gpu_batch_info(const NphGpuBatch *batch, NphGpuBatchInfo *out);

/* ------------------------------------------------------------------------------------
 * The constraint graph's colouring on the device
 * ---------------------------------------------------------------------------------- */

/* Colours `count` constraints inserted in order into an empty constraint graph, as the
 * reference's phys_graph_add / phys_graph_add_joint do one at a time (graph_pick_color,
 * island.c:34-56; graph_set_bodies, island.c:58-75): a pair of dynamic bodies takes the
 * first of colours 0..19 free for both, a constraint with one dynamic body the first of
 * colours 1..23 free for it, and the rest overflow (NPH_GPU_OVERFLOW). `body_a`/`body_b`
 * are body slots below `body_slots`; `dynamic_bits` bit 0 says A is dynamic, bit 1 B, and
 * bit 2 that the constraint is a joint (joints and contacts share the colours' body sets,
 * but each colour keeps a contact list and a joint list: island.c:77-88, 106-118). Writes
 * each constraint's colour and its slot in its colour's list of its kind (the list order
 * is the insertion order). The result equals the sequential first-fit bit for bit.
 * Cost: one launch per round of the parallel fixpoint, as many rounds as the longest chain of
 * constraints each sharing a dynamic body with an earlier one (about 320 for the 1,048,576-body
 * lattice); a longer chain (a rope or stack inserted in order) is finished after
 * max(512, count / 512) rounds by the sequential rule on one warp, about 60 ns a constraint.
 * Counts at or above 2^30 and body_slots at or above 2^31 - 1 return NPH_GPU_TOO_LARGE. */
NPH_GPU_API NphGpuResult nph_gpu_graph_color(NphGpuSolver *solver, const uint32_t *body_a,
                                             const uint32_t *body_b, const uint8_t *dynamic_bits,
                                             uint32_t count, uint32_t body_slots,
                                             uint32_t *out_color, uint32_t *out_slot);

/* The same colouring without allocating anything: no counterpart in the reference. For
 * callers that may not allocate device memory while they run (an engine that reserves its
 * memory up front, a fixed per-frame budget, an allocator owned by another runtime). Its
 * scratch is one fixed device array of NPH_GPU_GRAPH_COLOR_STATIC_SCRATCH_BYTES that every
 * GPU loading this library holds until exit; inputs and outputs are the caller's host
 * arrays, as in nph_gpu_graph_color. At most NPH_GPU_GRAPH_COLOR_STATIC_MAX_CONSTRAINTS
 * constraints over NPH_GPU_GRAPH_COLOR_STATIC_MAX_BODY_SLOTS body slots: larger inputs
 * return NPH_GPU_TOO_LARGE. Runs on the current device, on `stream` (a cudaStream_t, NULL for
 * the default stream). Each call looks the array's address up in the current context (so a
 * context reset or a context the caller makes current is followed); the first call in a
 * context also loads the library's device code and should come before any stream capture.
 * All calls share the one array and it keeps the last call's contents (what must start at
 * zero is cleared by each call): calls that overlap on the GPU (other threads, other streams
 * of the device) race and must be serialised by the caller. The result equals
 * nph_gpu_graph_color's. */
#define NPH_GPU_GRAPH_COLOR_STATIC_MAX_CONSTRAINTS 131072u
#define NPH_GPU_GRAPH_COLOR_STATIC_MAX_BODY_SLOTS 131072u
#define NPH_GPU_GRAPH_COLOR_STATIC_SCRATCH_BYTES (8u << 20)
NPH_GPU_API NphGpuResult nph_gpu_graph_color_static(void *stream, const uint32_t *body_a,
                                                    const uint32_t *body_b,
                                                    const uint8_t *dynamic_bits, uint32_t count,
                                                    uint32_t body_slots, uint32_t *out_color,
                                                    uint32_t *out_slot);

/* ------------------------------------------------------------------------------------
 * The narrow phase's closed-form pairs on the device
 * ---------------------------------------------------------------------------------- */

/* Convex shapes (NphPhysicsShapeType, geometry.h:38-44, in its order). */
#define NPH_GPU_SHAPE_SPHERE 0u  /* dims[0]: radius */
#define NPH_GPU_SHAPE_CAPSULE 1u /* dims[0]: half the core's length (along y), dims[1]: radius */
#define NPH_GPU_SHAPE_BOX 2u     /* dims: half extents */

typedef struct NphGpuShape {
    uint32_t type;
    float dims[3];
} NphGpuShape;

/* A shape's pose (NphPhysicsPose, types.h:65-68). */
typedef struct NphGpuPose {
    float position[3];
    float rotation[4]; /* x, y, z, w */
} NphGpuPose;

/* NphPhysicsManifold (collide.h:66-79). */
typedef struct NphGpuManifoldPoint {
    float point[3];   /* midway between the surfaces */
    float separation; /* along the normal; negative when overlapping */
    uint32_t id;      /* the features that made the point */
} NphGpuManifoldPoint;

typedef struct NphGpuManifold {
    float normal[3]; /* from shape A towards shape B */
    uint32_t point_count;
    NphGpuManifoldPoint points[NPH_GPU_MAX_POINTS];
} NphGpuManifold;

/* nph_physics_collide (collide.c:524-535) for `count` pairs (host arrays), on the device, for
 * every pair of spheres, capsules and boxes, in either order: sphere-sphere, capsule-sphere,
 * capsule-capsule and box-sphere (collide.c:281-458), box-capsule (collide_hull.c:207-378) and
 * box-box (collide_hull.c:1085-1266: the oriented-box axis test, face clipping with the
 * reduction to four points, edge pairs, GJK for shapes apart); each manifold is the same bits as
 * the reference's. A pair of an unknown type gets the cleared manifold and makes the call
 * return NPH_GPU_UNSUPPORTED (nph_gpu_collide, below). */
/* The same on DEVICE arrays, enqueued on `stream` (a cudaStream_t; NULL: the default stream)
 * without allocating or waiting: the caller owns the arrays and synchronises the stream. With a
 * device `workspace` of at least nph_gpu_collide_workspace_bytes(count) bytes (4-byte aligned)
 * the pairs are first sorted by kind on the device, so that each warp runs one pair kind's code
 * (the results are the same; NULL: unsorted, one launch). A pair with an unknown type gets the
 * cleared manifold (+y, no points) and adds one to the device counter `bad_pairs` when it is
 * not NULL. At most 2^28 - 1 pairs a call. */
NPH_GPU_API uint64_t nph_gpu_collide_workspace_bytes(uint32_t count);
NPH_GPU_API NphGpuResult nph_gpu_collide_async(const NphGpuShape *a, const NphGpuPose *pose_a,
                                               const NphGpuShape *b, const NphGpuPose *pose_b,
                                               const float *speculative, uint32_t count,
                                               NphGpuManifold *out, uint32_t *bad_pairs,
                                               void *workspace, uint64_t workspace_bytes,
                                               void *stream);

/* The same on host arrays, synchronous, on the current device. A pair of an unknown type gets
 * the cleared manifold and the call returns NPH_GPU_UNSUPPORTED, with every other pair's
 * manifold written (the types are checked on the device). The pairs go in chunks of about a sixteenth of them
 * (at least 65,536) through three streams: a chunk's upload follows the previous chunk's, its
 * collision and the copy of its manifolds back follow its upload, so results come back while
 * later chunks go up (page-locked host arrays let the copies overlap). The chunks' device arrays
 * are kept between calls, one set per device; calls are serialised by a lock. */
NPH_GPU_API NphGpuResult nph_gpu_collide(const NphGpuShape *a, const NphGpuPose *pose_a,
                                         const NphGpuShape *b, const NphGpuPose *pose_b,
                                         const float *speculative, uint32_t count,
                                         NphGpuManifold *out);
/* Frees the device arrays and streams nph_gpu_collide keeps between calls, on every device
 * (the next call makes them again). */
NPH_GPU_API void nph_gpu_collide_release(void);

/* The broad phase for worlds the caller steps with the library's own stages: the pairs (a < b,
 * by index) of boxes of the same group whose axis-aligned boxes overlap (closed intervals, as
 * boxes_overlap, contact.c:286-290; the reference pairs its fattened boxes from AABB trees,
 * phys_update_pairs, contact.c:811). `lo`/`hi`: count x 3 floats; `group`: a world number per
 * box; `cell`: a grid spacing no smaller than any box's extent on any axis. The first
 * min(total, capacity) pairs in (a, b) order go to pair_a/pair_b, the total to *pair_count (a
 * caller with too small a capacity calls again). Host arrays; device arrays per call. */
NPH_GPU_API NphGpuResult nph_gpu_broad_phase(const float *lo, const float *hi, const uint32_t *group,
                                             uint32_t count, float cell, uint32_t *pair_a,
                                             uint32_t *pair_b, uint32_t capacity, uint32_t *pair_count);

/* phys_contact_update's warm start (contact.c:516-565) for `count` contacts on host arrays:
 * out[i] is fresh[i] (the narrow phase's manifold as a contact record: anchors from each body's
 * centre, separation, feature ids, impulses zero) with the pair and flags of old[i] and the
 * impulses of old[i]'s points carried over by feature id, then by place (warm_by_id,
 * warm_by_place, contact.c:332-380). A pair new this step passes an old record with its bodies,
 * flags 0 and no points. On the device; device arrays per call. */
NPH_GPU_API NphGpuResult nph_gpu_warm_start_contacts(const NphGpuContact *old, const NphGpuContact *fresh,
                                                     uint32_t count, NphGpuContact *out);

/* ------------------------------------------------------------------------------------
 * The contact update on the device
 * ---------------------------------------------------------------------------------- */

/* The next step's contacts, warm-started on the device from the records the last step
 * stored, as the reference's contact update does for pairs of convex shapes
 * (phys_contact_update, contact.c:516-565: by feature id, then by place within twice the
 * linear slop on both anchors; warm_by_id and warm_by_place, contact.c:332-380). `fresh`
 * holds this step's manifolds from the narrow phase for the uploaded contacts, in the same
 * order (normal, surface, points with anchors, separations and ids; impulses zero); each
 * takes its pair and flags from the uploaded record and, point by point, the impulses last
 * step's points carry over. Bodies and joints stay on the device: a step that keeps its
 * contact set needs this and nph_gpu_world_step_async, not a re-upload. Refuses a count
 * that differs from the uploaded one (NPH_GPU_INVALID_STATE) and point counts outside 1..4. */
NPH_GPU_API NphGpuResult nph_gpu_world_update_contacts(NphGpuSolver *solver,
                                                       const NphGpuContact *fresh, uint32_t count);

/* ------------------------------------------------------------------------------------
 * The learned warm start: no counterpart in the reference, whose contact points that are new
 * this step start at zero impulse (contact.c:547-565) and whose persisted points start at
 * their matched impulses. A small network predicts a new point's normal and two friction
 * impulses from features of its contact; the plain warm start stays for every other point.
 * ---------------------------------------------------------------------------------- */

/* The network: NPH_GPU_MLP_INPUTS -> 3 x NPH_GPU_MLP_HIDDEN (ReLU) -> NPH_GPU_MLP_OUTPUTS,
 * BF16 weights and activations on the tensor cores with FP32 accumulation, FP32 master
 * weights trained with Adam. Parameters, in order: W1 [64][16], b1 [64], W2 [64][64], b2,
 * W3 [64][64], b3, W4 [3][64], b4 [3] (weights row-major by output unit). */
#define NPH_GPU_MLP_INPUTS 16
#define NPH_GPU_MLP_HIDDEN 64
#define NPH_GPU_MLP_OUTPUTS 3
#define NPH_GPU_MLP_PARAMS 9603

typedef struct NphGpuMlp NphGpuMlp;

/* A network on `device` with seeded initial weights (uniform, scale sqrt(6 / fan_in); the
 * output layer's a tenth of that; zero biases). */
NPH_GPU_API NphGpuResult nph_gpu_mlp_create(int32_t device, uint64_t seed, NphGpuMlp **out);
NPH_GPU_API void nph_gpu_mlp_destroy(NphGpuMlp *mlp);
/* NPH_GPU_MLP_PARAMS floats in the order above; setting resets the optimiser. */
NPH_GPU_API NphGpuResult nph_gpu_mlp_set_weights(NphGpuMlp *mlp, const float *params);
NPH_GPU_API NphGpuResult nph_gpu_mlp_get_weights(const NphGpuMlp *mlp, float *params);
/* Outputs (count x 3) of `count` feature rows (count x 16), host arrays. */
NPH_GPU_API NphGpuResult nph_gpu_mlp_predict(NphGpuMlp *mlp, const float *features, uint64_t count,
                                             float *out);
/* The gradient (NPH_GPU_MLP_PARAMS floats) and value of the mean over the samples of the
 * squared error summed over the three outputs. */
NPH_GPU_API NphGpuResult nph_gpu_mlp_gradients(NphGpuMlp *mlp, const float *features,
                                               const float *targets, uint64_t count, float *grad,
                                               float *loss);
/* `epochs` passes of Adam (beta 0.9, 0.999, eps 1e-8, step `lr`) over mini-batches of
 * `batch` samples in a seeded shuffled order; writes the final loss over all samples. */
NPH_GPU_API NphGpuResult nph_gpu_mlp_train(NphGpuMlp *mlp, const float *features,
                                           const float *targets, uint64_t count, uint32_t epochs,
                                           uint32_t batch, float lr, uint64_t shuffle_seed,
                                           float *final_loss);

/* Times the network's kernels on `count` device-resident rows (at most 2^31): features and
 * targets a seeded pattern in [-1, 1) written on the device, then `reps` forward launches and
 * `reps` gradient launches over all rows, each timed with CUDA events on the network's stream;
 * writes the average milliseconds of one launch of each. The weights are not changed. */
NPH_GPU_API NphGpuResult nph_gpu_mlp_time_kernels(NphGpuMlp *mlp, uint64_t count, uint32_t reps,
                                                  float *forward_ms, float *gradients_ms);

/* Point slots: manifold g's point k is slot 4 g + k (g in the uploaded colour order). */
#define NPH_GPU_POINT_NONE 0u /* k >= the manifold's point count */
#define NPH_GPU_POINT_WARM 1u /* starts at a persisted (non-zero) impulse */
#define NPH_GPU_POINT_COLD 2u /* starts at zero impulse: new this step */

/* The features of every point slot of the uploaded world at the step's start (host arrays of
 * 4 x manifolds entries; features 16 per slot): in the contact frame (n, t1 =
 * perpendicular(n), t2 = n x t1) with g = |gravity| (1 m/s^2 without gravity) and
 * h = dt / substeps,
 *   0-2  the relative velocity at the point along n, t1, t2, over g h
 *   3-5  n
 *   6    the separation over 0.02 m
 *   7-10 inverse masses of A and B and the angular terms (rA x n).IA^-1(rA x n), same for B,
 *        each over their sum kn (the inverse normal mass)
 *   11   point count / 4
 *   12   friction
 *   13   -n . gravity / |gravity|
 *   14   1 when one side is not dynamic
 *   15   the tangent effective-mass inverse's first entry times kn
 * `scale` is g h / kn, the impulse a network output of 1 stands for; `kind` a
 * NPH_GPU_POINT_* value. */
/* The island sleep decision of a step (phys_island_sleep_and_split, island.c:675-735; world.c:350-
 * 358) on the uploaded world, after its step: the bodies' sleep clocks are read on the device.
 * `island_of` (one per uploaded body, the view's order) gives the place of the body's island in
 * the world's awake-island list, or NPH_GPU_NULL for a body in no island (kinematic);
 * `removed` (one per awake island) its constraint_remove_count; `time_to_sleep` the world's
 * setting. Writes `sleep` (per awake island: 1 when the island falls asleep whole), `*split`
 * (the awake-island place of the island to split, or NPH_GPU_NULL) and `kinematic_sleep` (per
 * body: 1 for a kinematic body that falls asleep on its own clock). Each island's clock is its
 * stillest body's (a body that may not sleep counts as just moved); an island that lost
 * constraints is not put to sleep, and of those whose sleepiest body is ready, the one most
 * ready (first in the list on a tie) is split. The caller carries out the list moves
 * (island_sleep, island_split, the awake list). NPH_GPU_INVALID_ARGUMENT for an island index past
 * island_count. Host arrays. */
NPH_GPU_API NphGpuResult nph_gpu_world_sleep_decision(NphGpuSolver *solver, const uint32_t *island_of,
                                                     uint32_t island_count, const uint32_t *removed,
                                                     float time_to_sleep, uint8_t *sleep, uint32_t *split,
                                                     uint8_t *kinematic_sleep);

/* A hit of hit_events (solver.c:919-960): the manifold (its index in the view) and its point of
 * fastest approach. The caller makes NphPhysicsContactHitEvent from it: its shapes, the point
 * as body A's centre plus the point's anchor_a (nph_dvec3_add_vec3), the manifold's normal. */
typedef struct NphGpuHitEvent {
    uint32_t contact;     /* the manifold's index in its view */
    uint32_t point;
    float approach_speed; /* -relative_velocity, above the threshold */
    uint32_t world;       /* the view's place in a batch (0 for a single world) */
} NphGpuHitEvent;

/* hit_events after a step, on the device-resident records: for each manifold with
 * NPH_GPU_CONTACT_HIT_EVENTS, in the view's order (the colour lists, then the overflow: the
 * reference's order), the point whose approach speed is the largest above `threshold` (the
 * world's hit_threshold, nph_physics_world_set_hit_threshold) among those with a positive
 * max_normal_impulse, the first such point on a tie; manifolds with none make no event. Writes
 * the first min(*count, capacity) events to the host array `events` and the number of events to
 * `*count`. */
NPH_GPU_API NphGpuResult nph_gpu_world_hit_events(NphGpuSolver *solver, float threshold, NphGpuHitEvent *events,
                                                 uint32_t capacity, uint32_t *count);
/* The same for every world of a batch after its step (nph_gpu_phys_solve_worlds, split or not,
 * or resident steps): world by world in the batch's order, each world's hits in its view's
 * order, `world` its place in the batch. */
NPH_GPU_API NphGpuResult nph_gpu_batch_hit_events(NphGpuBatch *batch, float threshold, NphGpuHitEvent *events,
                                                 uint32_t capacity, uint32_t *count);

NPH_GPU_API NphGpuResult nph_gpu_world_features(NphGpuSolver *solver,
                                                const NphGpuWorldParams *params, float dt,
                                                float *features, float *scale, uint32_t *kind,
                                                uint64_t slots);

/* Attaches a network to the solver (NULL detaches it): every following step then starts
 * each cold point at the network's prediction (normal impulse max(out0, 0) x scale, friction
 * out1 and out2 x scale along t1 and t2, scaled back onto the friction cone) instead of
 * zero. */
NPH_GPU_API NphGpuResult nph_gpu_solver_set_warm_start_model(NphGpuSolver *solver, NphGpuMlp *mlp);

/* The starts of the residual-driven mode: cold points at zero (the reference's start); at the
 * attached network's predictions; or at the network's predictions with the plain start as the
 * fallback, kept only when the residual after the warm start is no larger than the plain
 * start's (the reference residual when one is given, else a plain start run first), otherwise
 * the plain start runs again from the records. Every start's device time counts in `ms`. */
#define NPH_GPU_START_PLAIN 0u
#define NPH_GPU_START_LEARNED 1u
#define NPH_GPU_START_GATED 2u

/* The residual-driven mode that judges a warm start. On the uploaded world: prepare, the
 * first substep's velocity integration and warm start (`learned`: an NPH_GPU_START_* value; a
 * network must be attached unless plain), then rigid passes (the relax pass: no softness, speculative rows for
 * separated points) over every colour until the velocity-constraint residual falls to
 * `tolerance` x the reference residual, or `max_passes`. The residual is the L2 norm over
 * points of r_n = |vn + b| where the normal impulse is positive, max(-(vn + b), 0) where not
 * (b = separation / h for a separated point, else 0), plus the slip |vt| of points whose
 * friction impulse is inside the cone. `reference_residual` <= 0 uses this run's own
 * initial residual. `residuals` (optional, max_passes + 1 floats) gets the residual after
 * the warm start and after each pass; `impulses` (optional, 12 per manifold) the final
 * normal, t1 and t2 impulses of every point slot. The uploaded records are not changed. */
typedef struct NphGpuConvergeStats {
    uint32_t passes;           /* passes run */
    uint32_t converged;        /* 1 when the residual reached the tolerance */
    uint32_t cold_points;      /* points that started cold */
    uint32_t predicted_points; /* cold points the network started */
    float initial_residual;    /* after the warm start */
    float final_residual;
    float reference_residual;  /* the denominator */
    float ms;                  /* device time from the first prepare to the last pass */
    uint32_t fell_back;        /* NPH_GPU_START_GATED: 1 when the plain start replaced the network's */
} NphGpuConvergeStats;
NPH_GPU_API NphGpuResult nph_gpu_world_converge(NphGpuSolver *solver,
                                                const NphGpuWorldParams *params, float dt,
                                                uint32_t learned, float tolerance,
                                                uint32_t max_passes, float reference_residual,
                                                float *residuals, float *impulses,
                                                NphGpuConvergeStats *out);

/* ------------------------------------------------------------------------------------
 * Version
 * ---------------------------------------------------------------------------------- */

NPH_GPU_API const char *nph_gpu_version(void);

#ifdef __cplusplus
}
#endif

#endif /* NEPHELINE_B200_H */

/* SPDX-License-Identifier: MIT
 * pmb200 core: the rigid AVBD tick on one B200, behind a plain C ABI.
 *
 * This is the internal operator seam that the reference's CUDA backend
 * implements with per-stage launch wrappers (reference
 * src/simulation/geometry_constraints_dispatch.hpp:12-52 prepare/solve,
 * src/simulation/geometry_dispatch.hpp and primitives.hpp for the spatial and
 * contact stages, sequenced by emit_rigid_solve in
 * src/simulation/production_realtime_backend.cu.inc:7664-7866). One call,
 * pmb_world_step, runs the whole tick on the device: predict, swept proxies,
 * broadphase, convex face narrowphase, contact cache, prepare, colouring,
 * per-colour primal / dual solve, commit, speed clamp, cache save.
 *
 * Records are little-endian, 4-byte fields, tightly packed.
 * Every function returns 0 on success or a negative PMB_ERROR_* code.
 */
#ifndef PMB200_CORE_H
#define PMB200_CORE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PMB_API __attribute__((visibility("default")))

enum {
    PMB_SUCCESS = 0,
    PMB_ERROR_INVALID_ARGUMENT = -1,
    PMB_ERROR_OUT_OF_DEVICE_MEMORY = -4,
    PMB_ERROR_FEATURE_NOT_PRESENT = -5,
    PMB_ERROR_CAPACITY_EXCEEDED = -7,
    PMB_ERROR_DEVICE_LOST = -8,
    PMB_ERROR_NO_DEVICE = -10
};

/* Status bits latched by a tick (pmb_step_stats.status). */
enum {
    PMB_STATUS_CANDIDATE_OVERFLOW = 1u << 0,
    PMB_STATUS_CONTACT_OVERFLOW = 1u << 1,
    PMB_STATUS_PAIR_OVERFLOW = 1u << 2,
    PMB_STATUS_INVALID_BOUNDS = 1u << 3,
    PMB_STATUS_BARRIER_TIMEOUT = 1u << 4,
    PMB_STATUS_COLOR_OVERFLOW = 1u << 5,
    PMB_STATUS_GRID_OVERFLOW = 1u << 6
};

/* BodyParameters order (reference src/slang/types.slang:81-95) without ids
 * or user data. motion: 0 static, 1 kinematic, 2 dynamic. */
typedef struct pmb_body {
    uint32_t motion, mesh;
    float inv_mass, inv_inertia[3], friction, restitution, linear_damping, angular_damping;
    float max_linear_speed, max_angular_speed, margin;
} pmb_body;

/* RigidBodyState / PmRigidState: position, orientation (x,y,z,w), linear and
 * angular velocity (reference include/parallel_mater/parallel_mater.h:392-397). */
typedef struct pmb_state {
    float x[3], q[4], v[3], w[3];
} pmb_state;

/* RigidConstraintOptions (reference src/slang/geometry.slang:95-113) with
 * dense body indices. type: 0 fixed, 1 point, 2 hinge, 3 slider, 4 piston,
 * 5 generic, 6 generic spring, 7 motor. */
typedef struct pmb_joint {
    uint32_t type, body_a, body_b;
    float anchor_a[3], anchor_b[3], frame_a[4], frame_b[4];
    uint32_t lin_limit_axes;
    float lin_lower[3], lin_upper[3];
    uint32_t ang_limit_axes;
    float ang_lower[3], ang_upper[3];
    uint32_t lin_spring_axes;
    float lin_stiffness[3], lin_damping[3];
    uint32_t ang_spring_axes;
    float ang_stiffness[3], ang_damping[3];
    uint32_t motor_linear, motor_angular;
    float motor_linear_velocity, motor_linear_max_impulse;
    float motor_angular_velocity, motor_angular_max_impulse;
    uint32_t enabled, disable_collisions;
    float breaking_threshold;
    uint32_t solver_iterations;
} pmb_joint;

/* Scene description. Meshes are triangle meshes; mesh m owns vertices
 * [vertex_offsets[m], vertex_offsets[m+1]) and indices [index_offsets[m],
 * index_offsets[m+1]). Capacities of 0 select defaults sized from body_count. */
typedef struct pmb_world_desc {
    uint32_t body_count;
    const pmb_body* bodies;
    const pmb_state* states;
    uint32_t mesh_count;
    const uint32_t* vertex_offsets; /* mesh_count + 1 */
    const float* vertices;          /* xyz */
    const uint32_t* index_offsets;  /* mesh_count + 1 */
    const uint32_t* indices;
    uint32_t joint_count;
    const pmb_joint* joints;
    uint32_t candidate_capacity; /* broadphase pairs */
    uint32_t pair_capacity;      /* non-empty manifolds */
    uint32_t contact_capacity;   /* contact points */
    int32_t device;              /* CUDA ordinal */
    /* Optional caller-owned device memory (both or neither, 256-byte
     * aligned), sized by pmb_world_memory_requirements. When given, every
     * device array of the world is carved from it and the world allocates no
     * device memory; otherwise the world allocates its own. */
    void* persistent_memory;
    uint64_t persistent_bytes;
    void* scratch_memory;
    uint64_t scratch_bytes;
    /* Optional batch of independent scenes stepped together (scene_count >
     * 1): body_scene[i] is body i's scene, non-decreasing (each scene's
     * bodies contiguous); bodies of different scenes never collide; joints
     * stay within a scene. Every scene sweeps its own budget: the tick's
     * rule applied per scene, with scene_iterations[s] (optional, 0 = none)
     * as the scene's requested iterations. The residual-driven schedule
     * does not apply to batches. */
    uint32_t scene_count;
    const uint32_t* body_scene;
    const uint32_t* scene_iterations;
    /* Contact events kept per tick when a step asks for them (0: none). */
    uint32_t event_capacity;
} pmb_world_desc;

/* Upper bounds for sizing caller-owned memory. Capacities of 0 select the
 * defaults pmb_world_create would derive from body_count. */
typedef struct pmb_world_capacity {
    uint32_t body_count, joint_count, mesh_count, mesh_vertex_count, mesh_triangle_count;
    uint32_t candidate_capacity, pair_capacity, contact_capacity;
    uint32_t event_capacity;
} pmb_world_capacity;

/* profile: 1 = realtime v1 (8 sweeps, 5% damping), otherwise legacy
 * (requested_iterations, or base_iterations raised by joint iteration hints,
 * plus the velocity impact phase). residual_tolerance > 0 switches to the
 * residual-driven schedule: sweep until the residual is at or below the
 * tolerance, at most max_iterations sweeps; residual_norm picks the residual
 * the schedule tests: 0 the largest row violation of the sweep (every
 * constraint within the tolerance, in metres), 1 the RMS over the rows, 2 the
 * 99.9th percentile (at most one active row in a thousand above the
 * tolerance). warm_start selects where each
 * contact's normal row (lambda, penalty) starts: 0 plain (the reference's
 * cached-and-decayed warm start), 1 learned (the world's MLP predictor, when
 * one is attached; plain otherwise), 2 the table set by
 * pmb_world_set_warm_table. */
typedef struct pmb_step_desc {
    float dt, gravity[3];
    uint32_t profile, requested_iterations, base_iterations;
    float residual_tolerance;
    uint32_t max_iterations;
    uint32_t warm_start;
    uint32_t collect_events; /* nonzero: record this tick's contact events */
    uint32_t residual_norm;  /* 0: largest row violation, 1: RMS, 2: 99.9th percentile (residual-driven schedule) */
} pmb_step_desc;

/* residual: RMS, over contact normal rows that carry force or penetrate and
 * hard joint rows, of the constraint violation after the last sweep (|C| for
 * rows with force, C for rows active by penetration only), in metres;
 * residual_max: the largest single row violation after the last sweep;
 * residual_over: the fraction of those rows whose violation exceeds the
 * step's residual_tolerance. */
typedef struct pmb_step_stats {
    uint32_t candidate_pairs, active_pairs, contacts, colors, islands, iterations, impact, status;
    float residual, residual_max, residual_over;
} pmb_step_stats;

typedef struct pmb_world pmb_world;

/* Create a world on a CUDA device; uploads the scene and prepares meshes.
 * Fails with PMB_ERROR_NO_DEVICE when no CUDA device is present: there is
 * no CPU fallback. */
PMB_API int pmb_world_create(const pmb_world_desc* desc, pmb_world** out);
PMB_API void pmb_world_destroy(pmb_world* world);

/* Bind a CUDA stream (cudaStream_t as void*) used by every later call. */
PMB_API int pmb_world_set_stream(pmb_world* world, void* stream);

/* One tick. Enqueued on the world's stream; returns without synchronising
 * unless stats is non-null, in which case it waits and fills stats. */
PMB_API int pmb_world_step(pmb_world* world, const pmb_step_desc* step, pmb_step_stats* stats);

/* Diagnostic: run one tick with CUDA events between its stages and write
 * "stage  ms" lines into report (synchronous). */
PMB_API int pmb_world_profile_step(pmb_world* world, const pmb_step_desc* step, char* report, uint32_t capacity);

/* Dominant-kernel timing: with enable != 0, later ticks bracket every solve
 * launch with CUDA events on the world's stream. Each call synchronises,
 * returns the summed duration and launch count of the launches recorded since
 * the previous call, and sets the enable state. */
PMB_API int pmb_world_solve_timer(pmb_world* world, int enable, float* total_ms, uint32_t* launches);

/* Mesh BVH build on the GPU, for meshes too large to prepare on the host:
 * the tree the host preparation builds (the reference's upload-time builder,
 * src/simulation/runtime_deformables.cu.inc:136-210: median split on the
 * longest axis of the node's triangle bounds, triangles ordered by centroid
 * on that axis with ties by index, leaves of at most 4 triangles, nodes in
 * pre-order). `vertices` (3 floats each), `indices` (3 per triangle),
 * `order` (one per triangle: the original index of the triangle stored at
 * each position) and `nodes` (10 words per node: lo[3], hi[3] as floats;
 * first, count (0 for an inner node), left, right as uint32) are device
 * memory; `node_count` (host) receives the node count, and a capacity below
 * it returns PMB_ERROR_CAPACITY_EXCEEDED; an index at or past `vertex_count`
 * returns PMB_ERROR_INVALID_ARGUMENT before any other device work. Work runs on `stream` (CUDA
 * stream, null for the default); the call allocates scratch with cudaMalloc
 * and returns after the stream has finished. */
PMB_API int pmb_mesh_bvh_build(const float* vertices, uint32_t vertex_count, const uint32_t* indices,
                               uint32_t index_count, uint32_t* order, float* nodes, uint32_t node_capacity,
                               uint32_t* node_count, void* stream);

/* Host mesh preparation used at world creation (no device work): triangles
 * reordered into median-split BVH leaf order, one outward plane (n, d) per
 * triangle when the mesh is a closed convex shell, bounds (lo, hi, centre,
 * radius). Mirrors the reference's upload path
 * (src/simulation/runtime_deformables.cu.inc:103-270). */
PMB_API int pmb_prepare_mesh(const float* vertices, uint32_t vertex_count, const uint32_t* indices,
                             uint32_t index_count, uint32_t* out_indices, float* out_planes, float* out_bounds,
                             int* convex);

/* First-fit colouring of a caller-supplied graph without allocating memory.
 * No counterpart in the reference: it is this library's own entry point for
 * callers that cannot call cudaMalloc -- a pm* driver working only in memory
 * the application binds to it, or a real-time thread that must not stall on
 * an allocation. All pointers are device pointers on `device`, owned by the
 * caller: offsets[vertex_count + 1] and neighbors[] form an undirected
 * adjacency (CSR), dynamic[v] != 0 marks vertices that take a colour; each
 * dynamic vertex gets, in index order, the smallest colour absent among its
 * lower-index dynamic neighbours (the tick's constraint-graph colouring);
 * others get 0xffffffff. Enqueued on `stream` (cudaStream_t), then waited for.
 * Working memory is a fixed array inside the library (one per GPU, held until
 * the process exits) for at most 1,048,576 vertices; larger graphs return
 * PMB_ERROR_CAPACITY_EXCEEDED, and so do graphs needing more than 256 colours.
 * The first call on a device resolves that array's address, so make it before
 * any stream capture. Every call reads its status back and waits for `stream`;
 * a `stream` in capture mode is rejected with PMB_ERROR_INVALID_ARGUMENT
 * before any work is enqueued. The caller's current device is restored before
 * the call returns. Calls share the array: calls that overlap on the GPU
 * (other streams, other threads) race and must be serialised by the caller. */
PMB_API int pmb_graph_color_noalloc(const uint32_t* offsets, const uint32_t* neighbors, const uint32_t* dynamic,
                                    uint32_t vertex_count, uint32_t* colors, int32_t device, void* stream);

/* Number of CUDA kernels this library has enqueued in this process. */
PMB_API int pmb_kernel_launches(unsigned long long* count);

/* Capture `steps` ticks into a CUDA graph (replayed by pmb_world_replay). */
PMB_API int pmb_world_capture(pmb_world* world, const pmb_step_desc* step, uint32_t steps);
PMB_API int pmb_world_replay(pmb_world* world);

/* Host <-> device state transfer (synchronous on the world's stream). */
PMB_API int pmb_world_get_states(pmb_world* world, pmb_state* out);
PMB_API int pmb_world_set_states(pmb_world* world, const pmb_state* in);
/* Stats of the last tick (synchronises). */
PMB_API int pmb_world_last_stats(pmb_world* world, pmb_step_stats* out);
/* Linear and angular impulse applied by the next tick's predictor. */
PMB_API int pmb_world_apply_impulse(pmb_world* world, uint32_t body, const float* linear, const float* angular);

/* Inspection of the last tick (synchronous). Counts are returned even when
 * the output pointer is null or the capacity is too small. A pair code is
 * a * N + b for query body a, other body b and N bodies, held in 64 bits (the
 * reference's 32-bit code, geometry.slang:907-913, overflows above 65,535
 * bodies); codes ascend in the active-pair order. */
PMB_API int pmb_world_candidate_pairs(pmb_world* world, uint64_t* codes, uint32_t capacity, uint32_t* count);
/* Per non-empty manifold: pair code, point count; 8 contact slots of 22
 * floats (normal, point, penetration, error, dual lambda/penalty x3,
 * anchor a, anchor b). */
PMB_API int pmb_world_manifolds(pmb_world* world, uint64_t* codes, uint32_t* counts, float* contacts,
                                uint32_t capacity, uint32_t* count);
PMB_API int pmb_world_graph(pmb_world* world, uint32_t* colors, uint32_t* parents);
PMB_API int pmb_world_residual_trace(pmb_world* world, float* out, uint32_t capacity, uint32_t* count);

/* Snapshot / restore of the complete dynamic state (states, contact cache,
 * warm-start history) into a second device buffer owned by the world.
 * Worlds in caller-owned memory have none: PMB_ERROR_FEATURE_NOT_PRESENT. */
PMB_API int pmb_world_snapshot(pmb_world* world);
PMB_API int pmb_world_restore(pmb_world* world);

/* Bytes of persistent (state kept between ticks) and scratch (rebuilt by
 * every tick) device memory a world within these bounds needs. The split
 * follows the reference's PmSimulationMemoryRequirements
 * (include/parallel_mater/parallel_mater.h:381-384). */
PMB_API int pmb_world_memory_requirements(const pmb_world_capacity* capacity, uint64_t* persistent,
                                          uint64_t* scratch);

/* Per-body inputs for the next tick, which consumes and clears them
 * (reference SimulationRuntime::apply_rigid_input,
 * src/simulation/runtime_rigid.cu.inc:265-294, and pm_clear_rigid_inputs,
 * src/slang/geometry.slang:2877-2886). values: 12 floats per body -- force,
 * torque, linear impulse, angular impulse -- replacing the body's pending
 * inputs; bodies must be distinct. Enqueued on the world's stream. */
PMB_API int pmb_world_set_inputs(pmb_world* world, uint32_t count, const uint32_t* bodies, const float* values);

/* Kinematic targets for the next tick (position and orientation of each
 * record are used; reference set_kinematic_target, runtime_rigid.cu.inc:197-230).
 * The predictor moves each kinematic body onto its target and derives its
 * velocity from the motion. */
PMB_API int pmb_world_set_targets(pmb_world* world, uint32_t count, const uint32_t* bodies,
                                  const pmb_state* targets);

/* Overwrite the states of bodies [first, first + count) (reference
 * set_rigid_body_state, runtime_rigid.cu.inc:147-195): orientation
 * normalised, velocity history, pending inputs and targets of those bodies
 * cleared, rows of joints touching them restarted. */
PMB_API int pmb_world_write_states(pmb_world* world, uint32_t first, uint32_t count, const pmb_state* states);

/* Enqueue a copy of states [first, first + count) as pmb_state records into
 * device memory `dst` (4-byte aligned) on the world's stream. */
PMB_API int pmb_world_copy_states_to_device(pmb_world* world, uint32_t first, uint32_t count, void* dst);

/* Work telemetry of the latest tick, in the reference's realtime work phases
 * (realtime_telemetry.hpp: boundary, predict, index, candidates, domain,
 * coupling, commit): kernel dispatches and thread blocks enqueued per phase,
 * algorithmic bytes per phase (the per-body and per-contact costs of the
 * kernels), grid-wide barriers (colour rounds and sweeps), sweeps and
 * spatial-index builds. Feeds PM_QUERY_REALTIME_STEP_STATISTICS. */
typedef struct pmb_tick_telemetry {
    uint64_t tick;
    uint64_t dispatches[7], workgroups[7], bytes_moved[7], barriers[7];
    uint64_t sweeps, spatial_builds;
} pmb_tick_telemetry;
PMB_API int pmb_world_tick_telemetry(pmb_world* world, pmb_tick_telemetry* out);

/* One contact point of the last tick that collected events, in active-pair
 * order (pm_prepare_parallel_contact_events, geometry.slang:2902-2939, and
 * the impulses of pm_save_rigid_contact_cache, :3028-3043): the pair's
 * bodies (dense indices, query body first), the point and normal, the
 * penetration (>= 0) and the normal and friction impulses of the tick. */
typedef struct pmb_contact_event {
    uint32_t body, collider;
    float position[3], normal[3];
    float penetration, normal_impulse;
    float friction_impulse[3];
} pmb_contact_event;
/* Copies at most `capacity` events of the last tick into `out` (host
 * memory); `count` receives the tick's event count (min(contact points,
 * event capacity); 0 when the tick did not collect). */
PMB_API int pmb_world_contact_events(pmb_world* world, pmb_contact_event* out, uint32_t capacity, uint32_t* count);

/* Joint state after the last tick (synchronous): flags bit 0 enabled, bit 1
 * broken; applied impulse; number of solver rows. capacity >= joint_count. */
PMB_API int pmb_world_joints(pmb_world* world, uint32_t* flags, float* applied, uint32_t* counts,
                             uint32_t capacity);

/* (lambda, penalty) of the first `rows` rows (1: normal; 3: normal and both
 * friction rows) of every contact point after the last tick, in contact
 * order, `rows` values per point (synchronous). Counts are returned even when
 * the output pointers are null or the capacity is too small. */
PMB_API int pmb_world_contact_duals(pmb_world* world, uint32_t rows, float* lambda, float* penalty,
                                    uint32_t capacity, uint32_t* count);

/* Per-contact start values for ticks run with warm_start = 2: row x of
 * contact point c (in contact order) starts from (lambda[rows*c+x],
 * penalty[rows*c+x]) for c < count and x < rows. A penalty <= 0 keeps the
 * plain penalty; a negative normal lambda or a NaN friction lambda keeps the
 * plain lambda. Copied to the device (synchronous). */
PMB_API int pmb_world_set_warm_table(pmb_world* world, uint32_t rows, const float* lambda, const float* penalty,
                                     uint32_t count);

/* ---- learned warm start ----
 * An 8 -> 64 -> 64 -> 2 MLP (BF16 tensor-core kernels, FP32 accumulation and
 * FP32 master weights) predicting each contact's converged normal-row
 * (lambda, penalty) from its features at the start of the tick, as a
 * log-space correction of the plain warm start (an all-zero output layer,
 * the initial state, reproduces the plain warm start). It has no
 * counterpart in the reference: the reference's warm start is the cached,
 * decayed dual (constraint_math.slang:30-37), which stays the default
 * (warm_start = 0) and the fallback for non-finite predictions.
 * Parameter vector (PMB_MLP_PARAMS floats, row-major): W1[64][16],
 * W2[64][80], W3[16][80]; biases live in column 8 of W1 and column 64 of W2
 * and W3 (constant-one inputs); rows 2..15 of W3 and padding columns are 0. */
#define PMB_MLP_PARAMS 7424u

/* Attach a predictor to a world (device buffers allocated once): params, or
 * a deterministic initialisation from seed when params is null. Resets the
 * optimiser. Not available for worlds in caller-owned memory. */
PMB_API int pmb_world_mlp_attach(pmb_world* world, const float* params, uint32_t seed);
/* What learned ticks take from the predictor: bit 0 the normal lambda, bit 1
 * the normal penalty, bit 2 lambda corrections averaged over each
 * manifold's points (keeping the carried-over split of the pair's force).
 * Default 3 (lambda and penalty per point): on the settled 65,536-box pile,
 * under the 99.9th-percentile residual rule, the predicted lambda and
 * penalty take a quarter of the sweeps off the plain warm start's, the
 * penalty alone a tenth. */
PMB_API int pmb_world_mlp_apply_mode(pmb_world* world, uint32_t mode);
/* Online training: when enabled, every tick ends with steps_per_tick Adam
 * steps (learning_rate) on that tick's contacts, target = the converged
 * normal-row (lambda, penalty), loss = mean squared error of the normalised
 * pair. */
PMB_API int pmb_world_mlp_train(pmb_world* world, int enable, float learning_rate, uint32_t steps_per_tick);
/* Current master parameters, the last training step's loss, the loss the
 * plain warm start (a zero correction) has on the same rows, and the gate:
 * learned ticks apply predictions only while the gate is open (1), which
 * online training sets after each tick's first step from loss < 0.9 x plain
 * loss; attaching given parameters opens it. Null pointers are skipped;
 * synchronous. */
PMB_API int pmb_world_mlp_params(pmb_world* world, float* params, float* last_loss, float* plain_loss,
                                 float* gate);
/* The last tick's MLP rows (synchronous): 8 features per contact (as stored,
 * BF16 values widened to float) and 4 metadata floats (y0, y1, weight,
 * scale: after a training tick y0/y1 are the targets, otherwise the plain
 * warm start in the model's log space). For inspection and tests. */
PMB_API int pmb_world_mlp_rows(pmb_world* world, float* features, float* meta, uint32_t capacity, uint32_t* count);
/* One forward and backward pass over `rows` given rows (features: 8 per row,
 * targets: 2 per row, weights: loss weight per row), host buffers; returns
 * the outputs (2 per row), the gradient of the weighted squared-error loss
 * with respect to every parameter, and the loss. For checking the device
 * kernels against a CPU restatement. */
PMB_API int pmb_mlp_forward_backward(int32_t device, uint32_t rows, const float* features, const float* targets,
                                     const float* weights, const float* params, float* outputs, float* grads,
                                     float* loss);

/* Per-scene results of the last tick of a batched world (synchronous): RMS
 * and largest row violation of the scene's last sweep (the tick's residual
 * definition), sweeps run, contact points. Null pointers are skipped;
 * capacity >= scene_count. */
PMB_API int pmb_world_scene_stats(pmb_world* world, float* residual, float* residual_max, uint32_t* iterations,
                                  uint32_t* contacts, uint32_t capacity);

/* ---- launch plan ----
 * How the cooperative solve kernel is launched: solve_variant 0, 1, 2 = 512,
 * 384, 256 threads per CTA (one CTA per SM; fewer threads leave each thread
 * more registers), 3, 4 = the staged solve with fused dual updates at 512 and
 * 384 threads; solve_policy 0 = 8, 16 or 32 lanes per body chosen per colour
 * by its size, 1 = always 8, 2 = per body by its contact rows (more than 16:
 * 32 lanes, 9-16: 16, else 8; heaviest bodies first) unless 32-lane groups
 * cover the whole colour, 3 = widths as 0 with the colour's bodies claimed
 * dynamically from a counter, 4 = one thread per body in colours with more
 * bodies than 16-lane groups, else as 0. Every plan computes bit-identical
 * results; only the speed differs. A new world starts with (0, 0). */
PMB_API int pmb_world_set_launch_plan(pmb_world* world, uint32_t solve_variant, uint32_t solve_policy);
/* Bound on the polls a thread block makes at a grid barrier of the tick's
 * cooperative kernels (colouring fixpoint, solve) before it gives up (0: the
 * default, 2^26 polls, seconds). A barrier that runs out latches
 * PMB_STATUS_BARRIER_TIMEOUT in the tick's status, the remaining cooperative
 * kernels of the tick return at once and the host reads the status after the
 * tick (the pm* driver reports it as PM_ERROR_DEVICE_LOST); the next tick
 * starts with clean counters. A small limit makes the waits run out on
 * purpose, which is how failure detection is exercised without a GPU fault.
 * Takes effect for ticks enqueued afterwards (not for graphs already
 * captured). */
PMB_API int pmb_world_set_barrier_limit(pmb_world* world, uint32_t spins);
/* Time `ticks` ticks of every plan from the current state (restored before
 * each plan and at the end, so the world does not advance), keep the fastest
 * and report it; `report` receives one line per plan. Needs snapshot
 * storage (not for worlds in caller-owned memory). */
PMB_API int pmb_world_autotune(pmb_world* world, const pmb_step_desc* step, uint32_t ticks,
                               uint32_t* solve_variant, uint32_t* solve_policy, char* report, uint32_t capacity);

/* The CUDA stream (cudaStream_t) the world enqueues its work on. */
PMB_API int pmb_world_stream(pmb_world* world, void** stream);

/* ---- device services ----
 * The pm* driver (libpm_b200_driver.so) reaches CUDA only through these, so
 * that a single CUDA runtime serves the process. Pointers are CUDA device or
 * managed pointers; streams and events are cudaStream_t / cudaEvent_t. */
typedef struct pmb_device_info_t {
    char name[256];
    uint8_t uuid[16];
    uint64_t total_memory;
    uint32_t multiprocessors, compute_major, compute_minor, pci_device, driver_version;
} pmb_device_info_t;
PMB_API int pmb_device_count(int32_t* count);
PMB_API int pmb_device_info(int32_t device, pmb_device_info_t* info);
PMB_API int pmb_device_memory_info(int32_t device, uint64_t* free_bytes, uint64_t* total_bytes);
/* host_visible != 0: managed memory (one pointer for host and device). */
PMB_API int pmb_device_alloc(int32_t device, uint64_t bytes, int host_visible, void** out);
PMB_API int pmb_device_free(int32_t device, void* ptr);
PMB_API int pmb_stream_create(int32_t device, void** stream);
PMB_API int pmb_stream_destroy(int32_t device, void* stream);
PMB_API int pmb_stream_synchronize(int32_t device, void* stream);
PMB_API int pmb_copy_async(int32_t device, void* dst, const void* src, uint64_t bytes, void* stream);
PMB_API int pmb_event_create(int32_t device, void** event);
PMB_API int pmb_event_destroy(int32_t device, void* event);
PMB_API int pmb_event_record(int32_t device, void* event, void* stream);
PMB_API int pmb_event_query(int32_t device, void* event, int* ready);
PMB_API int pmb_event_elapsed_ms(int32_t device, void* start, void* end, float* ms);

/* Core AVBD math on the device, one thread per record, for parity checks
 * against the CPU restatement. Host pointers; synchronous.
 * block: in 27 floats (h[21], g[6]) -> out 7 floats (delta[6], solved).
 * dual:  in 7 floats -> out 5 (warm lambda/penalty, force, updated lambda/penalty).
 * contact: in 4 floats (trial n,t0,t1, friction) -> out 6 (projected, scales).
 * row: in 42 floats -> out 7 (see tests).
 * trig (kind 4): in 3 floats (y, x, t) -> out 2 (atan2(y, x) for y, x >= 0,
 * t cos(t) / sin(t) for t in [0, pi/2]), the tick's own evaluations. */
PMB_API int pmb_math_eval(uint32_t kind, uint32_t count, const float* in, float* out);

#ifdef __cplusplus
}
#endif
#endif

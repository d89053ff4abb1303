// SPDX-License-Identifier: MIT
// Device-side layout of one rigid world. Everything the tick touches lives in
// HBM as structure-of-arrays, float4-packed so a warp's loads coalesce:
//   bodies    N   x (params 3 x float4, state 4 x float4 current + target)
//   pairs     P   (a, b, contact offset, count) for non-empty manifolds, code order
//   contacts  C   8 float4 per point (normal|pen, point|impact, error|speed,
//                 anchor a|cached, anchor b, lambda|acc_n, penalty, acc_f)
//   graph     per-body CSR of incident pairs (descending pair index, which is
//             the reference's head-inserted list order), joints likewise
// Counters live in one device struct so no stage needs a host round trip and
// a whole tick can be captured into a CUDA graph.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "pmb_math.cuh"

namespace pmb {

enum : uint32_t { kStatic = 0, kKinematic = 1, kDynamic = 2 };
enum : uint32_t { kFixed, kPoint, kHinge, kSlider, kPiston, kGeneric, kGenericSpring, kMotor };
constexpr uint32_t kMaxColors = 256;
constexpr uint32_t kQueryLanes = 8;  // broadphase query lanes per body
// The colour fixpoint runs one 1024-thread CTA per SM: its ~30 rounds are
// two grid barriers each, and a barrier's cost grows with the CTA count.
constexpr int kColorThreads = 1024;
// Sort classes of a colour's bodies by the length of their row lists,
// heaviest first, in steps of 8 rows (an 8-lane group stages 8 rows at a
// time): more than 40, 33-40, 25-32, 17-24, 9-16, at most 8. A colour phase
// ends with its slowest lane group, and the static assignment deals the
// colour's bodies out in rounds of alternating direction, so with the bodies
// in this order a group that draws a heavy body in one round draws a light
// one in the next. The lane widths of solve policy 2 take unions of them:
// more than 16 rows (classes 0-3) 32 lanes, 9-16 (class kClass16) 16 lanes,
// at most 8 (class kClass8) 8 lanes.
constexpr uint32_t kSortClasses = 6;
constexpr uint32_t kClass16 = 4, kClass8 = 5;
__host__ __device__ inline uint32_t sort_class(uint32_t rows) {
    return rows > 40u ? 0u : rows > 32u ? 1u : rows > 24u ? 2u : rows > 16u ? 3u : rows > 8u ? kClass16 : kClass8;
}
constexpr uint32_t kMaxIterations = 256;
constexpr int kBlock = 256;

// Status bits (pmb200_core.h).
enum : uint32_t {
    kStCandidateOverflow = 1u << 0,
    kStContactOverflow = 1u << 1,
    kStPairOverflow = 1u << 2,
    kStInvalidBounds = 1u << 3,
    kStBarrierTimeout = 1u << 4,
    kStColorOverflow = 1u << 5,
    kStGridOverflow = 1u << 6,
};

struct Counters {
    uint32_t n_cand, n_stage, n_act, n_contacts;
    uint32_t n_large, colors, islands, iterations;
    uint32_t impact, status, changed, rounds;
    uint32_t bar_count, bar_gen, budget, joint_iters;
    float hs, residual, pad1, pad2;
    uint32_t budget_max;  // batched scenes: the largest scene budget of the tick
    uint32_t n_surv;      // narrowphase candidates left for the manifold pass
    uint32_t n_events;    // contact events recorded by the tick
    uint32_t n_mesh;      // candidates left for the triangle-mesh path
    uint32_t n_mesh_leaves, n_mesh_items;  // their overlapping leaf pairs and triangle-pair items
    uint32_t claim[2];    // solve policy 3: next unclaimed body of the colour (alternating)
    // Bodies bucketed by (colour, sort class): bucket col * kSortClasses + k.
    uint32_t color_count[kMaxColors * kSortClasses];
    uint32_t color_off[kMaxColors * kSortClasses + 1];
    float residual_trace[kMaxIterations];
    double res_sum[1024];  // per-block partial residual sums of the latest dual pass
    uint32_t res_cnt[1024];
    float res_mx[1024];
    uint32_t res_over[1024];  // per-block rows above the tolerance
    float residual_max;
    float residual_over;  // fraction of active rows above the tolerance after the last sweep
    unsigned long long dbg_work[20], dbg_release[20], dbg_start;
    unsigned long long dbg_body[8];
    unsigned long long dbg_sum[8];  // colour 0 of the first sweep: stage sums, bodies, rows
    uint32_t dbg_rn;
};

struct StepParams {
    float dt;
    float gx, gy, gz;
    uint32_t realtime;
    uint32_t budget_request;  // requested or base iterations
    uint32_t requested;
    float tolerance;
    uint32_t max_iterations;
    uint32_t debug_timing;  // record solve-kernel timestamps for iteration 0
    uint32_t warm_start;    // 0 plain, 1 learned, 2 table
    uint32_t collect_events;
    uint32_t residual_norm;  // residual-driven schedule: 0 largest row violation, 1 RMS, 2 99.9th percentile
};

struct ContactEvent {  // pmb_contact_event
    uint32_t body, collider;
    float position[3], normal[3];
    float penetration, normal_impulse;
    float friction_impulse[3];
};
static_assert(sizeof(ContactEvent) == 52, "event record");

struct JointRow {  // constraint_math.slang AvbdRow, packed for the device
    float a[6], b[6];
    float lambda, penalty, error, velocity, lower, upper, stiffness, damping, beta, reference_force;
};

struct Joint {
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
};
static_assert(sizeof(Joint) == 220, "joint record");

struct JointState {
    uint32_t enabled, broken, count, dense_a, dense_b, pad0, pad1, pad2;
    float applied;
};

// Every device pointer of a world. Passed by value to kernels.
struct Dev {
    uint32_t n, nm, nj;
    uint32_t cap_cand, cap_stage, cap_pair, cap_contact;
    uint32_t grid_size;  // hash table buckets (power of two)
    float large_extent;  // AABB extent above which a body is tested by brute force
    // body parameters
    uint32_t* motion;
    uint32_t* mesh;
    float4* p0;  // inv_mass, inv_inertia xyz
    float4* p1;  // friction, restitution, linear damping, angular damping
    float4* p2;  // max linear, max angular, margin, correction reach
    float* expand;  // proxy expansion: min(1, correction) + reach
    float* rotb;    // |max-abs mesh corner| for the rotational motion bound
    // state: current (start of tick) and target (predicted, then solved)
    float4 *x, *q, *v, *w;
    float4 *tx, *tq, *tv, *tw;
    // per-tick inputs, cleared by the predictor that consumes them
    float4 *force, *torque, *lin_imp, *ang_imp;
    float4 *tgt_x, *tgt_q;  // kinematic target (w of tgt_x: 1 = set)
    // Launch plan (pmb_world_autotune): solve kernel variant, colour width
    // policy (0: 8/16/32 lanes per body by colour size, 1: always 8).
    uint32_t solve_variant, solve_policy;
    // Spins a block waits at a grid barrier before it gives up, latches
    // kStBarrierTimeout and abandons the tick (pmb_world_set_barrier_limit).
    uint32_t barrier_spins;
    // Batched independent scenes (n_scenes > 1): bodies of scene s are the
    // contiguous range [scene_body_off[s], scene_body_off[s+1]). Bodies of
    // different scenes never pair: grid buckets are keyed by scene, large
    // bodies are listed per scene, and every scene sweeps its own budget.
    uint32_t n_scenes;
    uint32_t* scene_of;          // per body
    uint32_t* scene_body_off;    // n_scenes + 1
    uint32_t *scene_large_count, *scene_large_off, *scene_large_cursor, *scene_large_list;
    uint32_t* scene_iters;       // requested iterations per scene (0: base, raised by joint hints)
    uint32_t* scene_jiters;      // per tick: largest joint iteration hint
    uint32_t* scene_budget;      // per tick: the scene's sweeps
    float *scene_res_sq, *scene_res_mx;  // per tick: residual of the scene's last sweep
    float* scene_hs;                     // per tick: the scene's broadphase cell size
    uint32_t* scene_res_n;
    // warm-start table: per contact point, lambda (x, y, z rows) and penalty
    float4* warm_table;  // 2 per contact: lambda, penalty
    uint32_t warm_count, warm_rows;
    // host-to-device staging for sparse per-body records
    uint32_t* io_index;
    float4* io_rec;  // 4 per record
    // meshes
    uint32_t *m_vo, *m_vc, *m_to, *m_tc, *m_convex;
    float4* m_verts;
    float4* m_planes;
    // triangle-mesh path: convex at any size; first BVH node; first shell
    // normal (kInvalid: the mesh has none); local bounds; BVH nodes as three
    // float4 (lo, first), (hi, count), (left, right); a certified outward
    // normal per triangle
    uint32_t *m_solid, *m_bo, *m_so;
    float4 *m_lo, *m_hi;
    float4* m_bvh;
    float4* m_shell;
    // hinge contact frames of the tick (reference point; flags in w) and
    // each body's joints in ascending index
    float4 *frame, *frame_prev;  // at the predicted and at the previous poses
    float4 *frame_guide, *frame_anchor;  // guide axis + inverse mass, anchor + inverse moment (predicted poses)
    uint32_t *jb_off, *jb_list;
    uint32_t* np_mesh;  // candidates for the triangle-mesh path
    // the flat mesh path: per pair leaf-pair and item counts, their exclusive
    // scans and flags; per leaf pair (first, count) of both ranges and its
    // first item; per item the contact (point, impact), (normal, depth)
    uint32_t cap_mesh, cap_mesh_leaves, cap_mesh_items;
    uint32_t *mp_leaves, *mp_items, *mp_flags, *mp_leaf_off, *mp_item_off;
    uint4* ml_rec;
    uint32_t *ml_item, *ml_pair;
    uint8_t* mi_valid;
    float4 *mi_p, *mi_n;
    // AVBD body state
    float4 *dxl, *dxa, *dq;
    float4 *inA, *inB;  // inertia block: (m/dt2, h33, h43, h44), (h53, h54, h55, -)
    float4* prev_vel;   // xyz + history flag in w
    uint32_t *color, *parent, *impact, *anchored;
    uint32_t* island_end;  // largest member index of each island (at its root)
    float4* mean;       // free-island mean displacement (roots)
    // broadphase
    float4 *lo, *hi;
    uint32_t* is_large;
    uint32_t* large_list;
    uint32_t *bucket_count, *bucket_off, *bucket_cursor;
    uint32_t* grid_body;
    int4* grid_cell;
    uint32_t *cand_count, *cand_off;
    uint32_t* cand_lane;  // per query body, each query lane's candidate count
    uint32_t *cand_a, *cand_b;
    // narrowphase
    uint32_t* np_count;
    uint64_t* np_scan;
    uint32_t* np_stage;
    uint32_t* np_list;  // candidates surviving the separating-axis pass
    uint2* np_sat;      // their separation (float bits) and reference face (bit 31: side)
    float4 *st_n, *st_p;
    // active pairs / contacts
    uint32_t *act_a, *act_b, *act_off, *act_cnt, *act_impact;
    uint64_t* act_code;  // a * N + b in 64 bits (the reference's uint32 code while N <= 65,535)
    uint32_t* c_pair;
    uint2* c_bodies;  // (a, b) of the contact's pair
    float4* c_jac;    // 9 per contact: jacobian rows n,t0,t1 of body a then body b
    float4 *c_n, *c_p, *c_e, *c_aa, *c_ab, *c_lam, *c_pen, *c_accf;
    // Velocity phase: per contact the force offsets of its rows (lambda.w /
    // dt, and the accumulated friction along each tangent / dt), fixed for
    // the phase and formed once with its jacobians.
    float4* c_foff;
    // Per contact, fixed for the tick: friction sqrt(mu_a mu_b) and the
    // penalty growth factor 100 / (max(w_a + w_b, 1e-6) dt^2) of its pair,
    // formed with the position phase's jacobians.
    float2* c_mub;
    // contact cache from the previous tick (double-buffered by the host)
    uint64_t* sv_code;
    uint32_t *sv_off, *sv_cnt;
    uint32_t* sv_n_pairs;  // device count of saved pairs
    float4 *sv_local, *sv_normal, *sv_fimp, *sv_lam, *sv_pen, *sv_aa, *sv_ab;
    float* sv_dt;
    uint64_t* out_code;
    uint32_t *out_off, *out_cnt, *out_n_pairs;
    float4 *out_local, *out_normal, *out_fimp, *out_lam, *out_pen, *out_aa, *out_ab;
    float* out_dt;
    // graph
    uint32_t *deg, *inc_off, *inc_cursor, *inc_list;
    uint32_t *jdeg, *jinc_off, *jinc_cursor, *jinc_list;
    uint32_t* corder;
    uint4* crec;  // per colour-order slot: body, row offset, row count, impact flag (the solve's body records)
    uint8_t* cdirty;  // colour rounds: two flag arrays of n (bodies to revisit)
    uint32_t *nbr, *nlow, *nhigh;  // dynamic neighbours per body (k_neighbour_lists)
    ContactEvent* events;
    uint32_t event_capacity;
    uint32_t *rcount, *roff, *blist;  // per-body flattened contact rows (bit 31: second body)
    uint32_t* bother;                 // the other body of each flattened row
    uint32_t *mem_count, *mem_off, *mem_cursor, *mem_list;
    // joints
    Joint* joints;
    JointState* jstate;
    JointRow* jrows;  // 18 per joint
    uint32_t* dis_keys;    // sorted (min<<32|max) keys of collision-disabling joints
    uint32_t* dis_joint;   // the joint of each key (a pair may have several)
    uint32_t n_dis;
    // fixed collision groups: fixed, collision-disabling joints (ascending)
    // and each body's group root, rebuilt every tick from the joints' state
    uint32_t* fixed_list;
    uint32_t* fixed_root;
    uint32_t n_fixed;
    // hinge joints (ascending index) grouped by scene: segment k is
    // hinge_list[hinge_seg[k] .. hinge_seg[k+1]); scenes share no bodies
    uint32_t* hinge_list;
    uint32_t* hinge_seg;
    uint32_t n_hinge_segs;
    // scratch for scans
    uint64_t* scan_tmp;
    uint32_t* scan_tmp32;
    Counters* ctr;
};

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ uint32_t grid_stride_begin() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint32_t grid_stride() { return gridDim.x * blockDim.x; }

// Grid barrier for cooperative launches: arrive on a counter, the last block
// bumps the generation. Waits are bounded by `spins` polls (about 2^26 by
// default, seconds); a timeout latches kStBarrierTimeout and the caller
// abandons the tick: every later cooperative kernel of the tick returns at
// once, and the host reports the status.
constexpr uint32_t kDefaultBarrierSpins = 1u << 26;
__device__ __forceinline__ bool grid_sync(Counters* c, uint32_t spins_limit) {
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        ok = 1;
        volatile uint32_t* gen = &c->bar_gen;
        uint32_t g = *gen;
        __threadfence();
        uint32_t arrived = atomicAdd(&c->bar_count, 1u);
        if (arrived == gridDim.x - 1) {
            c->bar_count = 0;
            __threadfence();
            atomicAdd(&c->bar_gen, 1u);
        } else {
            uint32_t spins = 0;
            while (*gen == g) {
                if (++spins > spins_limit) {
                    atomicOr(&c->status, kStBarrierTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Host-side stage launchers (defined in the .cu files).
void launch_broadphase(const Dev& d, cudaStream_t s);
void launch_scene_budgets(const Dev& d, const StepParams& sp, cudaStream_t s);
__device__ __forceinline__ bool batched(const Dev& d) { return d.n_scenes > 1; }
void launch_narrowphase(const Dev& d, const StepParams& sp, cudaStream_t s);
// Per-body hinge contact frames of the tick (worlds with joints) and the
// triangle-mesh narrowphase over the candidates the face path left to it.
void launch_hinge_frames(const Dev& d, cudaStream_t s);
void launch_mesh_narrowphase(const Dev& d, const StepParams& sp, cudaStream_t s);
// Hinge contact frame flags (d.frame[i].w bits).
constexpr uint32_t kFramePresent = 1u, kFrameAxial = 2u, kFrameFixedMember = 4u, kFrameStatic = 8u,
                   kFrameAxialRotation = 16u;
// rigid_guided_pair (geometry.slang:373-377): a body guided along a static
// rail meets a static body.
__host__ __device__ __forceinline__ bool frames_guided(uint32_t fa, uint32_t fb) {
    return ((fa & kFrameAxial) && (fb & kFrameStatic)) || ((fb & kFrameAxial) && (fa & kFrameStatic));
}
void launch_prepare(const Dev& d, const StepParams& sp, cudaStream_t s);
void launch_graph(const Dev& d, const StepParams& sp, cudaStream_t s, int coop_blocks);
struct SolveBuffers { float4 *ox, *oq, *ov, *ow; };
void launch_integrate(const Dev& d, const StepParams& sp, cudaStream_t s, const SolveBuffers& o);
void launch_solve_all(const Dev& d, const StepParams& sp, cudaStream_t s, const int* coop_blocks,
                      const SolveBuffers& o);
void launch_body_constants(const Dev& d, const float4* lo, const float4* hi, const float4* sph, cudaStream_t s);
void launch_finish(const Dev& d, const StepParams& sp, cudaStream_t s);
void scan_u32(const uint32_t* in, uint32_t* out, const uint32_t* count_ptr, uint32_t capacity, uint32_t* total,
              uint32_t* tmp, cudaStream_t s);
void scan_u64(const uint64_t* in, uint64_t* out, const uint32_t* count_ptr, uint32_t capacity, uint64_t* tmp,
              cudaStream_t s);
int coop_blocks_for(const void* kernel, int threads, size_t smem);
// Stage timing for diagnosis: records a CUDA event named `stage` when a
// profiled step is being enqueued (never during graph capture).
void prof_mark(cudaStream_t s, const char* stage);
// Kernels enqueued by this library since the last reset (all stages).
extern unsigned long long g_kernel_launches;
// Launch ledger of the tick being enqueued on this thread (telemetry):
// dispatches and thread blocks per work phase, in the reference's phase
// order (boundary, predict, index, candidates, domain, coupling, commit).
constexpr int kPhases = 7;
enum : int { kPhBoundary, kPhPredict, kPhIndex, kPhCandidates, kPhDomain, kPhCoupling, kPhCommit };
struct LaunchLedger {
    unsigned long long dispatches[kPhases];
    unsigned long long workgroups[kPhases];
};
extern thread_local LaunchLedger* g_ledger;
extern thread_local int g_phase;
inline void set_phase(int phase) { g_phase = phase; }
inline void note_launch(unsigned long long blocks) {
    ++g_kernel_launches;
    if (g_ledger) {
        ++g_ledger->dispatches[g_phase];
        g_ledger->workgroups[g_phase] += blocks;
    }
}
// Dominant-kernel timing: brackets each solve launch with CUDA events when on.
void solve_timer_begin(cudaStream_t s);
void solve_timer_end(cudaStream_t s);
// Cooperative solve kernel variants (threads per CTA) and their smem. Each
// has a build per feature set: bit 0 the world has joints, bit 1 the
// body-per-thread sweep (policy 4) is compiled in.
constexpr int kFeatJoints = 1;
constexpr int kFeatThread = 2;
constexpr int kSolveFeatures = 4;
struct SolveVariant {
    const void* ptr[kSolveFeatures];    // the tick's kernel
    const void* timed[kSolveFeatures];  // the same with per-colour timestamps (profiling)
    int threads;
    size_t smem;
};
constexpr uint32_t kSolveVariants = 5;
constexpr uint32_t kStagedFirst = 3;  // variants 3, 4: the staged solve with fused duals (512, 384 threads)
const SolveVariant& solve_variant(uint32_t v);
// The feature set a world's launches use.
inline int solve_features(const Dev& d) { return (d.nj ? kFeatJoints : 0) | (d.solve_policy == 4 ? kFeatThread : 0); }
// Group-per-body builds, one translation unit per CTA size.
SolveVariant solve_group_variant_512();
SolveVariant solve_group_variant_384();
SolveVariant solve_group_variant_256();
void launch_contact_jacobians(const Dev& d, uint32_t phase, float dt, cudaStream_t s);
// Sparse per-body record writes staged in io_index / io_rec (kind 0: inputs,
// 1: kinematic targets, 2: states), and AoS state packing into `dst`.
void launch_scatter_records(const Dev& d, uint32_t kind, uint32_t count, cudaStream_t s);
void launch_unpack_states(const Dev& d, uint32_t count, const float* src, cudaStream_t s);
void launch_pack_states(const Dev& d, uint32_t first, uint32_t count, float* dst, cudaStream_t s);
extern const void* color_kernel_ptr;
// Learned warm start (pmb_mlp.cu).
struct MlpMeta;
size_t mlp_smem_bytes();
int mlp_configure_kernels();
uint32_t mlp_grid(uint32_t tiles);
void launch_mlp_images(const float* params, uint8_t* img, cudaStream_t s);
void launch_mlp_features(const Dev& d, const StepParams& sp, uint8_t* x, MlpMeta* meta, cudaStream_t s);
void launch_mlp_targets(const Dev& d, MlpMeta* meta, cudaStream_t s);
void launch_mlp_pack_rows(const float* feat, const float* y, const float* w, uint32_t n, uint8_t* x, MlpMeta* meta,
                          uint32_t tiles, cudaStream_t s);
void launch_mlp_tiles(bool train, const uint8_t* x, const MlpMeta* meta, const uint8_t* img, uint32_t rows,
                      uint32_t tiles, const uint32_t* rows_ptr, float* out, float* partial, uint32_t* status,
                      uint32_t status_bit, uint32_t grid, cudaStream_t s);
void launch_mlp_apply(const Dev& d, const MlpMeta* meta, const float* out, uint32_t mode, const float* gate,
                      cudaStream_t s);
void launch_mlp_reduce_adam(const float* partial, uint32_t parts, float* grad, float* params, float* m, float* v,
                            float lr, float b1, float b2, float c1, float c2, float eps, float* gate, cudaStream_t s);

inline uint32_t blocks_for(uint32_t n, int threads = kBlock) {
    uint32_t b = (n + threads - 1) / threads;
    return b == 0 ? 1 : b;
}
// Grid for a grid-stride kernel sized by a capacity (most of which is
// usually unused): at most enough blocks to fill a B200's 148 SMs.
constexpr uint32_t kGridSms = 148;
inline uint32_t cap_blocks(size_t cap, int threads = kBlock) {
    const uint32_t full = kGridSms * (2048u / uint32_t(threads));
    const uint32_t need = blocks_for(uint32_t(cap < 0xffffffffu ? cap : 0xffffffffu), threads);
    return need < full ? need : full;
}

}  // namespace pmb

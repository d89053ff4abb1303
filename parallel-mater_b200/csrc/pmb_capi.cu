// SPDX-License-Identifier: MIT
// C ABI of the pmb200 core (include/pmb200_core.h): world allocation and
// upload, the tick sequence, graph capture, inspection and snapshots.
#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/pmb200_core.h"
#include "pmb_joint.cuh"
#include "pmb_mesh.hpp"
#include "pmb_mlp.cuh"

namespace pmb {
__global__ void k_math_eval(uint32_t kind, uint32_t count, const float* in, float* out);

struct Prof {
    bool on{};
    std::vector<cudaEvent_t> events;
    std::vector<const char*> names;
};
static Prof g_prof;
unsigned long long g_kernel_launches = 0;
thread_local LaunchLedger* g_ledger = nullptr;
thread_local int g_phase = 0;

void prof_mark(cudaStream_t s, const char* stage) {
    if (!g_prof.on) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, s);
    g_prof.events.push_back(e);
    g_prof.names.push_back(stage);
}

struct SolveTimer {
    bool on{};
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pairs;
};
static SolveTimer g_timer;

void solve_timer_begin(cudaStream_t s) {
    if (!g_timer.on) return;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
    g_timer.pairs.push_back({a, b});
}
void solve_timer_end(cudaStream_t s) {
    if (!g_timer.on || g_timer.pairs.empty()) return;
    cudaEventRecord(g_timer.pairs.back().second, s);
}

int coop_blocks_for(const void* kernel, int threads, size_t smem) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
    return std::max(1, per) * sms;
}
}  // namespace pmb

using namespace pmb;

struct pmb_world {
    int device{};
    cudaStream_t stream{};
    bool own_stream{};
    Dev d{};
    SolveBuffers out{};
    std::vector<void*> allocs;
    std::vector<std::pair<void*, size_t>> dynamic_state;  // snapshot set
    // Caller-bound memory (persistent, scratch): when set, every device array
    // is carved from it and nothing is allocated. counting: only sum sizes.
    char* arena[2]{};
    size_t arena_size[2]{}, arena_used[2]{};
    bool counting{};
    std::vector<pmb_joint> host_joints;
    std::vector<void*> snapshot;
    int coop_solve[kSolveVariants]{}, coop_color{};
    cudaGraphExec_t graph{};
    uint32_t step_parity{}, snapshot_parity{};
    Counters host_ctr{};
    LaunchLedger ledger{};          // launches of the latest enqueued tick
    uint64_t ticks_enqueued{};
    // Learned warm start (allocated by pmb_world_mlp_attach).
    struct Mlp {
        bool attached{}, train{};
        float lr{1e-3f};
        uint32_t steps_per_tick{1}, grid{};
        uint64_t adam_t{};
        float *params{}, *m{}, *v{}, *grad{}, *partial{}, *gate{}, *out{};
        uint32_t mode{3};
        uint8_t *img{}, *x{};
        MlpMeta* meta{};
        std::vector<void*> allocs;
    } mlp;
};

namespace {

enum { kPersistent = 0, kScratch = 1 };
constexpr size_t kArenaAlign = 256;

template <class T> int alloc(pmb_world* w, T*& p, size_t count, int cls) {
    p = nullptr;
    if (count == 0) count = 1;
    const size_t bytes = sizeof(T) * count;
    const size_t padded = (bytes + kArenaAlign - 1) & ~(kArenaAlign - 1);
    if (w->counting) {
        w->arena_used[cls] += padded;
        return PMB_SUCCESS;
    }
    if (w->arena[cls]) {
        if (w->arena_used[cls] + padded > w->arena_size[cls]) return PMB_ERROR_CAPACITY_EXCEEDED;
        p = reinterpret_cast<T*>(w->arena[cls] + w->arena_used[cls]);
        w->arena_used[cls] += padded;
    } else {
        if (cudaMalloc(reinterpret_cast<void**>(&p), bytes) != cudaSuccess) return PMB_ERROR_OUT_OF_DEVICE_MEMORY;
        w->allocs.push_back(p);
    }
    cudaMemsetAsync(p, 0, bytes, w->stream);
    return PMB_SUCCESS;
}
// Persistent arrays that make up the dynamic state (snapshot set).
template <class T> int alloc_state(pmb_world* w, T*& p, size_t count) {
    int r = alloc(w, p, count, kPersistent);
    if (r == PMB_SUCCESS && !w->counting) w->dynamic_state.push_back({p, sizeof(T) * (count ? count : 1)});
    return r;
}

uint32_t next_pow2(uint32_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

StepParams params_from(const pmb_step_desc& s) {
    StepParams p{};
    p.dt = s.dt;
    p.gx = s.gravity[0];
    p.gy = s.gravity[1];
    p.gz = s.gravity[2];
    p.realtime = s.profile == 1 ? 1u : 0u;
    p.requested = s.requested_iterations;
    p.budget_request = p.realtime ? 8u : (s.requested_iterations ? s.requested_iterations : s.base_iterations);
    p.tolerance = s.residual_tolerance;
    p.max_iterations = s.max_iterations;
    p.warm_start = s.warm_start;
    p.collect_events = s.collect_events;
    p.residual_norm = s.residual_norm;
    return p;
}

__global__ void k_reset_counters(Counters* c) {
    // bar_gen is left alone: it only ever increases.
    uint32_t* w = reinterpret_cast<uint32_t*>(c);
    const uint32_t words = sizeof(Counters) / 4;
    const uint32_t skip = offsetof(Counters, bar_gen) / 4;
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x)
        if (i != skip) w[i] = 0;
}

void enqueue_step(pmb_world* w, const StepParams& sp) {
    cudaStream_t s = w->stream;
    Dev& d = w->d;
    w->ledger = LaunchLedger{};
    g_ledger = &w->ledger;
    set_phase(kPhBoundary);
    k_reset_counters<<<1, 256, 0, s>>>(d.ctr);
    note_launch(1);
    set_phase(kPhPredict);
    launch_integrate(d, sp, s, w->out);
    set_phase(kPhIndex);
    launch_broadphase(d, s);  // switches to the candidate phase for the query
    launch_hinge_frames(d, s);
    launch_narrowphase(d, sp, s);
    set_phase(kPhDomain);
    launch_prepare(d, sp, s);
    auto& mlp = w->mlp;
    const bool learned = mlp.attached && sp.warm_start == 1;
    if (mlp.attached && (learned || mlp.train)) launch_mlp_features(d, sp, mlp.x, mlp.meta, s);
    if (learned) {
        launch_mlp_tiles(false, mlp.x, mlp.meta, mlp.img, 0, 0, &d.ctr->n_contacts, mlp.out, nullptr, &d.ctr->status,
                         kStBarrierTimeout, mlp.grid, s);
        launch_mlp_apply(d, mlp.meta, mlp.out, mlp.mode, mlp.gate, s);
    }
    prof_mark(s, "mlp features+inference");
    launch_graph(d, sp, s, w->coop_color);
    launch_scene_budgets(d, sp, s);
    launch_solve_all(d, sp, s, w->coop_solve, w->out);
    set_phase(kPhDomain);
    if (mlp.attached && mlp.train) {
        // Online training on this tick's converged normal rows.
        launch_mlp_targets(d, mlp.meta, s);
        for (uint32_t k = 0; k < mlp.steps_per_tick; ++k) {
            launch_mlp_tiles(true, mlp.x, mlp.meta, mlp.img, 0, 0, &d.ctr->n_contacts, nullptr, mlp.partial,
                             &d.ctr->status, kStBarrierTimeout, mlp.grid, s);
            ++mlp.adam_t;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.0f - std::pow(b1, float(mlp.adam_t)), c2 = 1.0f - std::pow(b2, float(mlp.adam_t));
            // The gate follows the first step of each tick: its loss is
            // measured before the model has seen this tick's targets.
            launch_mlp_reduce_adam(mlp.partial, mlp.grid, mlp.grad, mlp.params, mlp.m, mlp.v, mlp.lr, b1, b2, c1, c2,
                                   1e-8f, k == 0 ? mlp.gate : nullptr, s);
            launch_mlp_images(mlp.params, mlp.img, s);
        }
        prof_mark(s, "mlp training");
    }
    g_ledger = nullptr;
    ++w->ticks_enqueued;
    // The cache written this tick is read by the next one.
    std::swap(d.sv_code, d.out_code);
    std::swap(d.sv_off, d.out_off);
    std::swap(d.sv_cnt, d.out_cnt);
    std::swap(d.sv_n_pairs, d.out_n_pairs);
    std::swap(d.sv_local, d.out_local);
    std::swap(d.sv_normal, d.out_normal);
    std::swap(d.sv_fimp, d.out_fimp);
    std::swap(d.sv_lam, d.out_lam);
    std::swap(d.sv_pen, d.out_pen);
    std::swap(d.sv_aa, d.out_aa);
    std::swap(d.sv_ab, d.out_ab);
    std::swap(d.sv_dt, d.out_dt);
    w->step_parity ^= 1u;
}

void swap_cache(pmb_world* w) {
    Dev& d = w->d;
    std::swap(d.sv_code, d.out_code);
    std::swap(d.sv_off, d.out_off);
    std::swap(d.sv_cnt, d.out_cnt);
    std::swap(d.sv_n_pairs, d.out_n_pairs);
    std::swap(d.sv_local, d.out_local);
    std::swap(d.sv_normal, d.out_normal);
    std::swap(d.sv_fimp, d.out_fimp);
    std::swap(d.sv_lam, d.out_lam);
    std::swap(d.sv_pen, d.out_pen);
    std::swap(d.sv_aa, d.out_aa);
    std::swap(d.sv_ab, d.out_ab);
    std::swap(d.sv_dt, d.out_dt);
    w->step_parity ^= 1u;
}

int check(cudaError_t e) {
    if (e == cudaSuccess) return PMB_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return PMB_ERROR_OUT_OF_DEVICE_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return PMB_ERROR_NO_DEVICE;
    std::fprintf(stderr, "pmb200: CUDA error %s\n", cudaGetErrorString(e));
    return PMB_ERROR_DEVICE_LOST;
}

void fill_stats(const Counters& c, pmb_step_stats* s) {
    s->candidate_pairs = c.n_cand;
    s->active_pairs = c.n_act;
    s->contacts = c.n_contacts;
    s->colors = c.colors;
    s->islands = c.islands;
    s->iterations = c.iterations;
    s->impact = c.impact;
    s->status = c.status;
    s->residual = c.residual;
    s->residual_max = c.residual_max;
    s->residual_over = c.residual_over;
}

// The float whose bits are u (index fields packed into float4 records).
float host_bits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

struct Sizes {
    uint32_t n, nm, nj, scenes;
    size_t verts, planes, dis, hinges, hinge_segs;
    uint32_t cap_cand, cap_pair, cap_contact;
    uint32_t events;
    size_t fixed;  // fixed collision-disabling joints
    size_t bvh_nodes, shell_normals;
};
struct Extra {
    float4 *lo, *hi, *sph;  // mesh bounds, read once at creation
    uint64_t* dis;
};

// The world's device layout. The same sequence runs in counting mode to size
// caller-bound memory, so every array of a world comes from here.
int allocate_world(pmb_world* w, Dev& d, const Sizes& z, Extra& e) {
    const uint32_t n = z.n, nm = z.nm, nj = z.nj;
    const uint32_t grid_size = next_pow2(std::max(2u * n, 1024u));
    const size_t cap_cand = z.cap_cand, cap_pair = z.cap_pair, cap_contact = z.cap_contact;
    int r = PMB_SUCCESS;
#define ALLOCP(p, c) if (r == PMB_SUCCESS) r = alloc(w, p, c, kPersistent)
#define ALLOC(p, c) if (r == PMB_SUCCESS) r = alloc(w, p, c, kScratch)
#define ALLOCS(p, c) if (r == PMB_SUCCESS) r = alloc_state(w, p, c)
    ALLOCP(d.motion, n); ALLOCP(d.mesh, n); ALLOCP(d.p0, n); ALLOCP(d.p1, n); ALLOCP(d.p2, n);
    ALLOCP(d.expand, n); ALLOCP(d.rotb, n);
    ALLOCS(d.x, n); ALLOCS(d.q, n); ALLOCS(d.v, n); ALLOCS(d.w, n);
    ALLOC(d.tx, n); ALLOC(d.tq, n); ALLOC(d.tv, n); ALLOC(d.tw, n);
    ALLOC(w->out.ox, n); ALLOC(w->out.oq, n); ALLOC(w->out.ov, n); ALLOC(w->out.ow, n);
    ALLOCS(d.force, n); ALLOCS(d.torque, n); ALLOCS(d.lin_imp, n); ALLOCS(d.ang_imp, n);
    ALLOCS(d.tgt_x, n); ALLOCS(d.tgt_q, n);
    ALLOC(d.io_index, n); ALLOC(d.io_rec, 4 * size_t(n));
    ALLOC(d.warm_table, 2 * cap_contact);
    ALLOCP(d.m_vo, nm); ALLOCP(d.m_vc, nm); ALLOCP(d.m_to, nm); ALLOCP(d.m_tc, nm); ALLOCP(d.m_convex, nm);
    ALLOCP(d.m_verts, z.verts); ALLOCP(d.m_planes, z.planes);
    ALLOCP(d.m_solid, nm); ALLOCP(d.m_bo, nm); ALLOCP(d.m_so, nm); ALLOCP(d.m_lo, nm); ALLOCP(d.m_hi, nm);
    ALLOCP(d.m_bvh, 3 * z.bvh_nodes); ALLOCP(d.m_shell, z.shell_normals);
    ALLOCP(d.jb_off, nj ? size_t(n) + 1 : 0); ALLOCP(d.jb_list, 2 * size_t(nj)); ALLOC(d.frame, nj ? size_t(n) : 0);
    ALLOC(d.frame_prev, nj ? size_t(n) : 0);
    ALLOC(d.frame_guide, nj ? size_t(n) : 0); ALLOC(d.frame_anchor, nj ? size_t(n) : 0);
    ALLOC(d.np_mesh, cap_cand);
    d.cap_mesh = uint32_t(cap_pair);
    d.cap_mesh_leaves = d.cap_mesh_items = uint32_t(cap_contact);
    ALLOC(d.mp_leaves, cap_pair); ALLOC(d.mp_items, cap_pair); ALLOC(d.mp_flags, cap_pair);
    ALLOC(d.mp_leaf_off, cap_pair + 1); ALLOC(d.mp_item_off, cap_pair + 1);
    ALLOC(d.ml_rec, cap_contact); ALLOC(d.ml_item, cap_contact); ALLOC(d.ml_pair, cap_contact);
    ALLOC(d.mi_valid, cap_contact); ALLOC(d.mi_p, cap_contact); ALLOC(d.mi_n, cap_contact);
    ALLOC(d.dxl, n); ALLOC(d.dxa, n); ALLOC(d.dq, n); ALLOC(d.inA, n); ALLOC(d.inB, n);
    ALLOCS(d.prev_vel, n); ALLOCS(d.color, n);
    ALLOC(d.parent, n); ALLOC(d.impact, n); ALLOC(d.anchored, n); ALLOC(d.mean, n); ALLOC(d.island_end, n);
    ALLOC(d.lo, n); ALLOC(d.hi, n); ALLOC(d.is_large, n); ALLOC(d.large_list, n);
    ALLOC(d.bucket_count, grid_size + 1); ALLOC(d.bucket_off, grid_size + 1); ALLOC(d.bucket_cursor, grid_size);
    ALLOC(d.grid_body, n); ALLOC(d.grid_cell, n);
    ALLOC(d.cand_count, n + 1); ALLOC(d.cand_off, n + 1); ALLOC(d.cand_lane, kQueryLanes * size_t(n));
    ALLOC(d.cand_a, cap_cand); ALLOC(d.cand_b, cap_cand);
    ALLOC(d.np_count, cap_cand); ALLOC(d.np_scan, cap_cand + 1); ALLOC(d.np_stage, cap_cand);
    ALLOC(d.np_list, cap_cand); ALLOC(d.np_sat, cap_cand);
    ALLOC(d.st_n, cap_contact); ALLOC(d.st_p, cap_contact);
    ALLOC(d.act_a, cap_pair); ALLOC(d.act_b, cap_pair); ALLOC(d.act_code, cap_pair);
    ALLOC(d.act_off, cap_pair + 1); ALLOC(d.act_cnt, cap_pair); ALLOC(d.act_impact, cap_pair);
    ALLOC(d.c_pair, cap_contact); ALLOC(d.c_bodies, cap_contact); ALLOC(d.c_jac, 9 * cap_contact);
    ALLOC(d.c_n, cap_contact); ALLOC(d.c_p, cap_contact); ALLOC(d.c_e, cap_contact);
    ALLOC(d.c_aa, cap_contact); ALLOC(d.c_ab, cap_contact); ALLOC(d.c_lam, cap_contact);
    ALLOC(d.c_pen, cap_contact); ALLOC(d.c_accf, cap_contact); ALLOC(d.c_foff, cap_contact);
    ALLOC(d.c_mub, cap_contact);
    for (int side = 0; side < 2; ++side) {
        uint64_t** code = side ? &d.out_code : &d.sv_code;
        uint32_t** off = side ? &d.out_off : &d.sv_off;
        uint32_t** cnt = side ? &d.out_cnt : &d.sv_cnt;
        uint32_t** np = side ? &d.out_n_pairs : &d.sv_n_pairs;
        float4** f[7] = {side ? &d.out_local : &d.sv_local, side ? &d.out_normal : &d.sv_normal,
                         side ? &d.out_fimp : &d.sv_fimp, side ? &d.out_lam : &d.sv_lam,
                         side ? &d.out_pen : &d.sv_pen, side ? &d.out_aa : &d.sv_aa, side ? &d.out_ab : &d.sv_ab};
        float** dtp = side ? &d.out_dt : &d.sv_dt;
        ALLOCS(*code, cap_pair); ALLOCS(*off, cap_pair); ALLOCS(*cnt, cap_pair); ALLOCS(*np, 1);
        for (auto* p : f) ALLOCS(*p, cap_contact);
        ALLOCS(*dtp, 1);
    }
    ALLOC(d.deg, n); ALLOC(d.inc_off, n + 1); ALLOC(d.inc_cursor, n); ALLOC(d.inc_list, 2 * cap_pair);
    ALLOC(d.jdeg, n); ALLOC(d.jinc_off, n + 1); ALLOC(d.jinc_cursor, n); ALLOC(d.jinc_list, 2 * size_t(nj) + 2);
    ALLOC(d.corder, n); ALLOC(d.crec, n); ALLOC(d.cdirty, 2 * size_t(n));
    ALLOC(d.nbr, 2 * cap_pair + 2 * size_t(nj) + 2); ALLOC(d.nlow, n); ALLOC(d.nhigh, n);
    ALLOCP(d.events, z.events);
    ALLOC(d.rcount, n); ALLOC(d.roff, n + 1); ALLOC(d.blist, 2 * cap_contact); ALLOC(d.bother, 2 * cap_contact);
    ALLOCP(d.joints, nj); ALLOCS(d.jstate, nj); ALLOCS(d.jrows, size_t(nj) * 18);
    ALLOCP(d.hinge_list, z.hinges); ALLOCP(d.hinge_seg, z.hinge_segs + 1);
    {
        // Scan scratch: one slot per 2048-element tile of the longest scan plus the total.
        size_t longest = std::max<size_t>({cap_cand, grid_size, n, cap_pair});
        size_t tiles = (longest + 2047) / 2048 + 2;
        ALLOC(d.scan_tmp, tiles); ALLOC(d.scan_tmp32, tiles);
    }
    ALLOCP(d.ctr, 1);
    ALLOC(e.lo, nm); ALLOC(e.hi, nm); ALLOC(e.sph, nm);
    ALLOCP(e.dis, z.dis); ALLOCP(d.dis_joint, z.dis);
    ALLOCP(d.fixed_list, z.fixed); ALLOC(d.fixed_root, z.fixed ? size_t(n) : 0);
    if (z.scenes > 1) {
        const uint32_t ns = z.scenes;
        ALLOCP(d.scene_of, n); ALLOCP(d.scene_body_off, ns + 1); ALLOCP(d.scene_iters, ns); ALLOCP(d.scene_jiters, ns);
        ALLOC(d.scene_large_count, ns + 1); ALLOC(d.scene_large_off, ns + 1); ALLOC(d.scene_large_cursor, ns);
        ALLOC(d.scene_large_list, n); ALLOC(d.scene_budget, ns);
        ALLOC(d.scene_res_sq, ns); ALLOC(d.scene_res_mx, ns); ALLOC(d.scene_res_n, ns); ALLOC(d.scene_hs, ns);
    }
#undef ALLOCP
#undef ALLOC
#undef ALLOCS
    return r;
}

}  // namespace

namespace {
// Deterministic initial weights: He-uniform hidden layers from a counter-based
// hash of (seed, index); zero output layer (the predictor starts out as the
// plain warm start), zero biases and padding.
float init_uniform(uint32_t seed, uint32_t i) {
    uint64_t z = (uint64_t(seed) << 32) ^ (uint64_t(i) * 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return float((z >> 40) * (1.0 / 16777216.0)) * 2.0f - 1.0f;
}
void init_params(uint32_t seed, std::vector<float>& p) {
    p.assign(kMlpParams, 0.0f);
    const float a1 = std::sqrt(6.0f / float(kMlpFeatures)), a2 = std::sqrt(6.0f / float(kMlpHidden)), a3 = 0.0f;
    for (uint32_t j = 0; j < kMlpHidden; ++j) {
        for (uint32_t f = 0; f < kMlpFeatures; ++f)
            p[kMlpW1 + j * kMlpIn + f] = a1 * init_uniform(seed, kMlpW1 + j * kMlpIn + f);
        for (uint32_t k = 0; k < kMlpHidden; ++k)
            p[kMlpW2 + j * kMlpHiddenK + k] = a2 * init_uniform(seed, kMlpW2 + j * kMlpHiddenK + k);
    }
    for (uint32_t o = 0; o < kMlpOut; ++o)
        for (uint32_t k = 0; k < kMlpHidden; ++k)
            p[kMlpW3 + o * kMlpHiddenK + k] = a3 * init_uniform(seed, kMlpW3 + o * kMlpHiddenK + k);
}
template <class T> int mlp_alloc(pmb_world* w, T*& p, size_t count) {
    p = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess)
        return PMB_ERROR_OUT_OF_DEVICE_MEMORY;
    w->mlp.allocs.push_back(p);
    cudaMemsetAsync(p, 0, sizeof(T) * std::max<size_t>(count, 1), w->stream);
    return PMB_SUCCESS;
}
}  // namespace

extern "C" {

int pmb_world_create(const pmb_world_desc* desc, pmb_world** out) {
    if (!desc || !out || desc->body_count == 0 || !desc->bodies || !desc->states || desc->mesh_count == 0)
        return PMB_ERROR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PMB_ERROR_NO_DEVICE;
    if (desc->device < 0 || desc->device >= ndev) return PMB_ERROR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < desc->body_count; ++i)
        if (desc->bodies[i].mesh >= desc->mesh_count || desc->bodies[i].motion > 2) return PMB_ERROR_INVALID_ARGUMENT;
    for (uint32_t j = 0; j < desc->joint_count; ++j)
        if (desc->joints[j].type > 7 || desc->joints[j].body_a >= desc->body_count ||
            desc->joints[j].body_b >= desc->body_count)
            return PMB_ERROR_INVALID_ARGUMENT;
    if (desc->scene_count > 1) {
        if (!desc->body_scene || desc->scene_count > desc->body_count) return PMB_ERROR_INVALID_ARGUMENT;
        for (uint32_t i = 0; i < desc->body_count; ++i)
            if (desc->body_scene[i] >= desc->scene_count || (i && desc->body_scene[i] < desc->body_scene[i - 1]))
                return PMB_ERROR_INVALID_ARGUMENT;
        for (uint32_t j = 0; j < desc->joint_count; ++j)
            if (desc->body_scene[desc->joints[j].body_a] != desc->body_scene[desc->joints[j].body_b])
                return PMB_ERROR_INVALID_ARGUMENT;
    }
    if ((desc->persistent_memory == nullptr) != (desc->scratch_memory == nullptr) ||
        (reinterpret_cast<uintptr_t>(desc->persistent_memory) % kArenaAlign) != 0 ||
        (reinterpret_cast<uintptr_t>(desc->scratch_memory) % kArenaAlign) != 0)
        return PMB_ERROR_INVALID_ARGUMENT;
    pmb_world* w = new (std::nothrow) pmb_world;
    if (!w) return PMB_ERROR_OUT_OF_DEVICE_MEMORY;
    w->device = desc->device;
    w->arena[kPersistent] = static_cast<char*>(desc->persistent_memory);
    w->arena_size[kPersistent] = size_t(desc->persistent_bytes);
    w->arena[kScratch] = static_cast<char*>(desc->scratch_memory);
    w->arena_size[kScratch] = size_t(desc->scratch_bytes);
    if (desc->joint_count) w->host_joints.assign(desc->joints, desc->joints + desc->joint_count);
    cudaSetDevice(w->device);
    if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete w;
        return PMB_ERROR_NO_DEVICE;
    }
    w->own_stream = true;
    Dev& d = w->d;
    const uint32_t n = desc->body_count, nm = desc->mesh_count, nj = desc->joint_count;
    d.n = n;
    d.nm = nm;
    d.nj = nj;
    d.cap_cand = desc->candidate_capacity ? desc->candidate_capacity : 64u * n + 4096u;
    d.cap_pair = desc->pair_capacity ? desc->pair_capacity : 24u * n + 1024u;
    d.cap_contact = desc->contact_capacity ? desc->contact_capacity : 64u * n + 4096u;
    d.cap_stage = d.cap_contact;
    d.grid_size = next_pow2(std::max(2u * n, 1024u));

    // ---- meshes (host preparation, then upload)
    std::vector<uint32_t> m_vo(nm), m_vc(nm), m_to(nm), m_tc(nm), m_convex(nm), m_solid(nm), m_bo(nm), m_so(nm);
    std::vector<float4> verts, planes, mlo(nm), mhi(nm), msph(nm), bvh, shell;
    for (uint32_t m = 0; m < nm; ++m) {
        const uint32_t v0 = desc->vertex_offsets[m], v1 = desc->vertex_offsets[m + 1];
        const uint32_t i0 = desc->index_offsets[m], i1 = desc->index_offsets[m + 1];
        if (v1 <= v0 || i1 < i0 || (i1 - i0) % 3) {
            pmb_world_destroy(w);
            return PMB_ERROR_INVALID_ARGUMENT;
        }
        for (uint32_t k = i0; k < i1; ++k)
            if (desc->indices[k] >= v1 - v0) {
                pmb_world_destroy(w);
                return PMB_ERROR_INVALID_ARGUMENT;
            }
        PreparedMesh pm = prepare_mesh(desc->vertices + 3 * size_t(v0), v1 - v0, desc->indices + i0, i1 - i0);
        const uint32_t nt = (i1 - i0) / 3;
        m_vo[m] = uint32_t(verts.size());
        m_vc[m] = v1 - v0;
        for (uint32_t k = v0; k < v1; ++k)
            verts.push_back(make_float4(desc->vertices[3 * k], desc->vertices[3 * k + 1], desc->vertices[3 * k + 2], 0));
        m_to[m] = uint32_t(planes.size());
        m_tc[m] = nt;
        m_convex[m] = pm.convex && (i1 - i0) <= 96 ? 1u : 0u;
        m_solid[m] = pm.convex ? 1u : 0u;
        m_bo[m] = uint32_t(bvh.size() / 3);
        for (const BvhNodeHost& nd : pm.bvh) {
            bvh.push_back(make_float4(nd.lo[0], nd.lo[1], nd.lo[2], host_bits(nd.first)));
            bvh.push_back(make_float4(nd.hi[0], nd.hi[1], nd.hi[2], host_bits(nd.count)));
            bvh.push_back(make_float4(host_bits(nd.left), host_bits(nd.right), 0, 0));
        }
        m_so[m] = pm.shell.empty() ? kInvalid : uint32_t(shell.size());
        for (const auto& sn : pm.shell) shell.push_back(make_float4(sn[0], sn[1], sn[2], 0));
        for (uint32_t t = 0; t < nt; ++t)
            planes.push_back(pm.convex ? make_float4(pm.planes[t][0], pm.planes[t][1], pm.planes[t][2], pm.planes[t][3])
                                       : make_float4(0, 0, 0, 0));
        for (uint32_t t = 0; t < nt; ++t) {
            float4 pk;
            uint32_t tri[3] = {pm.indices[3 * t], pm.indices[3 * t + 1], pm.indices[3 * t + 2]};
            std::memcpy(&pk.x, &tri[0], 4);
            std::memcpy(&pk.y, &tri[1], 4);
            std::memcpy(&pk.z, &tri[2], 4);
            pk.w = 0;
            planes.push_back(pk);
        }
        mlo[m] = make_float4(pm.lo[0], pm.lo[1], pm.lo[2], 0);
        mhi[m] = make_float4(pm.hi[0], pm.hi[1], pm.hi[2], 0);
        msph[m] = make_float4(pm.center[0], pm.center[1], pm.center[2], pm.radius);
    }

    // Collision-disabling joints as (body pair key, joint) sorted by key then
    // joint; a pair is filtered while any of its joints is unbroken.
    std::vector<std::pair<uint64_t, uint32_t>> dis_entries;
    for (uint32_t j = 0; j < nj; ++j) {
        const pmb_joint& o = desc->joints[j];
        if (o.enabled && o.disable_collisions) {
            uint64_t a = std::min(o.body_a, o.body_b), b = std::max(o.body_a, o.body_b);
            dis_entries.push_back({(a << 32) | b, j});
        }
    }
    std::sort(dis_entries.begin(), dis_entries.end());
    // Fixed joints that disable collisions join their bodies' collision groups.
    std::vector<uint32_t> fixed_list;
    for (uint32_t j = 0; j < nj; ++j) {
        const pmb_joint& o = desc->joints[j];
        if (o.type == kFixed && o.enabled && o.disable_collisions && o.body_a < n && o.body_b < n)
            fixed_list.push_back(j);
    }
    std::vector<uint64_t> dis_keys(dis_entries.size());
    std::vector<uint32_t> dis_joint(dis_entries.size());
    for (size_t k = 0; k < dis_entries.size(); ++k) {
        dis_keys[k] = dis_entries[k].first;
        dis_joint[k] = dis_entries[k].second;
    }
    const uint32_t ns = desc->scene_count > 1 ? desc->scene_count : 0u;
    d.n_scenes = ns;
    // Hinge projection runs serially over hinge joints in index order; joints
    // of different scenes touch disjoint bodies, so each scene's hinges form
    // an independent segment.
    std::vector<uint32_t> hinge_list, hinge_seg;
    {
        std::vector<std::pair<uint32_t, uint32_t>> hs;
        for (uint32_t j = 0; j < nj; ++j)
            if (desc->joints[j].type == kHinge) {
                const uint32_t a = desc->joints[j].body_a;
                hs.push_back({ns > 1 && a < n ? desc->body_scene[a] : 0u, j});
            }
        std::stable_sort(hs.begin(), hs.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        for (size_t k = 0; k < hs.size(); ++k) {
            if (k == 0 || hs[k].first != hs[k - 1].first) hinge_seg.push_back(uint32_t(k));
            hinge_list.push_back(hs[k].second);
        }
        hinge_seg.push_back(uint32_t(hs.size()));
    }
    d.n_hinge_segs = uint32_t(hinge_seg.size() - 1);
    d.event_capacity = desc->event_capacity;
    const Sizes z{n, nm, nj, ns, verts.size(), planes.size(), dis_keys.size(), hinge_list.size(),
                  hinge_seg.size() - 1, d.cap_cand, d.cap_pair, d.cap_contact, desc->event_capacity,
                  fixed_list.size(), bvh.size() / 3, shell.size()};
    if (w->arena[kPersistent]) {
        // Bound memory must hold the whole layout before anything is carved.
        pmb_world probe;
        probe.counting = true;
        Extra ex{};
        allocate_world(&probe, probe.d, z, ex);
        if (probe.arena_used[kPersistent] > w->arena_size[kPersistent] ||
            probe.arena_used[kScratch] > w->arena_size[kScratch]) {
            pmb_world_destroy(w);
            return PMB_ERROR_CAPACITY_EXCEEDED;
        }
    }
    Extra ex{};
    int r = allocate_world(w, d, z, ex);
    float4 *dlo = ex.lo, *dhi = ex.hi, *dsph = ex.sph;
    uint64_t* dis = ex.dis;
    d.dis_keys = reinterpret_cast<uint32_t*>(dis);
    d.n_dis = uint32_t(dis_keys.size());
    d.n_fixed = uint32_t(fixed_list.size());
    if (r != PMB_SUCCESS) {
        pmb_world_destroy(w);
        return r;
    }
    // ---- upload
    std::vector<uint32_t> motion(n), mesh(n);
    std::vector<float4> p0(n), p1(n), p2(n), x(n), q(n), v(n), wv(n);
    for (uint32_t i = 0; i < n; ++i) {
        const pmb_body& b = desc->bodies[i];
        motion[i] = b.motion;
        mesh[i] = b.mesh;
        p0[i] = make_float4(b.inv_mass, b.inv_inertia[0], b.inv_inertia[1], b.inv_inertia[2]);
        p1[i] = make_float4(b.friction, b.restitution, b.linear_damping, b.angular_damping);
        p2[i] = make_float4(b.max_linear_speed, b.max_angular_speed, b.margin, 0.0f);
        const pmb_state& s = desc->states[i];
        Q4 qq = qnormalize(Q4{s.q[0], s.q[1], s.q[2], s.q[3]});
        x[i] = make_float4(s.x[0], s.x[1], s.x[2], 0);
        q[i] = f4(qq);
        v[i] = make_float4(s.v[0], s.v[1], s.v[2], 0);
        wv[i] = make_float4(s.w[0], s.w[1], s.w[2], 0);
    }
    cudaStream_t s = w->stream;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (bytes) cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    };
    up(d.motion, motion.data(), 4 * n);
    up(d.mesh, mesh.data(), 4 * n);
    up(d.p0, p0.data(), 16 * n);
    up(d.p1, p1.data(), 16 * n);
    up(d.p2, p2.data(), 16 * n);
    up(d.x, x.data(), 16 * n);
    up(d.q, q.data(), 16 * n);
    up(d.v, v.data(), 16 * n);
    up(d.w, wv.data(), 16 * n);
    up(d.m_vo, m_vo.data(), 4 * nm);
    up(d.m_vc, m_vc.data(), 4 * nm);
    up(d.m_to, m_to.data(), 4 * nm);
    up(d.m_tc, m_tc.data(), 4 * nm);
    up(d.m_convex, m_convex.data(), 4 * nm);
    up(d.m_verts, verts.data(), 16 * verts.size());
    up(d.m_planes, planes.data(), 16 * planes.size());
    up(dlo, mlo.data(), 16 * nm);
    up(dhi, mhi.data(), 16 * nm);
    up(dsph, msph.data(), 16 * nm);
    if (nj) up(d.joints, desc->joints, sizeof(Joint) * nj);
    up(d.hinge_list, hinge_list.data(), 4 * hinge_list.size());
    up(d.hinge_seg, hinge_seg.data(), 4 * hinge_seg.size());
    std::vector<uint32_t> scene_off, scene_iters;
    if (ns > 1) {
        scene_off.assign(ns + 1, 0);
        for (uint32_t i = 0; i < n; ++i) ++scene_off[desc->body_scene[i] + 1];
        for (uint32_t k = 0; k < ns; ++k) scene_off[k + 1] += scene_off[k];
        scene_iters.assign(ns, 0);
        if (desc->scene_iterations) scene_iters.assign(desc->scene_iterations, desc->scene_iterations + ns);
        up(d.scene_of, desc->body_scene, 4 * size_t(n));
        up(d.scene_body_off, scene_off.data(), 4 * size_t(ns + 1));
        up(d.scene_iters, scene_iters.data(), 4 * size_t(ns));
    }
    if (!dis_keys.empty()) {
        up(dis, dis_keys.data(), 8 * dis_keys.size());
        up(d.dis_joint, dis_joint.data(), 4 * dis_joint.size());
    }
    if (!fixed_list.empty()) up(d.fixed_list, fixed_list.data(), 4 * fixed_list.size());
    up(d.m_solid, m_solid.data(), 4 * size_t(nm));
    up(d.m_bo, m_bo.data(), 4 * size_t(nm));
    up(d.m_so, m_so.data(), 4 * size_t(nm));
    up(d.m_lo, mlo.data(), 16 * size_t(nm));
    up(d.m_hi, mhi.data(), 16 * size_t(nm));
    if (!bvh.empty()) up(d.m_bvh, bvh.data(), 16 * bvh.size());
    if (!shell.empty()) up(d.m_shell, shell.data(), 16 * shell.size());
    if (nj) {
        // Each body's joints in ascending index (a joint on one body twice
        // is listed once), for the per-tick hinge contact frames.
        std::vector<uint32_t> jb_off(n + 1, 0), jb_list;
        std::vector<std::vector<uint32_t>> by_body(n);
        for (uint32_t j = 0; j < nj; ++j) {
            const pmb_joint& o = desc->joints[j];
            if (o.body_a < n) by_body[o.body_a].push_back(j);
            if (o.body_b < n && o.body_b != o.body_a) by_body[o.body_b].push_back(j);
        }
        for (uint32_t i = 0; i < n; ++i) {
            jb_off[i] = uint32_t(jb_list.size());
            jb_list.insert(jb_list.end(), by_body[i].begin(), by_body[i].end());
        }
        jb_off[n] = uint32_t(jb_list.size());
        up(d.jb_off, jb_off.data(), 4 * size_t(n + 1));
        if (!jb_list.empty()) up(d.jb_list, jb_list.data(), 4 * jb_list.size());
    }
    std::vector<uint32_t> colors(n, kInvalid);
    up(d.color, colors.data(), 4 * n);
    launch_body_constants(d, dlo, dhi, dsph, s);
    // Bodies larger than 4x the median proxy extent are tested by brute force.
    std::vector<float> expand(n);
    cudaMemcpyAsync(expand.data(), d.expand, 4 * n, cudaMemcpyDeviceToHost, s);
    r = check(cudaStreamSynchronize(s));
    if (r != PMB_SUCCESS) {
        pmb_world_destroy(w);
        return r;
    }
    std::vector<float> sorted = expand;
    std::nth_element(sorted.begin(), sorted.begin() + n / 2, sorted.end());
    d.large_extent = 2.0f * sorted[n / 2] * 4.0f;
    d.solve_variant = 0;  // 512 threads: the fastest plan on a settled 65k-box pile
    d.solve_policy = 0;
    d.barrier_spins = kDefaultBarrierSpins;
    for (uint32_t v = 0; v < kSolveVariants; ++v) {
        const SolveVariant& sv = solve_variant(v);
        // One grid for every build of the variant: the smallest of their
        // co-resident counts.
        int blocks = 1 << 30;
        for (int f = 0; f < kSolveFeatures; ++f)
            for (const void* k : {sv.ptr[f], sv.timed[f]}) {
                cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sv.smem));
                blocks = std::min(blocks, coop_blocks_for(k, sv.threads, sv.smem));
            }
        w->coop_solve[v] = blocks;
    }
    {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        w->coop_color = std::min(coop_blocks_for(color_kernel_ptr, kColorThreads, 0), std::max(1, sms));
    }
    // A world in caller-bound memory allocates nothing, so it has no
    // snapshot storage (pmb_world_snapshot reports FEATURE_NOT_PRESENT).
    for (auto& p : w->dynamic_state) {
        if (w->arena[kPersistent]) break;
        void* snap = nullptr;
        if (cudaMalloc(&snap, p.second) != cudaSuccess) {
            pmb_world_destroy(w);
            return PMB_ERROR_OUT_OF_DEVICE_MEMORY;
        }
        w->snapshot.push_back(snap);
    }
    *out = w;
    return PMB_SUCCESS;
}

void pmb_world_destroy(pmb_world* w) {
    if (!w) return;
    cudaSetDevice(w->device);
    if (w->stream) cudaStreamSynchronize(w->stream);
    if (w->graph) cudaGraphExecDestroy(w->graph);
    for (void* p : w->allocs) cudaFree(p);
    for (void* p : w->snapshot) cudaFree(p);
    for (void* p : w->mlp.allocs) cudaFree(p);
    if (w->own_stream && w->stream) cudaStreamDestroy(w->stream);
    delete w;
}

int pmb_world_set_stream(pmb_world* w, void* stream) {
    if (!w) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    cudaStreamSynchronize(w->stream);
    if (w->own_stream) cudaStreamDestroy(w->stream);
    w->own_stream = false;
    w->stream = static_cast<cudaStream_t>(stream);
    return PMB_SUCCESS;
}

int pmb_world_step(pmb_world* w, const pmb_step_desc* step, pmb_step_stats* stats) {
    if (!w || !step || !(step->dt > 0.0f)) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    enqueue_step(w, params_from(*step));
    int r = check(cudaGetLastError());
    if (r != PMB_SUCCESS) return r;
    if (stats) return pmb_world_last_stats(w, stats);
    return PMB_SUCCESS;
}

int pmb_world_profile_step(pmb_world* w, const pmb_step_desc* step, char* report, uint32_t capacity) {
    if (!w || !step || !report || capacity == 0) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    g_prof = Prof{};
    g_prof.on = true;
    prof_mark(w->stream, "start");
    StepParams sp = params_from(*step);
    sp.debug_timing = 1;
    enqueue_step(w, sp);
    g_prof.on = false;
    int r = check(cudaStreamSynchronize(w->stream));
    std::string text;
    for (size_t k = 1; k < g_prof.events.size(); ++k) {
        float ms = 0;
        cudaEventElapsedTime(&ms, g_prof.events[k - 1], g_prof.events[k]);
        char line[160];
        std::snprintf(line, sizeof(line), "%-24s %9.3f ms\n", g_prof.names[k], ms);
        text += line;
    }
    for (auto e : g_prof.events) cudaEventDestroy(e);
    Counters hc;
    cudaMemcpy(&hc, w->d.ctr, sizeof(Counters), cudaMemcpyDeviceToHost);
    {
        char line[160];
        std::snprintf(line, sizeof(line),
                      "colour fixpoint rounds %u, candidates %u, narrowphase survivors %u, triangle-mesh pairs %u "
                      "(leaf pairs %u, triangle-pair items %u)\n",
                      hc.rounds, hc.n_cand, hc.n_surv, hc.n_mesh, hc.n_mesh_leaves, hc.n_mesh_items);
        text += line;
        std::snprintf(line, sizeof(line), "solve iteration 0 (us from kernel start): colours %u\n", hc.colors);
        text += line;
        for (uint32_t k = 0; k < 20; ++k) {
            if (!hc.dbg_work[k]) continue;
            std::snprintf(line, sizeof(line), "  %s %2u work-end %8.1f release %8.1f\n", k == 19 ? "dual  " : "colour", k,
                          (hc.dbg_work[k] - hc.dbg_start) * 1e-3, (hc.dbg_release[k] - hc.dbg_start) * 1e-3);
            text += line;
        }
        std::snprintf(line, sizeof(line), "  last colour body (max rn %u): stage %.1f gather %.1f solve %.1f crossing %.1f solve2 %.1f us\n",
                      hc.dbg_rn, hc.dbg_body[0] * 1e-3, hc.dbg_body[1] * 1e-3, hc.dbg_body[2] * 1e-3, hc.dbg_body[3] * 1e-3,
                      hc.dbg_body[4] * 1e-3);
        text += line;
        if (hc.dbg_sum[6] && w->d.solve_variant >= kStagedFirst) {
            const double nb = double(hc.dbg_sum[6]);
            std::snprintf(line, sizeof(line),
                          "  colour 0 mean over %.0f batches (mean rows %.1f): formation %.1f staging %.1f solve %.1f us\n",
                          nb, hc.dbg_sum[7] / nb, hc.dbg_sum[0] * 1e-3 / nb, hc.dbg_sum[1] * 1e-3 / nb,
                          hc.dbg_sum[2] * 1e-3 / nb);
            text += line;
        } else if (hc.dbg_sum[6]) {
            const double nb = double(hc.dbg_sum[6]);
            std::snprintf(line, sizeof(line),
                          "  colour 0 mean over %.0f bodies (mean rn %.1f): stage %.1f gather %.1f solve %.1f crossing "
                          "%.1f solve2 %.1f us\n",
                          nb, hc.dbg_sum[7] / nb, hc.dbg_sum[0] * 1e-3 / nb, hc.dbg_sum[1] * 1e-3 / nb,
                          hc.dbg_sum[2] * 1e-3 / nb, hc.dbg_sum[3] * 1e-3 / nb, hc.dbg_sum[4] * 1e-3 / nb);
            text += line;
        }
    }
    g_prof = Prof{};
    std::snprintf(report, capacity, "%s", text.c_str());
    return r;
}

int pmb_world_solve_timer(pmb_world* w, int enable, float* total_ms, uint32_t* launches) {
    if (!w) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    int r = check(cudaStreamSynchronize(w->stream));
    float total = 0.0f;
    for (auto& p : g_timer.pairs) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, p.first, p.second);
        total += ms;
        cudaEventDestroy(p.first);
        cudaEventDestroy(p.second);
    }
    if (total_ms) *total_ms = total;
    if (launches) *launches = uint32_t(g_timer.pairs.size());
    g_timer.pairs.clear();
    g_timer.on = enable != 0;
    return r;
}

int pmb_prepare_mesh(const float* vertices, uint32_t vertex_count, const uint32_t* indices, uint32_t index_count,
                     uint32_t* out_indices, float* out_planes, float* out_bounds, int* convex) {
    if (!vertices || !indices || vertex_count == 0 || index_count % 3 || !out_indices || !out_planes || !out_bounds ||
        !convex)
        return PMB_ERROR_INVALID_ARGUMENT;
    for (uint32_t k = 0; k < index_count; ++k)
        if (indices[k] >= vertex_count) return PMB_ERROR_INVALID_ARGUMENT;
    PreparedMesh pm = prepare_mesh(vertices, vertex_count, indices, index_count);
    std::memcpy(out_indices, pm.indices.data(), 4 * size_t(index_count));
    for (size_t t = 0; t < pm.planes.size(); ++t)
        for (int k = 0; k < 4; ++k) out_planes[4 * t + k] = pm.planes[t][k];
    const float b[10] = {pm.lo[0], pm.lo[1], pm.lo[2], pm.hi[0], pm.hi[1], pm.hi[2],
                         pm.center[0], pm.center[1], pm.center[2], pm.radius};
    std::memcpy(out_bounds, b, sizeof(b));
    *convex = pm.convex ? 1 : 0;
    return PMB_SUCCESS;
}

int pmb_kernel_launches(unsigned long long* count) {
    if (!count) return PMB_ERROR_INVALID_ARGUMENT;
    *count = g_kernel_launches;
    return PMB_SUCCESS;
}

int pmb_world_capture(pmb_world* w, const pmb_step_desc* step, uint32_t steps) {
    if (!w || !step || steps == 0 || (steps & 1u)) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    if (w->graph) {
        cudaGraphExecDestroy(w->graph);
        w->graph = nullptr;
    }
    StepParams sp = params_from(*step);
    cudaGraph_t g;
    int r = check(cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal));
    if (r != PMB_SUCCESS) return r;
    for (uint32_t k = 0; k < steps; ++k) enqueue_step(w, sp);
    r = check(cudaStreamEndCapture(w->stream, &g));
    if (r != PMB_SUCCESS) return r;
    r = check(cudaGraphInstantiate(&w->graph, g, 0));
    cudaGraphDestroy(g);
    return r;
}

int pmb_world_replay(pmb_world* w) {
    if (!w || !w->graph) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    return check(cudaGraphLaunch(w->graph, w->stream));
}

int pmb_world_last_stats(pmb_world* w, pmb_step_stats* out) {
    if (!w || !out) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    cudaMemcpyAsync(&w->host_ctr, w->d.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, w->stream);
    int r = check(cudaStreamSynchronize(w->stream));
    if (r != PMB_SUCCESS) return r;
    fill_stats(w->host_ctr, out);
    return PMB_SUCCESS;
}

// Whole-world state transfer through the record staging buffer (64 B per
// body): one packing kernel and one copy each way, straight from or into the
// caller's host memory (pinned memory makes both copies DMA transfers).
int pmb_world_get_states(pmb_world* w, pmb_state* out) {
    if (!w || !out) return PMB_ERROR_INVALID_ARGUMENT;
    static_assert(sizeof(pmb_state) == 52, "state record");
    cudaSetDevice(w->device);
    const uint32_t n = w->d.n;
    float* staging = reinterpret_cast<float*>(w->d.io_rec);
    launch_pack_states(w->d, 0, n, staging, w->stream);
    cudaMemcpyAsync(out, staging, sizeof(pmb_state) * size_t(n), cudaMemcpyDeviceToHost, w->stream);
    return check(cudaStreamSynchronize(w->stream));
}

int pmb_world_set_states(pmb_world* w, const pmb_state* in) {
    if (!w || !in) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    const uint32_t n = w->d.n;
    float* staging = reinterpret_cast<float*>(w->d.io_rec);
    cudaMemcpyAsync(staging, in, sizeof(pmb_state) * size_t(n), cudaMemcpyHostToDevice, w->stream);
    launch_unpack_states(w->d, n, staging, w->stream);
    return check(cudaStreamSynchronize(w->stream));
}

int pmb_world_apply_impulse(pmb_world* w, uint32_t body, const float* linear, const float* angular) {
    if (!w || body >= w->d.n) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    float4 l{0, 0, 0, 0}, a{0, 0, 0, 0};
    cudaMemcpyAsync(&l, w->d.lin_imp + body, 16, cudaMemcpyDeviceToHost, w->stream);
    cudaMemcpyAsync(&a, w->d.ang_imp + body, 16, cudaMemcpyDeviceToHost, w->stream);
    cudaStreamSynchronize(w->stream);
    if (linear) { l.x += linear[0]; l.y += linear[1]; l.z += linear[2]; }
    if (angular) { a.x += angular[0]; a.y += angular[1]; a.z += angular[2]; }
    cudaMemcpyAsync(w->d.lin_imp + body, &l, 16, cudaMemcpyHostToDevice, w->stream);
    cudaMemcpyAsync(w->d.ang_imp + body, &a, 16, cudaMemcpyHostToDevice, w->stream);
    return check(cudaStreamSynchronize(w->stream));
}

int pmb_world_candidate_pairs(pmb_world* w, uint64_t* codes, uint32_t capacity, uint32_t* count) {
    if (!w) return PMB_ERROR_INVALID_ARGUMENT;
    pmb_step_stats st;
    int r = pmb_world_last_stats(w, &st);
    if (r) return r;
    const uint32_t n = w->host_ctr.n_cand;
    if (count) *count = n;
    if (codes && capacity >= n && n) {
        std::vector<uint32_t> a(n), b(n);
        cudaMemcpy(a.data(), w->d.cand_a, 4 * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(b.data(), w->d.cand_b, 4 * n, cudaMemcpyDeviceToHost);
        for (uint32_t k = 0; k < n; ++k) codes[k] = uint64_t(a[k]) * w->d.n + b[k];
    }
    return check(cudaGetLastError());
}

int pmb_world_manifolds(pmb_world* w, uint64_t* codes, uint32_t* counts, float* contacts, uint32_t capacity,
                        uint32_t* count) {
    if (!w) return PMB_ERROR_INVALID_ARGUMENT;
    pmb_step_stats st;
    int r = pmb_world_last_stats(w, &st);
    if (r) return r;
    const uint32_t n = w->host_ctr.n_act, nc = w->host_ctr.n_contacts;
    if (count) *count = n;
    if (!codes || capacity < n || n == 0) return PMB_SUCCESS;
    std::vector<uint32_t> off(n), cnt(n);
    cudaMemcpy(codes, w->d.act_code, 8 * size_t(n), cudaMemcpyDeviceToHost);
    cudaMemcpy(off.data(), w->d.act_off, 4 * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(cnt.data(), w->d.act_cnt, 4 * n, cudaMemcpyDeviceToHost);
    if (counts) std::memcpy(counts, cnt.data(), 4 * n);
    if (contacts) {
        std::vector<float4> cn(nc), cp(nc), ce(nc), cl(nc), ck(nc), ca(nc), cb(nc);
        cudaMemcpy(cn.data(), w->d.c_n, 16 * nc, cudaMemcpyDeviceToHost);
        cudaMemcpy(cp.data(), w->d.c_p, 16 * nc, cudaMemcpyDeviceToHost);
        cudaMemcpy(ce.data(), w->d.c_e, 16 * nc, cudaMemcpyDeviceToHost);
        cudaMemcpy(cl.data(), w->d.c_lam, 16 * nc, cudaMemcpyDeviceToHost);
        cudaMemcpy(ck.data(), w->d.c_pen, 16 * nc, cudaMemcpyDeviceToHost);
        cudaMemcpy(ca.data(), w->d.c_aa, 16 * nc, cudaMemcpyDeviceToHost);
        cudaMemcpy(cb.data(), w->d.c_ab, 16 * nc, cudaMemcpyDeviceToHost);
        std::memset(contacts, 0, sizeof(float) * 22 * 8 * size_t(n));
        for (uint32_t k = 0; k < n; ++k)
            for (uint32_t p = 0; p < cnt[k] && p < 8; ++p) {
                const uint32_t c = off[k] + p;
                float* o = contacts + (size_t(k) * 8 + p) * 22;
                float v[22] = {cn[c].x, cn[c].y, cn[c].z, cp[c].x, cp[c].y, cp[c].z, cn[c].w, ce[c].x,
                               ce[c].y, ce[c].z, cl[c].x, ck[c].x, cl[c].y, ck[c].y, cl[c].z, ck[c].z,
                               ca[c].x, ca[c].y, ca[c].z, cb[c].x, cb[c].y, cb[c].z};
                std::memcpy(o, v, sizeof(v));
            }
    }
    return check(cudaGetLastError());
}

int pmb_world_graph(pmb_world* w, uint32_t* colors, uint32_t* parents) {
    if (!w) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    cudaStreamSynchronize(w->stream);
    if (colors) cudaMemcpy(colors, w->d.color, 4 * w->d.n, cudaMemcpyDeviceToHost);
    if (parents) cudaMemcpy(parents, w->d.parent, 4 * w->d.n, cudaMemcpyDeviceToHost);
    return check(cudaGetLastError());
}

int pmb_world_residual_trace(pmb_world* w, float* out, uint32_t capacity, uint32_t* count) {
    if (!w) return PMB_ERROR_INVALID_ARGUMENT;
    pmb_step_stats st;
    int r = pmb_world_last_stats(w, &st);
    if (r) return r;
    uint32_t n = std::min<uint32_t>(w->host_ctr.iterations, kMaxIterations);
    if (count) *count = n;
    if (out)
        for (uint32_t k = 0; k < n && k < capacity; ++k) out[k] = w->host_ctr.residual_trace[k];
    return PMB_SUCCESS;
}

int pmb_world_snapshot(pmb_world* w) {
    if (!w) return PMB_ERROR_INVALID_ARGUMENT;
    if (w->snapshot.size() != w->dynamic_state.size()) return PMB_ERROR_FEATURE_NOT_PRESENT;
    cudaSetDevice(w->device);
    w->snapshot_parity = w->step_parity;
    for (size_t k = 0; k < w->dynamic_state.size(); ++k)
        cudaMemcpyAsync(w->snapshot[k], w->dynamic_state[k].first, w->dynamic_state[k].second,
                        cudaMemcpyDeviceToDevice, w->stream);
    return check(cudaStreamSynchronize(w->stream));
}

int pmb_world_restore(pmb_world* w) {
    if (!w) return PMB_ERROR_INVALID_ARGUMENT;
    if (w->snapshot.size() != w->dynamic_state.size()) return PMB_ERROR_FEATURE_NOT_PRESENT;
    cudaSetDevice(w->device);
    if (w->step_parity != w->snapshot_parity) swap_cache(w);
    for (size_t k = 0; k < w->dynamic_state.size(); ++k)
        cudaMemcpyAsync(w->dynamic_state[k].first, w->snapshot[k], w->dynamic_state[k].second,
                        cudaMemcpyDeviceToDevice, w->stream);
    return check(cudaStreamSynchronize(w->stream));
}

namespace {
bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }
bool valid_quaternion(const float* q) {
    if (!std::isfinite(q[0]) || !std::isfinite(q[1]) || !std::isfinite(q[2]) || !std::isfinite(q[3])) return false;
    const float size = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    return size > kEps * kEps;
}
// Stage sparse per-body records (4 float4 each) and scatter them on the
// world's stream. Pageable sources are staged by the copy before it returns.
int stage_records(pmb_world* w, uint32_t kind, uint32_t count, const uint32_t* bodies, const float4* recs) {
    if (count == 0) return PMB_SUCCESS;
    cudaSetDevice(w->device);
    cudaMemcpyAsync(w->d.io_index, bodies, 4 * size_t(count), cudaMemcpyHostToDevice, w->stream);
    cudaMemcpyAsync(w->d.io_rec, recs, 64 * size_t(count), cudaMemcpyHostToDevice, w->stream);
    launch_scatter_records(w->d, kind, count, w->stream);
    return check(cudaGetLastError());
}
bool unique_bodies(uint32_t n, uint32_t count, const uint32_t* bodies) {
    std::vector<uint8_t> seen(n, 0);
    for (uint32_t k = 0; k < count; ++k) {
        if (bodies[k] >= n || seen[bodies[k]]) return false;
        seen[bodies[k]] = 1;
    }
    return true;
}
}  // namespace

int pmb_world_set_inputs(pmb_world* w, uint32_t count, const uint32_t* bodies, const float* values) {
    if (!w || (count && (!bodies || !values)) || count > w->d.n || !unique_bodies(w->d.n, count, bodies))
        return PMB_ERROR_INVALID_ARGUMENT;
    std::vector<float4> rec(4 * size_t(count));
    for (uint32_t k = 0; k < count; ++k) {
        const float* v = values + 12 * size_t(k);
        for (int f = 0; f < 4; ++f) {
            if (!finite3(v + 3 * f)) return PMB_ERROR_INVALID_ARGUMENT;
            rec[4 * k + f] = make_float4(v[3 * f], v[3 * f + 1], v[3 * f + 2], 0.0f);
        }
    }
    return stage_records(w, 0, count, bodies, rec.data());
}

int pmb_world_set_targets(pmb_world* w, uint32_t count, const uint32_t* bodies, const pmb_state* targets) {
    if (!w || (count && (!bodies || !targets)) || count > w->d.n || !unique_bodies(w->d.n, count, bodies))
        return PMB_ERROR_INVALID_ARGUMENT;
    std::vector<float4> rec(4 * size_t(count));
    for (uint32_t k = 0; k < count; ++k) {
        const pmb_state& t = targets[k];
        if (!finite3(t.x) || !valid_quaternion(t.q) || !finite3(t.v) || !finite3(t.w))
            return PMB_ERROR_INVALID_ARGUMENT;
        rec[4 * k] = make_float4(t.x[0], t.x[1], t.x[2], 0.0f);
        rec[4 * k + 1] = make_float4(t.q[0], t.q[1], t.q[2], t.q[3]);
    }
    return stage_records(w, 1, count, bodies, rec.data());
}

int pmb_world_write_states(pmb_world* w, uint32_t first, uint32_t count, const pmb_state* states) {
    if (!w || (count && !states) || first > w->d.n || count > w->d.n - first) return PMB_ERROR_INVALID_ARGUMENT;
    std::vector<uint32_t> idx(count);
    std::vector<float4> rec(4 * size_t(count));
    for (uint32_t k = 0; k < count; ++k) {
        const pmb_state& t = states[k];
        if (!finite3(t.x) || !valid_quaternion(t.q) || !finite3(t.v) || !finite3(t.w))
            return PMB_ERROR_INVALID_ARGUMENT;
        idx[k] = first + k;
        rec[4 * k] = make_float4(t.x[0], t.x[1], t.x[2], 0.0f);
        rec[4 * k + 1] = make_float4(t.q[0], t.q[1], t.q[2], t.q[3]);
        rec[4 * k + 2] = make_float4(t.v[0], t.v[1], t.v[2], 0.0f);
        rec[4 * k + 3] = make_float4(t.w[0], t.w[1], t.w[2], 0.0f);
    }
    int r = stage_records(w, 2, count, idx.data(), rec.data());
    if (r != PMB_SUCCESS) return r;
    // Joints touching a rewritten body restart their rows from zero.
    for (uint32_t j = 0; j < uint32_t(w->host_joints.size()); ++j) {
        const pmb_joint& o = w->host_joints[j];
        const bool touches = (o.body_a >= first && o.body_a - first < count) ||
                             (o.body_b >= first && o.body_b - first < count);
        if (touches) cudaMemsetAsync(w->d.jrows + 18 * size_t(j), 0, 18 * sizeof(JointRow), w->stream);
    }
    return check(cudaGetLastError());
}

int pmb_world_copy_states_to_device(pmb_world* w, uint32_t first, uint32_t count, void* dst) {
    if (!w || (count && !dst) || first > w->d.n || count > w->d.n - first ||
        (reinterpret_cast<uintptr_t>(dst) & 3u))
        return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    launch_pack_states(w->d, first, count, static_cast<float*>(dst), w->stream);
    return check(cudaGetLastError());
}

int pmb_world_memory_requirements(const pmb_world_capacity* c, uint64_t* persistent, uint64_t* scratch) {
    if (!c || !persistent || !scratch || c->body_count == 0) return PMB_ERROR_INVALID_ARGUMENT;
    const uint32_t n = c->body_count;
    pmb_world probe;
    probe.counting = true;
    const Sizes z{n,
                  std::max(1u, c->mesh_count),
                  c->joint_count,
                  0u,
                  size_t(c->mesh_vertex_count),
                  2 * size_t(c->mesh_triangle_count),
                  size_t(c->joint_count),
                  size_t(c->joint_count),
                  size_t(c->joint_count),
                  c->candidate_capacity ? c->candidate_capacity : 64u * n + 4096u,
                  c->pair_capacity ? c->pair_capacity : 24u * n + 1024u,
                  c->contact_capacity ? c->contact_capacity : 64u * n + 4096u,
                  c->event_capacity,
                  size_t(c->joint_count),
                  2 * size_t(c->mesh_triangle_count) + std::max(1u, c->mesh_count),
                  size_t(c->mesh_triangle_count)};
    Extra ex{};
    allocate_world(&probe, probe.d, z, ex);
    *persistent = probe.arena_used[kPersistent];
    *scratch = probe.arena_used[kScratch];
    return PMB_SUCCESS;
}

// Telemetry of the latest tick: the host's launch ledger plus counts the
// device recorded (colour rounds, sweeps, colours, contacts), with the
// algorithmic byte model of each phase.
int pmb_world_tick_telemetry(pmb_world* w, pmb_tick_telemetry* out) {
    if (!w || !out) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    Counters c;
    cudaMemcpyAsync(&c, w->d.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, w->stream);
    const int r = check(cudaStreamSynchronize(w->stream));
    if (r != PMB_SUCCESS) return r;
    *out = pmb_tick_telemetry{};
    out->tick = w->ticks_enqueued;
    for (int p = 0; p < kPhases; ++p) {
        out->dispatches[p] = w->ledger.dispatches[p];
        out->workgroups[p] = w->ledger.workgroups[p];
    }
    const uint64_t n = w->d.n, con = c.n_contacts;
    const uint64_t sweeps = uint64_t(c.iterations) + (c.impact ? uint64_t(c.budget) : 0u);
    out->sweeps = sweeps;
    out->spatial_builds = 1;
    out->barriers[kPhDomain] = 2ull * c.rounds + sweeps * (uint64_t(c.colors) + 1u);
    out->bytes_moved[kPhPredict] = 250u * n;
    out->bytes_moved[kPhIndex] = 100u * n;
    out->bytes_moved[kPhCandidates] = 8ull * c.n_cand + 64u * con;
    out->bytes_moved[kPhDomain] = 604u * con + sweeps * (124u * n + 384u * con);
    out->bytes_moved[kPhCommit] = 200u * n + 250u * con;
    return PMB_SUCCESS;
}

int pmb_world_contact_events(pmb_world* w, pmb_contact_event* out, uint32_t capacity, uint32_t* count) {
    if (!w || !count || (capacity && !out)) return PMB_ERROR_INVALID_ARGUMENT;
    static_assert(sizeof(pmb_contact_event) == sizeof(ContactEvent), "event record");
    cudaSetDevice(w->device);
    uint32_t n = 0;
    cudaMemcpyAsync(&n, &w->d.ctr->n_events, sizeof(n), cudaMemcpyDeviceToHost, w->stream);
    int r = check(cudaStreamSynchronize(w->stream));
    if (r != PMB_SUCCESS) return r;
    n = std::min(n, w->d.event_capacity);
    *count = n;
    const uint32_t m = std::min(n, capacity);
    if (m) {
        cudaMemcpyAsync(out, w->d.events, sizeof(ContactEvent) * size_t(m), cudaMemcpyDeviceToHost, w->stream);
        r = check(cudaStreamSynchronize(w->stream));
    }
    return r;
}

int pmb_world_joints(pmb_world* w, uint32_t* flags, float* applied, uint32_t* counts, uint32_t capacity) {
    if (!w || capacity < w->d.nj) return PMB_ERROR_INVALID_ARGUMENT;
    const uint32_t nj = w->d.nj;
    if (nj == 0) return PMB_SUCCESS;
    cudaSetDevice(w->device);
    std::vector<JointState> js(nj);
    cudaMemcpyAsync(js.data(), w->d.jstate, sizeof(JointState) * nj, cudaMemcpyDeviceToHost, w->stream);
    int r = check(cudaStreamSynchronize(w->stream));
    if (r != PMB_SUCCESS) return r;
    for (uint32_t j = 0; j < nj; ++j) {
        if (flags) flags[j] = js[j].enabled | (js[j].broken << 1);
        if (applied) applied[j] = js[j].applied;
        if (counts) counts[j] = js[j].count;
    }
    return PMB_SUCCESS;
}

int pmb_world_contact_duals(pmb_world* w, uint32_t rows, float* lambda, float* penalty, uint32_t capacity,
                            uint32_t* count) {
    if (!w || rows < 1 || rows > 3) return PMB_ERROR_INVALID_ARGUMENT;
    pmb_step_stats st;
    int r = pmb_world_last_stats(w, &st);
    if (r) return r;
    const uint32_t nc = w->host_ctr.n_contacts;
    if (count) *count = nc;
    if (!lambda || !penalty || capacity < nc || nc == 0) return PMB_SUCCESS;
    std::vector<float4> lam(nc), pen(nc);
    cudaMemcpyAsync(lam.data(), w->d.c_lam, 16 * size_t(nc), cudaMemcpyDeviceToHost, w->stream);
    cudaMemcpyAsync(pen.data(), w->d.c_pen, 16 * size_t(nc), cudaMemcpyDeviceToHost, w->stream);
    r = check(cudaStreamSynchronize(w->stream));
    if (r) return r;
    for (uint32_t c = 0; c < nc; ++c) {
        const float l[3] = {lam[c].x, lam[c].y, lam[c].z}, k[3] = {pen[c].x, pen[c].y, pen[c].z};
        for (uint32_t x = 0; x < rows; ++x) {
            lambda[rows * size_t(c) + x] = l[x];
            penalty[rows * size_t(c) + x] = k[x];
        }
    }
    return PMB_SUCCESS;
}

int pmb_world_set_warm_table(pmb_world* w, uint32_t rows, const float* lambda, const float* penalty,
                             uint32_t count) {
    if (!w || rows < 1 || rows > 3 || (count && (!lambda || !penalty)) || count > w->d.cap_contact)
        return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    std::vector<float4> t(2 * size_t(count));
    for (uint32_t c = 0; c < count; ++c) {
        float l[3] = {-1.0f, std::nanf(""), std::nanf("")}, k[3] = {0.0f, 0.0f, 0.0f};
        for (uint32_t x = 0; x < rows; ++x) {
            l[x] = lambda[rows * size_t(c) + x];
            k[x] = penalty[rows * size_t(c) + x];
        }
        t[2 * size_t(c)] = make_float4(l[0], l[1], l[2], 0.0f);
        t[2 * size_t(c) + 1] = make_float4(k[0], k[1], k[2], 0.0f);
    }
    if (count) cudaMemcpyAsync(w->d.warm_table, t.data(), 32 * size_t(count), cudaMemcpyHostToDevice, w->stream);
    w->d.warm_count = count;
    w->d.warm_rows = rows;
    return check(cudaStreamSynchronize(w->stream));
}


int pmb_world_mlp_attach(pmb_world* w, const float* params, uint32_t seed) {
    if (!w) return PMB_ERROR_INVALID_ARGUMENT;
    if (w->arena[kPersistent]) return PMB_ERROR_FEATURE_NOT_PRESENT;
    cudaSetDevice(w->device);
    auto& m = w->mlp;
    if (!m.attached) {
        if (mlp_configure_kernels() != 0) return PMB_ERROR_DEVICE_LOST;
        const size_t tiles = (size_t(w->d.cap_contact) + kMlpTile - 1) / kMlpTile;
        m.grid = mlp_grid(uint32_t(tiles));
        int r = PMB_SUCCESS;
        if (!r) r = mlp_alloc(w, m.params, kMlpParams);
        if (!r) r = mlp_alloc(w, m.m, kMlpParams);
        if (!r) r = mlp_alloc(w, m.v, kMlpParams);
        if (!r) r = mlp_alloc(w, m.grad, kMlpPartial);
        if (!r) r = mlp_alloc(w, m.partial, size_t(m.grid) * kMlpPartial);
        if (!r) r = mlp_alloc(w, m.gate, 1);
        if (!r) r = mlp_alloc(w, m.out, tiles * kMlpTile * 2);
        if (!r) r = mlp_alloc(w, m.img, kImgBytes);
        if (!r) r = mlp_alloc(w, m.x, tiles * 4096);
        if (!r) r = mlp_alloc(w, m.meta, tiles * kMlpTile);
        if (r) return r;
        m.attached = true;
    }
    std::vector<float> host;
    if (params)
        host.assign(params, params + kMlpParams);
    else
        init_params(seed, host);
    cudaMemcpyAsync(m.params, host.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, w->stream);
    cudaMemsetAsync(m.m, 0, sizeof(float) * kMlpParams, w->stream);
    cudaMemsetAsync(m.v, 0, sizeof(float) * kMlpParams, w->stream);
    // Given parameters apply at once; a fresh model waits for training to
    // show it beats the plain warm start.
    const float open = params ? 1.0f : 0.0f;
    cudaMemcpyAsync(m.gate, &open, sizeof(float), cudaMemcpyHostToDevice, w->stream);
    m.adam_t = 0;
    launch_mlp_images(m.params, m.img, w->stream);
    return check(cudaStreamSynchronize(w->stream));
}

int pmb_world_mlp_apply_mode(pmb_world* w, uint32_t mode) {
    if (!w || !w->mlp.attached || mode == 0 || mode > 7) return PMB_ERROR_INVALID_ARGUMENT;
    w->mlp.mode = mode;
    return PMB_SUCCESS;
}

int pmb_world_mlp_train(pmb_world* w, int enable, float learning_rate, uint32_t steps_per_tick) {
    if (!w || !w->mlp.attached || !(learning_rate >= 0.0f) || steps_per_tick == 0) return PMB_ERROR_INVALID_ARGUMENT;
    w->mlp.train = enable != 0;
    w->mlp.lr = learning_rate;
    w->mlp.steps_per_tick = steps_per_tick;
    return PMB_SUCCESS;
}

int pmb_world_mlp_params(pmb_world* w, float* params, float* last_loss, float* plain_loss, float* gate) {
    if (!w || !w->mlp.attached) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    if (params)
        cudaMemcpyAsync(params, w->mlp.params, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, w->stream);
    if (last_loss)
        cudaMemcpyAsync(last_loss, w->mlp.grad + kMlpParams, sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    if (plain_loss)
        cudaMemcpyAsync(plain_loss, w->mlp.grad + kMlpParams + 1, sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    if (gate) cudaMemcpyAsync(gate, w->mlp.gate, sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    return check(cudaStreamSynchronize(w->stream));
}

int pmb_world_mlp_rows(pmb_world* w, float* features, float* meta, uint32_t capacity, uint32_t* count) {
    if (!w || !w->mlp.attached) return PMB_ERROR_INVALID_ARGUMENT;
    pmb_step_stats st;
    int r = pmb_world_last_stats(w, &st);
    if (r) return r;
    const uint32_t nc = w->host_ctr.n_contacts;
    if (count) *count = nc;
    if (!features || !meta || capacity < nc || nc == 0) return PMB_SUCCESS;
    const uint32_t tiles = (nc + kMlpTile - 1) / kMlpTile;
    std::vector<uint16_t> x(size_t(tiles) * 2048);
    cudaMemcpyAsync(x.data(), w->mlp.x, size_t(tiles) * 4096, cudaMemcpyDeviceToHost, w->stream);
    cudaMemcpyAsync(meta, w->mlp.meta, sizeof(MlpMeta) * size_t(nc), cudaMemcpyDeviceToHost, w->stream);
    r = check(cudaStreamSynchronize(w->stream));
    if (r) return r;
    for (uint32_t c = 0; c < nc; ++c)
        for (uint32_t k = 0; k < kMlpFeatures; ++k) {
            const uint32_t bits = uint32_t(x[(size_t(c / kMlpTile) * 4096 + tile_offset(c % kMlpTile, k)) / 2]) << 16;
            std::memcpy(&features[kMlpFeatures * size_t(c) + k], &bits, 4);
        }
    return PMB_SUCCESS;
}

int pmb_mlp_forward_backward(int32_t device, uint32_t rows, const float* features, const float* targets,
                             const float* weights, const float* params, float* outputs, float* grads, float* loss) {
    if (!features || !targets || !weights || !params || rows == 0) return PMB_ERROR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PMB_ERROR_NO_DEVICE;
    if (device < 0 || device >= ndev) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(device);
    if (mlp_configure_kernels() != 0) return PMB_ERROR_DEVICE_LOST;
    const uint32_t tiles = (rows + kMlpTile - 1) / kMlpTile, grid = mlp_grid(tiles);
    std::vector<void*> owned;
    auto get = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
        owned.push_back(p);
        return p;
    };
    float* d_feat = static_cast<float*>(get(sizeof(float) * kMlpFeatures * rows));
    float* d_y = static_cast<float*>(get(sizeof(float) * 2 * rows));
    float* d_w = static_cast<float*>(get(sizeof(float) * rows));
    float* d_p = static_cast<float*>(get(sizeof(float) * kMlpParams));
    float* d_out = static_cast<float*>(get(sizeof(float) * 2 * rows));
    float* d_grad = static_cast<float*>(get(sizeof(float) * kMlpPartial));
    float* d_part = static_cast<float*>(get(sizeof(float) * grid * kMlpPartial));
    uint8_t* d_img = static_cast<uint8_t*>(get(kImgBytes));
    uint8_t* d_x = static_cast<uint8_t*>(get(size_t(tiles) * 4096));
    MlpMeta* d_meta = static_cast<MlpMeta*>(get(sizeof(MlpMeta) * tiles * kMlpTile));
    uint32_t* d_status = static_cast<uint32_t*>(get(sizeof(uint32_t)));
    int r = PMB_SUCCESS;
    for (void* p : owned)
        if (!p) r = PMB_ERROR_OUT_OF_DEVICE_MEMORY;
    if (owned.size() != 11) r = PMB_ERROR_OUT_OF_DEVICE_MEMORY;
    uint32_t status = 0;
    if (r == PMB_SUCCESS) {
        cudaStream_t s = nullptr;
        cudaMemcpy(d_feat, features, sizeof(float) * kMlpFeatures * rows, cudaMemcpyHostToDevice);
        cudaMemcpy(d_y, targets, sizeof(float) * 2 * rows, cudaMemcpyHostToDevice);
        cudaMemcpy(d_w, weights, sizeof(float) * rows, cudaMemcpyHostToDevice);
        cudaMemcpy(d_p, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice);
        cudaMemset(d_status, 0, sizeof(uint32_t));
        launch_mlp_images(d_p, d_img, s);
        launch_mlp_pack_rows(d_feat, d_y, d_w, rows, d_x, d_meta, tiles, s);
        launch_mlp_tiles(true, d_x, d_meta, d_img, rows, tiles, nullptr, d_out, d_part, d_status, 1u, grid, s);
        launch_mlp_reduce_adam(d_part, grid, d_grad, nullptr, nullptr, nullptr, 0.0f, 0.9f, 0.999f, 1.0f, 1.0f, 1e-8f,
                               nullptr, s);
        r = check(cudaDeviceSynchronize());
        if (r == PMB_SUCCESS) {
            cudaMemcpy(&status, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost);
            if (outputs) cudaMemcpy(outputs, d_out, sizeof(float) * 2 * rows, cudaMemcpyDeviceToHost);
            std::vector<float> g(kMlpPartial);
            cudaMemcpy(g.data(), d_grad, sizeof(float) * kMlpPartial, cudaMemcpyDeviceToHost);
            if (grads) std::memcpy(grads, g.data(), sizeof(float) * kMlpParams);
            if (loss) *loss = g[kMlpParams];
            r = check(cudaGetLastError());
        }
    }
    for (void* p : owned)
        if (p) cudaFree(p);
    if (r == PMB_SUCCESS && status) r = PMB_ERROR_DEVICE_LOST;
    return r;
}

int pmb_world_scene_stats(pmb_world* w, float* residual, float* residual_max, uint32_t* iterations,
                          uint32_t* contacts, uint32_t capacity) {
    if (!w || w->d.n_scenes <= 1 || capacity < w->d.n_scenes) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(w->device);
    const uint32_t ns = w->d.n_scenes;
    std::vector<float> sq(ns), mx(ns);
    std::vector<uint32_t> cnt(ns), bud(ns);
    cudaMemcpyAsync(sq.data(), w->d.scene_res_sq, 4 * size_t(ns), cudaMemcpyDeviceToHost, w->stream);
    cudaMemcpyAsync(mx.data(), w->d.scene_res_mx, 4 * size_t(ns), cudaMemcpyDeviceToHost, w->stream);
    cudaMemcpyAsync(cnt.data(), w->d.scene_res_n, 4 * size_t(ns), cudaMemcpyDeviceToHost, w->stream);
    cudaMemcpyAsync(bud.data(), w->d.scene_budget, 4 * size_t(ns), cudaMemcpyDeviceToHost, w->stream);
    std::vector<uint32_t> per_scene;
    if (contacts) {
        // Contact points per scene from the last tick's pairs.
        pmb_step_stats st;
        int r = pmb_world_last_stats(w, &st);
        if (r) return r;
        const uint32_t na = w->host_ctr.n_act;
        std::vector<uint32_t> a(na), c(na), scene(w->d.n);
        cudaMemcpyAsync(a.data(), w->d.act_a, 4 * size_t(na), cudaMemcpyDeviceToHost, w->stream);
        cudaMemcpyAsync(c.data(), w->d.act_cnt, 4 * size_t(na), cudaMemcpyDeviceToHost, w->stream);
        cudaMemcpyAsync(scene.data(), w->d.scene_of, 4 * size_t(w->d.n), cudaMemcpyDeviceToHost, w->stream);
        r = check(cudaStreamSynchronize(w->stream));
        if (r) return r;
        per_scene.assign(ns, 0);
        for (uint32_t k = 0; k < na; ++k) per_scene[scene[a[k]]] += c[k];
    }
    int r = check(cudaStreamSynchronize(w->stream));
    if (r) return r;
    for (uint32_t k = 0; k < ns; ++k) {
        if (residual) residual[k] = cnt[k] ? std::sqrt(sq[k] / float(cnt[k])) : 0.0f;
        if (residual_max) residual_max[k] = mx[k];
        if (iterations) iterations[k] = bud[k];
        if (contacts) contacts[k] = per_scene[k];
    }
    return PMB_SUCCESS;
}

constexpr uint32_t kSolvePolicies = 5;
const char* const kPolicyNames[kSolvePolicies] = {"per colour", "8 lanes   ", "per body  ", "claimed   ",
                                                  "thread/body"};

// The staged variants choose lanes per body per colour batch (policy 0) or
// always 8 (policy 1); policies 2 and 3 run them as policy 0.
bool plan_distinct(uint32_t variant, uint32_t policy) { return variant < kStagedFirst || policy < 2; }

int pmb_world_set_launch_plan(pmb_world* w, uint32_t solve_variant, uint32_t solve_policy) {
    if (!w || solve_variant >= kSolveVariants || solve_policy >= kSolvePolicies) return PMB_ERROR_INVALID_ARGUMENT;
    w->d.solve_variant = solve_variant;
    w->d.solve_policy = solve_policy;
    return PMB_SUCCESS;
}

int pmb_world_set_barrier_limit(pmb_world* w, uint32_t spins) {
    if (!w) return PMB_ERROR_INVALID_ARGUMENT;
    w->d.barrier_spins = spins ? spins : kDefaultBarrierSpins;
    return PMB_SUCCESS;
}

int pmb_world_autotune(pmb_world* w, const pmb_step_desc* step, uint32_t ticks, uint32_t* solve_variant,
                       uint32_t* solve_policy, char* report, uint32_t capacity) {
    if (!w || !step || ticks == 0) return PMB_ERROR_INVALID_ARGUMENT;
    if (w->snapshot.size() != w->dynamic_state.size()) return PMB_ERROR_FEATURE_NOT_PRESENT;
    cudaSetDevice(w->device);
    int r = pmb_world_snapshot(w);
    if (r) return r;
    const StepParams sp = params_from(*step);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 0.0f;
    uint32_t bv = 0, bp = 0;
    std::string text;
    for (uint32_t v = 0; v < kSolveVariants && r == PMB_SUCCESS; ++v)
        for (uint32_t p = 0; p < kSolvePolicies && r == PMB_SUCCESS; ++p) {
            if (!plan_distinct(v, p)) continue;
            r = pmb_world_restore(w);
            if (r) break;
            w->d.solve_variant = v;
            w->d.solve_policy = p;
            enqueue_step(w, sp);  // untimed: first launch of this plan
            cudaEventRecord(a, w->stream);
            for (uint32_t k = 0; k < ticks; ++k) enqueue_step(w, sp);
            cudaEventRecord(b, w->stream);
            r = check(cudaEventSynchronize(b));
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, a, b);
            char line[128];
            std::snprintf(line, sizeof(line), "solve %3d threads%s, widths %s: %8.3f ms/tick\n",
                          ::pmb::solve_variant(v).threads, v >= kStagedFirst ? " staged" : "", kPolicyNames[p],
                          ms / float(ticks));
            text += line;
            if ((v == 0 && p == 0) || ms < best) {
                best = ms;
                bv = v;
                bp = p;
            }
        }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    const int rr = pmb_world_restore(w);
    if (r == PMB_SUCCESS) r = rr;
    w->d.solve_variant = bv;
    w->d.solve_policy = bp;
    if (solve_variant) *solve_variant = bv;
    if (solve_policy) *solve_policy = bp;
    if (report && capacity) std::snprintf(report, capacity, "%s", text.c_str());
    return r;
}

int pmb_world_stream(pmb_world* w, void** stream) {
    if (!w || !stream) return PMB_ERROR_INVALID_ARGUMENT;
    *stream = w->stream;
    return PMB_SUCCESS;
}

int pmb_math_eval(uint32_t kind, uint32_t count, const float* in, float* out) {
    static const uint32_t in_w[5] = {27, 7, 4, 42, 3}, out_w[5] = {7, 5, 6, 7, 2};
    if (kind > 4 || !in || !out) return PMB_ERROR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PMB_ERROR_NO_DEVICE;
    if (count == 0) return PMB_SUCCESS;
    float *din = nullptr, *dout = nullptr;
    if (cudaMalloc(&din, 4 * size_t(count) * in_w[kind]) != cudaSuccess) return PMB_ERROR_OUT_OF_DEVICE_MEMORY;
    if (cudaMalloc(&dout, 4 * size_t(count) * out_w[kind]) != cudaSuccess) {
        cudaFree(din);
        return PMB_ERROR_OUT_OF_DEVICE_MEMORY;
    }
    cudaMemcpy(din, in, 4 * size_t(count) * in_w[kind], cudaMemcpyHostToDevice);
    k_math_eval<<<(count + 127) / 128, 128>>>(kind, count, din, dout);
    note_launch((count + 127) / 128);
    cudaMemcpy(out, dout, 4 * size_t(count) * out_w[kind], cudaMemcpyDeviceToHost);
    int r = check(cudaGetLastError());
    cudaFree(din);
    cudaFree(dout);
    return r;
}

}  // extern "C"

namespace pmb {
__global__ void k_math_eval(uint32_t kind, uint32_t count, const float* in, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    if (kind == 0) {
        const float* v = in + 27 * size_t(i);
        Blk b;
        for (int k = 0; k < 21; ++k) b.h[k] = v[k];
        for (int k = 0; k < 6; ++k) b.g[k] = v[21 + k];
        V6 dd;
        bool ok = block_solve(b, dd);
        float* o = out + 7 * size_t(i);
        for (int k = 0; k < 6; ++k) o[k] = dd.v[k];
        o[6] = ok ? 1.0f : 0.0f;
    } else if (kind == 1) {
        const float* v = in + 7 * size_t(i);
        Dual du{v[0], v[1]};
        Dual ws = warm_start(du, v[6]);
        Dual up = update_dual(du, v[2], v[3], v[4], v[5], v[6]);
        float* o = out + 5 * size_t(i);
        o[0] = ws.lambda;
        o[1] = ws.penalty;
        o[2] = dual_force(du, v[2], v[4], v[5]);
        o[3] = up.lambda;
        o[4] = up.penalty;
    } else if (kind == 2) {
        const float* v = in + 4 * size_t(i);
        F3 t{v[0], v[1], v[2]};
        F3 p = project_contact(t, v[3]), s = stiffness_scales(t, v[3]);
        float* o = out + 6 * size_t(i);
        o[0] = p.n;
        o[1] = p.t0;
        o[2] = p.t1;
        o[3] = s.n;
        o[4] = s.t0;
        o[5] = s.t1;
    } else if (kind == 4) {
        const float* v = in + 3 * size_t(i);
        out[2 * size_t(i)] = atan2_q1(v[0], v[1]);
        out[2 * size_t(i) + 1] = x_cot(v[2]);
    } else {
        const float* v = in + 42 * size_t(i);
        Row r;
        for (int k = 0; k < 6; ++k) {
            r.a.v[k] = v[k];
            r.b.v[k] = v[6 + k];
        }
        r.dual = {v[12], v[13]};
        r.error = v[14];
        r.velocity = v[15];
        r.lower = v[16];
        r.upper = v[17];
        r.stiffness = v[18];
        r.damping = v[19];
        r.beta = v[20];
        r.reference_force = v[21];
        V6 a, b;
        for (int k = 0; k < 6; ++k) {
            a.v[k] = v[22 + k];
            b.v[k] = v[28 + k];
        }
        const float dt = v[34];
        Blk blk;
        for (int k = 0; k < 21; ++k) blk.h[k] = 0.0f;
        for (int k = 0; k < 6; ++k) {
            blk.g[k] = 0.0f;
            blk.h[bidx(k, k)] = v[35 + k];
        }
        row_accumulate(blk, r, v[41] != 0.0f, a, b, dt);
        Row adv = row_advance(r, a, b);
        float* o = out + 7 * size_t(i);
        o[0] = row_error(r, a, b);
        o[1] = row_trial(r, a, b, dt);
        o[2] = row_force(r, a, b, dt);
        o[3] = adv.dual.lambda;
        o[4] = adv.dual.penalty;
        float gs = 0, ds = 0;
        for (int k = 0; k < 6; ++k) {
            gs += blk.g[k];
            ds += blk.h[bidx(k, k)];
        }
        o[5] = gs;
        o[6] = ds;
    }
}
}  // namespace pmb

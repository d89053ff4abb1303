// SPDX-License-Identifier: MIT
// The group-per-body cooperative solve kernel (a persistent CTA per SM),
// instantiated per CTA size in pmb_solve_t*.cu so that the instantiations
// compile in parallel.
#pragma once
#include "pmb_solve_common.cuh"

namespace pmb {

// T threads per CTA, one CTA per SM (cooperative): 512 threads cap a thread
// at 128 registers, 384 at 168, 256 at 255 -- fewer resident warps against
// fewer spills; the world picks one (pmb_world_autotune). Timed: the
// profiling build (pmb_world_profile_step), which records per-colour
// timestamps of the first sweep; the ticks run the untimed build. Feat: the
// code the world needs -- bit 0 (kFeatJoints) joint rows and joint duals,
// bit 1 (kFeatThread) the body-per-thread sweep of policy 4. A build without
// them has no call to the joint visit and no second body solver, so it needs
// far fewer registers (127 against 168 at 384 threads): more warps fit at
// 512 threads without spills. Every build computes the same bits.
template <int T, bool Timed, int Feat>
__global__ void __launch_bounds__(T, 1) k_solve(Dev d, StepParams sp, uint32_t phase) {
    constexpr int kSolveThreads = T;
    constexpr bool kJoints = (Feat & kFeatJoints) != 0;
    constexpr bool kThread = (Feat & kFeatThread) != 0;
    Counters* c = d.ctr;
    if (phase != 0 && c->impact == 0) return;
    if (c->status & kStBarrierTimeout) return;  // the tick was abandoned
    extern __shared__ __align__(16) uint8_t stage_raw[];
    const int lane = threadIdx.x & 31;
    uint8_t* warp_stage = stage_raw + (threadIdx.x >> 5) * kWarpStage;
    const uint32_t nthreads = gridDim.x * kSolveThreads;
    const float dt = sp.dt;
    const uint32_t colors = min(c->colors, kMaxColors);  // the colouring never exceeds kMaxColors
    uint32_t budget = sp.budget_request;
    if (!sp.realtime && sp.requested == 0) budget = max(budget, c->joint_iters);
    if (phase != 0 && sp.tolerance > 0.0f) budget = c->budget;
    // Batched worlds sweep every scene its own budget (no residual-driven stop).
    const bool adaptive = phase == 0 && sp.tolerance > 0.0f && !batched(d);
    const uint32_t iters = batched(d) ? min(c->budget_max, kMaxIterations)
                                      : adaptive ? min(max(sp.max_iterations, 1u), kMaxIterations)
                                                 : min(budget, kMaxIterations);
    const uint32_t n_con = c->n_contacts;
    __shared__ double wsq[kSolveThreads / 32];
    __shared__ uint32_t wn[kSolveThreads / 32], wov[kSolveThreads / 32];
    __shared__ float wmx[kSolveThreads / 32];
    const bool timing = Timed && phase == 0;
    auto now = [] {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        return t;
    };
    if (timing && blockIdx.x == 0 && threadIdx.x == 0) c->dbg_start = now();
    using W32 = std::integral_constant<int, 32>;
    using W16 = std::integral_constant<int, 16>;
    using W8 = std::integral_constant<int, 8>;
    // Each colour's body ranges, read once per launch: its first body, the
    // starts of its 16-lane and 8-lane sort classes, its end.
    __shared__ uint4 s_col[kMaxColors];
    for (uint32_t k = threadIdx.x; k < colors; k += kSolveThreads) {
        const uint32_t* off = c->color_off + k * kSortClasses;
        s_col[k] = make_uint4(off[0], off[kClass16], off[kClass8], off[kSortClasses]);
    }
    __syncthreads();
    // Lane widths of a colour (see the group-per-body comment): policy 0
    // (and 3) one width per colour by its size, 1 eight lanes, 2 a width per
    // body class (heaviest first) unless 32-lane groups cover the colour, 4
    // a body per thread when the colour has more bodies than 16-lane groups
    // could take in one round. Bodies [b0, r32) take 32 lanes, [r32, r16)
    // 16, [r16, r8) 8.
    struct Ranges {
        uint32_t b0, r32, r16, r8, b1;
        bool per_thread;
    };
    auto ranges = [&](uint32_t col) {
        const uint4 o = s_col[col];
        const uint32_t b0 = o.x, b1 = o.w, nb = b1 - b0;
        Ranges r{b0, b0, b0, b0, b1, false};
        if constexpr (kThread) r.per_thread = d.solve_policy == 4 && nb * 16u > nthreads;
        if (r.per_thread) {
        } else if (d.solve_policy != 1 && nb * 32u <= nthreads) {
            r.r32 = r.r16 = r.r8 = b1;
        } else if (d.solve_policy == 2) {
            r.r32 = o.y;
            r.r16 = o.z;
            r.r8 = b1;
        } else if ((d.solve_policy == 0 || d.solve_policy >= 3) && nb * 16u <= nthreads) {
            r.r16 = r.r8 = b1;
        } else {
            r.r8 = b1;
        }
        return r;
    };
    for (uint32_t it = 0; it < iters; ++it) {
        for (uint32_t col = 0; col < colors; ++col) {
            const Ranges rg = ranges(col);
            const uint32_t b0 = rg.b0, b1 = rg.b1;
            const uint32_t trace = !timing || it != 0 ? 0u : col + 1 == colors ? 1u : col == 0 ? 2u : 0u;
            // Bodies [lo, hi) with G lanes each. Consecutive bodies go to
            // consecutive CTAs (group rank = local group x grid + CTA), so the
            // heavy bodies at the front of a colour spread over all SMs.
            // Policy 3 hands the bodies out dynamically instead: each group
            // takes the next unclaimed body of the colour from a counter
            // (claiming its following one while it solves), so groups that
            // drew light bodies take more of them.
            const uint32_t step = it * colors + col;
            uint32_t* claim = &c->claim[step & 1u];
            if (d.solve_policy == 3 && blockIdx.x == 0 && threadIdx.x == 0) c->claim[(step + 1u) & 1u] = 0u;
            auto sweep = [&](auto width, uint32_t lo, uint32_t hi) {
                constexpr int G = decltype(width)::value;
                if (lo >= hi) return;
                const int gl = lane % G, gbase = lane - gl;
                const uint32_t gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << gbase;
                GroupRows<G>& sm = reinterpret_cast<GroupRows<G>*>(warp_stage)[gbase / G];
                // One call site of the body solve for both assignments (each
                // inlined copy adds its own stack frame). The group learns its
                // next body before solving the current one and fetches that
                // body's record and row codes during the solve.
                // Static assignment runs the rounds in alternating directions
                // (round r: slot r x groups + rank, or its mirror when r is
                // odd): the colour's bodies come heaviest class first, so a
                // group that drew a heavy body early draws a light one next.
                const bool dynamic = d.solve_policy == 3;
                const uint32_t groups = nthreads / G;
                const uint32_t rank = (threadIdx.x / G) * gridDim.x + blockIdx.x;
                uint32_t round = 0;
                uint32_t k = lo + rank;
                if (dynamic) {
                    uint32_t t = 0;
                    if (gl == 0) t = atomicAdd(claim, 1u);
                    k = lo + __shfl_sync(gmask, t, gbase);
                }
                Ahead ah{};
                if (k < hi) ah = fetch_ahead<G>(d, k, gl);
                while (k < hi) {
                    ++round;
                    uint32_t next = lo + round * groups + ((round & 1u) ? groups - 1u - rank : rank);
                    if (dynamic) {
                        uint32_t t = 0;
                        if (gl == 0) t = atomicAdd(claim, 1u);
                        next = lo + __shfl_sync(gmask, t, gbase);
                    }
                    const uint32_t kn = next < hi ? next : ~0u;
                    const uint32_t i = ah.i;
                    const bool skip = (phase != 0 && ah.impact == 0) ||
                                      (batched(d) && it >= d.scene_budget[d.scene_of[i]]);
                    if (skip) {
                        if (kn != ~0u) ah = fetch_ahead<G>(d, kn, gl);
                    } else {
                        solve_body_group<G, kJoints>(d, ah, kn, phase, dt, sm, gmask, gl, gbase, trace);
                    }
                    k = next;
                }
                __syncwarp();
            };
            if (rg.per_thread) {
                // A body per thread. Consecutive bodies go to consecutive
                // CTAs, as for the groups.
                if constexpr (kThread) {
                    Blk* slot = reinterpret_cast<Blk*>(warp_stage) + lane;
                    BodyView* views = reinterpret_cast<BodyView*>(warp_stage + kThreadViews) + 2 * lane;
                    for (uint32_t k = b0 + threadIdx.x * gridDim.x + blockIdx.x; k < b1; k += nthreads) {
                        const uint32_t i = d.corder[k];
                        if (phase != 0 && d.impact[i] == 0) continue;
                        if (batched(d) && it >= d.scene_budget[d.scene_of[i]]) continue;
                        solve_body_thread<kJoints>(d, i, phase, dt, slot, views);
                    }
                }
            }
            sweep(W32{}, b0, rg.r32);
            sweep(W16{}, rg.r32, rg.r16);
            sweep(W8{}, rg.r16, rg.r8);
            if (timing && it == 0 && col < 18) {
                __syncthreads();
                if (threadIdx.x == 0) atomicMax(&c->dbg_work[col], now());
            }
            if (!grid_sync(c, d.barrier_spins)) return;
            if (timing && it == 0 && col < 18 && blockIdx.x == 0 && threadIdx.x == 0) c->dbg_release[col] = now();
        }
        Res res{0.0, 0u, 0.0f, 0u, sp.tolerance};
        {
            // Each contact's bodies are loaded one contact ahead, so a
            // contact's body and row loads go out together.
            uint32_t k = grid_stride_begin();
            uint2 ab = k < n_con ? d.c_bodies[k] : make_uint2(0u, 0u);
            while (k < n_con) {
                const uint32_t kn = k + grid_stride();
                const uint2 abn = kn < n_con ? d.c_bodies[kn] : make_uint2(0u, 0u);
                dual_contact(d, k, ab, dt, phase, res, it);
                ab = abn;
                k = kn;
            }
        }
        if constexpr (kJoints) {
            BodyView* views = reinterpret_cast<BodyView*>(warp_stage + kThreadViews) + 2 * lane;
            JointRes* jres = reinterpret_cast<JointRes*>(warp_stage + kThreadJointRes) + lane;
            for (uint32_t j = grid_stride_begin(); j < d.nj; j += grid_stride())
                dual_joint(d, j, phase, dt, res, it, views, jres);
        }
        // Deterministic reduction: warp tree, warps in order, blocks in order.
        block_residual<kSolveThreads>(res, wsq, wn, wmx, wov, c, blockIdx.x);
        if (timing && it == 0 && threadIdx.x == 0) atomicMax(&c->dbg_work[19], now());
        if (!grid_sync(c, d.barrier_spins)) return;
        if (timing && it == 0 && blockIdx.x == 0 && threadIdx.x == 0) c->dbg_release[19] = now();
        const SweepResidual sw = sweep_residual(c, 0u, sp);
        if (phase == 0 && grid_stride_begin() == 0) c->residual_trace[it] = sw.measure;
        bool last = it + 1 == iters;
        if (adaptive && sw.met) last = true;
        // Every block has read the partials before the next pass rewrites them.
        if (!last && colors == 0 && !grid_sync(c, d.barrier_spins)) return;
        if (last) {
            if (grid_stride_begin() == 0) {
                c->claim[0] = c->claim[1] = 0u;  // every block is past its last claim
                if (phase == 0) {
                    c->iterations = it + 1;
                    c->residual = sw.rms;
                    c->residual_max = sw.mx;
                    c->residual_over = sw.over;
                }
                c->budget = it + 1;
            }
            return;
        }
    }
}

}  // namespace pmb

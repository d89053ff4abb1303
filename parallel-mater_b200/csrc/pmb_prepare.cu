// SPDX-License-Identifier: MIT
// AVBD prepare and the constraint graph.
//
// The reference prepares on one 128-thread block and builds the graph on
// lane 0 alone (geometry_constraints.slang:1213-1591). Here every part runs
// across the grid:
//   bodies    inertia blocks and the history-weighted gravity displacement
//   contacts  cold anchors, normal/tangent errors, warm-started duals
//   joints    row initialisation (visit_joint, init)
//   graph     per-body incident lists (CSR, descending pair index: the order
//             of the reference's head-inserted linked lists), islands by a
//             lock-free union-find that always hooks the larger root under
//             the smaller (so every root is its island's lowest index, as the
//             reference's serial union-find leaves it), impact marking
//   colours   the reference's first-fit greedy colouring in body-index order,
//             which gives body v the smallest colour absent among its
//             lower-index dynamic neighbours. That colouring is the unique
//             fixpoint of "colour(v) = mex(colours of lower neighbours)", so
//             a persistent kernel iterates that map from the previous tick's
//             colours until a round changes nothing: the result equals the
//             serial colouring exactly, in few rounds when the graph changed
//             little.
#include "pmb_joint.cuh"

namespace pmb {

__global__ void k_prepare_bodies(Dev d, StepParams sp) {
    const float dt = sp.dt;
    const V3 g{sp.gx, sp.gy, sp.gz};
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        const float4 pv = d.prev_vel[i];
        const V3 old_v = v3(pv);
        const bool hist = pv.w != 0.0f;
        d.parent[i] = i;
        d.impact[i] = 0;
        d.anchored[i] = 0;
        d.island_end[i] = 0;
        d.mean[i] = make_float4(0, 0, 0, 0);
        d.dq[i] = make_float4(0, 0, 0, 1);
        d.dxa[i] = make_float4(0, 0, 0, 0);
        d.deg[i] = 0;
        d.jdeg[i] = 0;
        d.inc_cursor[i] = 0;
        d.jinc_cursor[i] = 0;
        if (d.motion[i] != kDynamic) {
            d.color[i] = kInvalid;
            d.prev_vel[i] = make_float4(0, 0, 0, 0);
            d.dxl[i] = make_float4(0, 0, 0, 0);
            d.inA[i] = make_float4(0, 0, 0, 0);
            d.inB[i] = make_float4(0, 0, 0, 0);
            continue;
        }
        if (d.color[i] == kInvalid) d.color[i] = 0;
        const V3 vprev = v3(d.v[i]);
        float g2 = len2(g);
        V3 acc = mul(sub(vprev, old_v), 1.0f / dt);
        float wgt = hist && g2 > 0.0f ? fclamp(dot(acc, g) / g2, 0.0f, 1.0f) : 0.0f;
        if (!isfinite(wgt)) wgt = 0.0f;
        V3 corr = mul(g, -(1.0f - wgt) * dt * dt);
        d.dxl[i] = f4(corr);
        d.prev_vel[i] = f4(vprev, 1.0f);
        const float4 p0 = d.p0[i];
        const float mass = 1.0f / fmx(p0.x, 1.0e-12f);
        const Q4 q = q4(d.tq[i]);
        float h[6];  // h33 h43 h53 h44 h54 h55
        float inv[3] = {p0.y, p0.z, p0.w};
        for (unsigned ax = 0; ax < 3; ++ax) {
            V3 la = inv_rotate(q, unit_axis(ax));
            V3 col = rotate(q, V3{la.x / fmx(inv[0], 1.0e-12f), la.y / fmx(inv[1], 1.0e-12f),
                                  la.z / fmx(inv[2], 1.0e-12f)});
            for (unsigned r = ax; r < 3; ++r) {
                float v = comp(col, r) / (dt * dt);
                if (ax == 0) h[r] = v;
                else if (ax == 1) h[2 + r] = v;
                else h[5] = v;
            }
        }
        d.inA[i] = make_float4(mass / (dt * dt), h[0], h[1], h[3]);
        d.inB[i] = make_float4(h[2], h[4], h[5], 0.0f);
    }
}

__device__ __forceinline__ float pair_stiffness(float ima, float imb, float dt) {
    return 1.0f / (fmx(ima + imb, 1.0e-6f) * dt * dt);
}

// geometry_constraints.slang:1297-1389 and the impact test :983-1006.
__global__ void k_prepare_pairs(Dev d, StepParams sp) {
    const float dt = sp.dt;
    const bool realtime = sp.realtime != 0;
    const uint32_t n_act = d.ctr->n_act;
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t a = d.act_a[i], b = d.act_b[i];
        const float4 pa0 = d.p0[a], pb0 = d.p0[b], pa1 = d.p1[a], pb1 = d.p1[b], pa2 = d.p2[a], pb2 = d.p2[b];
        const float penalty = pair_stiffness(pa0.x, pb0.x, dt);
        const V3 xa0 = v3(d.x[a]), xb0 = v3(d.x[b]), xa = v3(d.tx[a]), xb = v3(d.tx[b]);
        const Q4 qa0 = q4(d.q[a]), qb0 = q4(d.q[b]), qa = q4(d.tq[a]), qb = q4(d.tq[b]);
        // rigid_avbd_contact_skin (geometry_constraints.slang:438-446): a
        // guided pair's contacts rest at the guided offset.
        const bool guided =
            d.nj && frames_guided(__float_as_uint(d.frame[a].w), __float_as_uint(d.frame[b].w));
        const float skin = fmn(pa2.z + pb2.z, guided ? 1.0e-4f : 1.0e-3f) + 2.0f * 1.0e-5f;
        const V3 mo_a = sub(xa, xa0), mo_b = sub(xb, xb0);
        const V3 an_a = mul(delta_velocity(qa0, qa, dt), dt);
        const V3 an_b = mul(delta_velocity(qb0, qb, dt), dt);
        const uint32_t off = d.act_off[i], cnt = d.act_cnt[i];
        bool impact = false;
        for (uint32_t p = 0; p < cnt; ++p) {
            const uint32_t c = off + p;
            const float4 n4 = d.c_n[c], p4 = d.c_p[c];
            float4 aa = d.c_aa[c], ab = d.c_ab[c];
            const bool cached = aa.w != 0.0f;
            const V3 n = v3(n4), pt = v3(p4);
            const float pen = n4.w;
            V3 anc_a = v3(aa), anc_b = v3(ab);
            if (!cached) {
                anc_a = inv_rotate(qa0, sub(pt, xa0));
                anc_b = inv_rotate(qb0, sub(pt, xb0));
                d.c_aa[c] = f4(anc_a, 0.0f);
                d.c_ab[c] = f4(anc_b, 0.0f);
            }
            const V3 arm_a = sub(pt, xa), arm_b = sub(pt, xb);
            const float closing = dot(n, sub(add(mo_b, cross(an_b, arm_b)), add(mo_a, cross(an_a, arm_a))));
            const float old_pen = pen - closing;
            V3 t0, t1;
            basis(n, t0, t1);
            const V3 anchor_motion = add(sub(mo_b, mo_a), sub(rotation_displacement(qb0, qb, anc_b),
                                                              rotation_displacement(qa0, qa, anc_a)));
            const V3 old_delta = !cached ? V3{0, 0, 0}
                                         : add(sub(xb0, xa0), sub(rotate(qb0, anc_b), rotate(qa0, anc_a)));
            const V3 terr = add(anchor_motion, mul(old_delta, 1.0f - kAlpha));
            const float speed = -closing / dt;
            const float impact_disp = realtime && !cached && speed < -0.1f
                                          ? -(1.0f + fmn(pa1.y, pb1.y)) * speed * dt
                                          : 0.0f;
            const V3 err{pen - fclamp(old_pen, 0.0f, skin) + impact_disp, dot(terr, t0), dot(terr, t1)};
            d.c_e[c] = f4(err, speed);
            float4 lam = d.c_lam[c], pk = d.c_pen[c];
            Dual du[3];
            if (cached) {
                du[0] = {lam.x, pk.x};
                du[1] = {lam.y, pk.y};
                du[2] = {lam.z, pk.z};
            } else {
                du[0] = du[1] = du[2] = {0.0f, penalty};
            }
            for (int x = 0; x < 3; ++x) du[x] = warm_start(du[x], kMaxPenalty);
            const float plain_lambda = du[0].lambda;
            if (sp.warm_start == 2 && c < d.warm_count) {
                // Per row: a negative lambda or a non-positive penalty keeps
                // the plain value of that half (friction lambdas are signed;
                // NaN keeps them).
                const float4 tl = d.warm_table[2 * size_t(c)], tk = d.warm_table[2 * size_t(c) + 1];
                const float tla[3] = {tl.x, tl.y, tl.z}, tka[3] = {tk.x, tk.y, tk.z};
                for (uint32_t x = 0; x < d.warm_rows; ++x) {
                    if (x == 0 ? tla[0] >= 0.0f : tla[x] == tla[x]) du[x].lambda = tla[x];
                    if (tka[x] > 0.0f) du[x].penalty = tka[x];
                }
            }
            d.c_lam[c] = make_float4(du[0].lambda, du[1].lambda, du[2].lambda, lam.w);
            d.c_pen[c] = make_float4(du[0].penalty, du[1].penalty, du[2].penalty, 0.0f);
            const float impact_fraction = p4.w;
            bool fresh = (!cached || plain_lambda <= 1.0e-6f || (impact_fraction > 0.0f && impact_fraction < 1.0f)) &&
                         speed < -0.1f && pen >= -1.0e-5f;
            float prev_pen = pen + speed * dt;
            impact = impact || fresh || prev_pen > skin + 1.0e-4f;
        }
        d.act_impact[i] = impact ? 1u : 0u;
    }
}

__global__ void k_prepare_joints(Dev d, StepParams sp) {
    const float dt = sp.dt;
    for (uint32_t j = grid_stride_begin(); j < d.nj; j += grid_stride()) {
        JointState st = d.jstate[j];
        const Joint& o = d.joints[j];
        st.count = 0;
        st.enabled = (o.enabled != 0 && st.broken == 0) ? 1u : 0u;
        if (st.enabled) {
            st.applied = 0.0f;
            st.dense_a = o.body_a < d.n ? o.body_a : kInvalid;
            st.dense_b = o.body_b < d.n ? o.body_b : kInvalid;
            if (st.dense_a != kInvalid && st.dense_b != kInvalid) {
                const uint32_t a = st.dense_a, b = st.dense_b;
                BodyView A = load_body(d, a), B = load_body(d, b);
                Blk scratch{};
                uint32_t count = 0;
                visit_joint(o, d.jrows + size_t(j) * 18, A, B, v3(d.x[a]), q4(d.q[a]), v3(d.x[b]), q4(d.q[b]),
                            d.p0[a], d.p0[b], dt, &scratch, true, kVisitInit, &count);
                st.count = count;
            }
        }
        d.jstate[j] = st;
    }
}

// ---------------------------------------------------------------- graph
// Lock-free union-find over parent[] with parent[i] <= i: finds shorten paths
// in place, unions hook the larger root under the smaller by CAS.
__device__ uint32_t uf_find(uint32_t* parent, uint32_t i) {
    volatile uint32_t* P = parent;
    uint32_t cur = P[i];
    if (cur != i) {
        uint32_t prev = i, next;
        while (cur > (next = P[cur])) {
            P[prev] = next;
            prev = cur;
            cur = next;
        }
    }
    return cur;
}
__device__ void uf_unite(uint32_t* parent, uint32_t a, uint32_t b) {
    uint32_t ra = uf_find(parent, a), rb = uf_find(parent, b);
    for (int guard = 0; guard < (1 << 24) && ra != rb; ++guard) {
        if (ra < rb) {
            uint32_t old = atomicCAS(&parent[rb], rb, ra);
            if (old == rb) return;
            rb = old;
        } else {
            uint32_t old = atomicCAS(&parent[ra], ra, rb);
            if (old == ra) return;
            ra = old;
        }
    }
}

__global__ void k_graph_degrees(Dev d, StepParams sp) {
    const uint32_t n_act = d.ctr->n_act;
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t a = d.act_a[i], b = d.act_b[i];
        const bool da = d.motion[a] == kDynamic, db = d.motion[b] == kDynamic;
        if (da) atomicAdd(&d.deg[a], 1u);
        if (db) atomicAdd(&d.deg[b], 1u);
        if (da && db) uf_unite(d.parent, a, b);
        if (d.act_impact[i]) d.ctr->impact = 1;
    }
    for (uint32_t j = grid_stride_begin(); j < d.nj; j += grid_stride()) {
        const JointState st = d.jstate[j];
        if (st.count == 0) continue;
        const uint32_t a = st.dense_a, b = st.dense_b;
        const bool da = d.motion[a] == kDynamic, db = d.motion[b] == kDynamic;
        if (da) atomicAdd(&d.jdeg[a], 1u);
        if (db) atomicAdd(&d.jdeg[b], 1u);
        if (da && db) uf_unite(d.parent, a, b);
        if (!sp.realtime && sp.requested == 0) atomicMax(&d.ctr->joint_iters, d.joints[j].solver_iterations);
        if (batched(d)) atomicMax(&d.scene_jiters[d.scene_of[a]], d.joints[j].solver_iterations);
    }
}

// Sweeps of every scene of a batched world, with the whole-world rule of
// k_solve applied per scene: the realtime profile sweeps 8 times; legacy
// sweeps the scene's requested iterations (or the tick's), else the base
// budget raised by the scene's largest joint iteration hint. Also clears the
// scene's residual accumulators and joint hints for the next tick.
__global__ void k_scene_budgets(Dev d, StepParams sp) {
    for (uint32_t s = grid_stride_begin(); s < d.n_scenes; s += grid_stride()) {
        const uint32_t req = d.scene_iters[s] ? d.scene_iters[s] : sp.requested;
        uint32_t budget = sp.realtime ? 8u : (req ? req : sp.budget_request);
        if (!sp.realtime && req == 0) budget = max(budget, d.scene_jiters[s]);
        budget = min(max(budget, 1u), kMaxIterations);
        d.scene_budget[s] = budget;
        d.scene_jiters[s] = 0;
        d.scene_res_sq[s] = 0.0f;
        d.scene_res_mx[s] = 0.0f;
        d.scene_res_n[s] = 0;
        atomicMax(&d.ctr->budget_max, budget);
    }
}
void launch_scene_budgets(const Dev& d, const StepParams& sp, cudaStream_t s) {
    if (d.n_scenes <= 1) return;
    k_scene_budgets<<<blocks_for(d.n_scenes), kBlock, 0, s>>>(d, sp);
    note_launch(blocks_for(d.n_scenes));
}

__global__ void k_graph_fill(Dev d) {
    const uint32_t n_act = d.ctr->n_act;
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t a = d.act_a[i], b = d.act_b[i];
        if (d.motion[a] == kDynamic) d.inc_list[d.inc_off[a] + atomicAdd(&d.inc_cursor[a], 1u)] = i;
        if (d.motion[b] == kDynamic) d.inc_list[d.inc_off[b] + atomicAdd(&d.inc_cursor[b], 1u)] = i;
    }
    for (uint32_t j = grid_stride_begin(); j < d.nj; j += grid_stride()) {
        const JointState st = d.jstate[j];
        if (st.count == 0) continue;
        const uint32_t a = st.dense_a, b = st.dense_b;
        if (d.motion[a] == kDynamic) d.jinc_list[d.jinc_off[a] + atomicAdd(&d.jinc_cursor[a], 1u)] = j;
        if (d.motion[b] == kDynamic) d.jinc_list[d.jinc_off[b] + atomicAdd(&d.jinc_cursor[b], 1u)] = j;
    }
}

__device__ __forceinline__ void sort_desc(uint32_t* seg, uint32_t n) {
    for (uint32_t i = 1; i < n; ++i) {
        uint32_t v = seg[i], j = i;
        while (j > 0 && seg[j - 1] < v) {
            seg[j] = seg[j - 1];
            --j;
        }
        seg[j] = v;
    }
}

// Sort lists; find every root. Concurrent finds may still shorten paths
// (writing ancestors), so roots go to a scratch array (corder, refilled by the
// colour pass later) and are published by a second kernel.
__global__ void k_graph_lists(Dev d) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        sort_desc(d.inc_list + d.inc_off[i], d.deg[i]);
        sort_desc(d.jinc_list + d.jinc_off[i], d.jdeg[i]);
        d.corder[i] = uf_find(d.parent, i);
    }
}
__global__ void k_graph_roots(Dev d) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        d.parent[i] = d.corder[i];
        uint32_t rc = 0;
        const uint32_t lo = d.inc_off[i], n = d.deg[i];
        for (uint32_t k = 0; k < n; ++k) rc += d.act_cnt[d.inc_list[lo + k]];
        d.rcount[i] = rc;
    }
}

// Flattened contact list per body, in the reference's visiting order
// (incident pairs by descending index, points in manifold order).
__global__ void k_row_lists(Dev d) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        uint32_t pos = d.roff[i];
        const uint32_t lo = d.inc_off[i], n = d.deg[i];
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t p = d.inc_list[lo + k];
            const uint32_t a = d.act_a[p], b = d.act_b[p];
            const uint32_t second = a == i ? 0u : 0x80000000u;
            const uint32_t other = a == i ? b : a;
            const uint32_t off = d.act_off[p], cnt = d.act_cnt[p];
            for (uint32_t q = 0; q < cnt; ++q) {
                d.bother[pos] = other;
                d.blist[pos++] = (off + q) | second;
            }
        }
    }
}

__global__ void k_graph_impact(Dev d) {
    const uint32_t n_act = d.ctr->n_act;
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        if (!d.act_impact[i]) continue;
        const uint32_t a = d.act_a[i], b = d.act_b[i];
        if (d.motion[a] == kDynamic) d.impact[d.parent[a]] = 1;
        if (d.motion[b] == kDynamic) d.impact[d.parent[b]] = 1;
    }
}

__global__ void k_graph_islands(Dev d) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        if (d.motion[i] != kDynamic) continue;
        const uint32_t r = d.parent[i];
        atomicMax(&d.island_end[r], i);
        if (r != i) d.impact[i] = d.impact[r];
        if (r == i && (d.deg[i] > 0 || d.jdeg[i] > 0)) atomicAdd(&d.ctr->islands, 1u);
    }
}

// Colour fixpoint (persistent cooperative kernel).
__device__ __forceinline__ uint32_t mex_lower(const Dev& d, uint32_t v, bool& overflow) {
    uint64_t mask[4] = {0, 0, 0, 0};
    const uint32_t base = d.inc_off[v] + d.jinc_off[v], nl = d.nlow[v];
    for (uint32_t k = 0; k < nl; ++k) {
        const uint32_t c = ((volatile uint32_t*)d.color)[d.nbr[base + k]];
        if (c < kMaxColors) mask[c >> 6] |= 1ull << (c & 63);
    }
    for (int w = 0; w < 4; ++w)
        if (~mask[w]) return uint32_t(w * 64 + __ffsll((long long)~mask[w]) - 1);
    overflow = true;
    return kMaxColors - 1;
}

// Each body's dynamic neighbours through contacts and joints, for the colour
// rounds: lower-indexed ones from the front of its segment (nlow of them),
// higher-indexed ones from the back (nhigh). Segment base = inc_off + jinc_off
// (room for deg + jdeg entries).
__global__ void k_neighbour_lists(Dev d) {
    for (uint32_t v = grid_stride_begin(); v < d.n; v += grid_stride()) {
        if (d.motion[v] != kDynamic) continue;
        const uint32_t base = d.inc_off[v] + d.jinc_off[v], len = d.deg[v] + d.jdeg[v];
        uint32_t lo = 0, hi = 0;
        auto add = [&](uint32_t u) {
            if (d.motion[u] != kDynamic || u == v) return;
            if (u < v) d.nbr[base + lo++] = u;
            else d.nbr[base + len - 1 - hi++] = u;
        };
        const uint32_t so = d.inc_off[v], sn = d.deg[v];
        for (uint32_t k = 0; k < sn; ++k) {
            const uint32_t p = d.inc_list[so + k];
            const uint32_t a = d.act_a[p], b = d.act_b[p];
            add(a == v ? b : a);
        }
        const uint32_t jo = d.jinc_off[v], jn = d.jdeg[v];
        for (uint32_t k = 0; k < jn; ++k) {
            const JointState st = d.jstate[d.jinc_list[jo + k]];
            add(st.dense_a == v ? st.dense_b : st.dense_a);
        }
        d.nlow[v] = lo;
        d.nhigh[v] = hi;
    }
}

// Mark v's higher-indexed dynamic neighbours for the next round: only their
// mex can depend on v's colour.
__device__ __forceinline__ void mark_higher(const Dev& d, uint32_t v, uint8_t* next) {
    const uint32_t end = d.inc_off[v] + d.jinc_off[v] + d.deg[v] + d.jdeg[v];
    for (uint32_t k = end - d.nhigh[v]; k < end; ++k) next[d.nbr[k]] = 1;
}

// Jacobi rounds towards the greedy colouring in index order (colour of v =
// smallest colour absent among its lower-indexed neighbours), warm-started
// from last tick's colours. Round 0 visits every body; later rounds only
// those with a lower neighbour that changed in the round before (the only
// bodies whose mex can change), so the fixpoint is the same.
__global__ void __launch_bounds__(kColorThreads) k_color(Dev d) {
    Counters* c = d.ctr;
    if (c->status & kStBarrierTimeout) return;  // the tick was abandoned
    // The change counter is read by one thread per block and shared: a read
    // by every thread of the grid per round piles onto one L2 line.
    __shared__ uint32_t s_before, s_after;
    for (uint32_t round = 0; round < d.n + 2; ++round) {
        if (threadIdx.x == 0) s_before = ((volatile uint32_t*)&c->changed)[0];
        if (!grid_sync(c, d.barrier_spins)) return;
        const uint32_t before = s_before;
        uint8_t* cur = d.cdirty + size_t(round & 1u) * d.n;
        uint8_t* next = d.cdirty + size_t((round + 1u) & 1u) * d.n;
        bool transient = false;  // a mex past 255 in this round (judged at the fixpoint)
        uint32_t changes = 0;
        for (uint32_t v = grid_stride_begin(); v < d.n; v += grid_stride()) {
            if (round != 0) {
                if (!cur[v]) continue;
                cur[v] = 0;
            }
            if (d.motion[v] != kDynamic) continue;
            uint32_t col = mex_lower(d, v, transient);
            if (col != d.color[v]) {
                ((volatile uint32_t*)d.color)[v] = col;
                ++changes;
                mark_higher(d, v, next);
            }
        }
        changes = __reduce_add_sync(0xffffffffu, changes);  // one atomic per warp
        if (changes && (threadIdx.x & 31) == 0) atomicAdd(&c->changed, changes);
        if (!grid_sync(c, d.barrier_spins)) return;
        if (threadIdx.x == 0) s_after = ((volatile uint32_t*)&c->changed)[0];
        __syncthreads();
        const uint32_t after = s_after;
        if (after == before) {
            // Converged. A body's mex can pass 255 colours in an intermediate
            // round and still settle below 256, so overflow is judged on the
            // final colours: a body left at the last colour whose lower
            // neighbours still use every colour below it.
            bool final_overflow = false;
            for (uint32_t v = grid_stride_begin(); v < d.n; v += grid_stride())
                if (d.motion[v] == kDynamic && d.color[v] == kMaxColors - 1) mex_lower(d, v, final_overflow);
            if (final_overflow) atomicOr(&c->status, kStColorOverflow);
            if (grid_stride_begin() == 0) c->rounds = round + 1;
            return;
        }
    }
    if (grid_stride_begin() == 0) atomicOr(&c->status, kStColorOverflow);
}

__global__ void k_color_count(Dev d) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        if (d.motion[i] != kDynamic) continue;
        const uint32_t col = d.color[i];
        atomicAdd(&d.ctr->color_count[col * kSortClasses + sort_class(d.rcount[i])], 1u);
        atomicMax(&d.ctr->colors, col + 1);
    }
}

// Exclusive scan of the bucket counts (one block, kPer consecutive buckets
// per thread); counts become cursors.
constexpr uint32_t kBuckets = kMaxColors * kSortClasses;
constexpr uint32_t kPer = (kBuckets + 1023) / 1024;
__global__ void __launch_bounds__(1024) k_color_offsets(Dev d) {
    __shared__ uint32_t part[32];
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    uint32_t v[kPer], sum = 0;
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
        const uint32_t b = t * kPer + k;
        v[k] = b < kBuckets ? d.ctr->color_count[b] : 0u;
        sum += v[k];
    }
    uint32_t x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= uint32_t(o)) x += y;
    }
    if (lane == 31) part[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t p = part[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, p, o);
            if (lane >= uint32_t(o)) p += y;
        }
        part[lane] = p;
    }
    __syncthreads();
    uint32_t run = x - sum + (warp ? part[warp - 1] : 0u);  // exclusive prefix of this thread's first bucket
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
        const uint32_t b = t * kPer + k;
        if (b < kBuckets) {
            d.ctr->color_off[b] = run;
            d.ctr->color_count[b] = 0;
        }
        run += v[k];
        if (b == kBuckets - 1) d.ctr->color_off[kBuckets] = run;
    }
}

__global__ void k_color_scatter(Dev d) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        if (d.motion[i] != kDynamic) continue;
        const uint32_t b = d.color[i] * kSortClasses + sort_class(d.rcount[i]);
        const uint32_t slot = d.ctr->color_off[b] + atomicAdd(&d.ctr->color_count[b], 1u);
        d.corder[slot] = i;
        d.crec[slot] = make_uint4(i, d.roff[i], d.rcount[i], d.impact[i]);
    }
}

void launch_prepare(const Dev& d, const StepParams& sp, cudaStream_t s) {
    k_prepare_bodies<<<blocks_for(d.n), kBlock, 0, s>>>(d, sp);
    note_launch(blocks_for(d.n));
    k_prepare_pairs<<<cap_blocks(d.cap_pair, 128), 128, 0, s>>>(d, sp);
    note_launch(cap_blocks(d.cap_pair, 128));
    if (d.nj) {
        k_prepare_joints<<<blocks_for(d.nj, 64), 64, 0, s>>>(d, sp);
        note_launch(blocks_for(d.nj, 64));
    }
    launch_contact_jacobians(d, 0, sp.dt, s);
    prof_mark(s, "prepare");
}

const void* color_kernel_ptr = reinterpret_cast<const void*>(&k_color);

void launch_graph(const Dev& d, const StepParams& sp, cudaStream_t s, int coop_blocks) {
    uint32_t gb = cap_blocks(d.cap_pair > d.nj ? d.cap_pair : d.nj);
    k_graph_degrees<<<gb, kBlock, 0, s>>>(d, sp);
    note_launch(gb);
    scan_u32(d.deg, d.inc_off, nullptr, d.n, nullptr, d.scan_tmp32, s);
    scan_u32(d.jdeg, d.jinc_off, nullptr, d.n, nullptr, d.scan_tmp32, s);
    k_graph_fill<<<gb, kBlock, 0, s>>>(d);
    note_launch(gb);
    k_graph_lists<<<blocks_for(d.n), kBlock, 0, s>>>(d);
    note_launch(blocks_for(d.n));
    k_graph_roots<<<blocks_for(d.n), kBlock, 0, s>>>(d);
    note_launch(blocks_for(d.n));
    scan_u32(d.rcount, d.roff, nullptr, d.n, nullptr, d.scan_tmp32, s);
    k_row_lists<<<blocks_for(d.n), kBlock, 0, s>>>(d);
    note_launch(blocks_for(d.n));
    k_graph_impact<<<cap_blocks(d.cap_pair), kBlock, 0, s>>>(d);
    note_launch(cap_blocks(d.cap_pair));
    k_graph_islands<<<blocks_for(d.n), kBlock, 0, s>>>(d);
    note_launch(blocks_for(d.n));
    prof_mark(s, "graph lists+islands");
    k_neighbour_lists<<<blocks_for(d.n), kBlock, 0, s>>>(d);
    note_launch(blocks_for(d.n));
    cudaMemsetAsync(d.cdirty, 0, 2 * size_t(d.n), s);
    void* args[] = {const_cast<Dev*>(&d)};
    cudaLaunchCooperativeKernel(color_kernel_ptr, dim3(coop_blocks), dim3(kColorThreads), args, 0, s);
    note_launch(coop_blocks);
    prof_mark(s, "colour fixpoint");
    k_color_count<<<blocks_for(d.n), kBlock, 0, s>>>(d);
    note_launch(blocks_for(d.n));
    static_assert(kPer * 1024 >= kBuckets, "bucket scan is one block");
    k_color_offsets<<<1, 1024, 0, s>>>(d);
    note_launch(1);
    k_color_scatter<<<blocks_for(d.n), kBlock, 0, s>>>(d);
    note_launch(blocks_for(d.n));
    prof_mark(s, "colour buckets");
}

}  // namespace pmb

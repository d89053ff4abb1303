// SPDX-License-Identifier: MIT
// AVBD solve (geometry_constraints_solve.slang:211-847) as one persistent
// cooperative kernel per phase: for each iteration, one grid-wide pass per
// colour (every body of that colour gathers its contact and joint rows into a
// register-resident 6x6 block and solves it by LDL^T, with the crossing
// safeguard), then one pass over contacts and joints for the duals, separated
// by bounded grid barriers. The dual pass also reduces the residual (largest
// remaining normal-row violation, and |C| of hard joint rows), so the
// residual-driven schedule can stop without a host round trip. The reference's
// last-iteration work (accumulated impulses, re-anchoring sliding contacts) is
// applied after the loop from the final duals and the stick flag each dual
// pass stores, which is the same arithmetic on the same values.
#include "pmb_solve_common.cuh"

namespace pmb {

// The position phase also forms each contact's friction and penalty growth
// factor (c_mub, from its bodies' materials and masses); the velocity phase
// its force offsets (the row forces are the projected trial forces less
// them): the normal impulse and the accumulated friction of the position
// phase, both fixed by then (k_contact_finalize), over dt.
__global__ void k_contact_jacobians(Dev d, uint32_t phase, float dt) {
    if (phase != 0 && d.ctr->impact == 0) return;
    const uint32_t n_con = d.ctr->n_contacts;
    for (uint32_t c = grid_stride_begin(); c < n_con; c += grid_stride()) {
        const uint2 ab = d.c_bodies[c];
        V6 ja[3], jb[3];
        contact_jacobians(v3(d.c_n[c]), v3(d.c_p[c]), v3(d.c_aa[c]), v3(d.c_ab[c]), v3(d.tx[ab.x]), q4(d.tq[ab.x]),
                          v3(d.tx[ab.y]), q4(d.tq[ab.y]), ja, jb);
        float f[36];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                f[6 * r + k] = ja[r].v[k];
                f[18 + 6 * r + k] = jb[r].v[k];
            }
        float4* p = d.c_jac + size_t(c) * 9;
#pragma unroll
        for (int k = 0; k < 9; ++k) p[k] = make_float4(f[4 * k], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]);
        if (phase == 0) {
            const uint32_t a = ab.x, b = ab.y;
            const float friction = sqrtf(d.p1[a].x * d.p1[b].x);
            const float beta = (1.0f / (fmx(d.p0[a].x + d.p0[b].x, 1.0e-6f) * dt * dt)) * 100.0f;
            d.c_mub[c] = make_float2(friction, beta);
        } else {
            V3 t0, t1;
            basis(v3(d.c_n[c]), t0, t1);
            const V3 af = v3(d.c_accf[c]);
            d.c_foff[c] = make_float4(d.c_lam[c].w / dt, dot(af, t0) / dt, dot(af, t1) / dt, 0.0f);
        }
    }
}
void launch_contact_jacobians(const Dev& d, uint32_t phase, float dt, cudaStream_t s) {
    k_contact_jacobians<<<cap_blocks(d.cap_contact), kBlock, 0, s>>>(d, phase, dt);
    note_launch(cap_blocks(d.cap_contact));
}

// ------------------------------------------------------------ staged solve
// The same sweep as k_solve, organised for memory-level parallelism and with
// the dual update fused into the colour passes:
//
//  * Per colour, each CTA takes its bodies (round-robin over CTAs) in batches
//    that fit a shared-memory row stage. All threads of the CTA first stage
//    every contact row of the batch -- one thread per row, every global load
//    independent -- then groups of G lanes accumulate each body's block from
//    the staged rows in list order (the serial loop's additions, in its
//    order), solve it, apply the crossing safeguard from the staged normal
//    rows and write the update.
//  * A contact's dual update (geometry_constraints_solve.slang:494-532) needs
//    only its two bodies' displacements after the sweep, and once the body
//    with the later colour has solved, neither body changes again in the
//    sweep and no other body reads the contact. So the group that solves the
//    later body (or the only dynamic one) updates the contact's duals right
//    away from the staged row; joints likewise. Every contact and joint is
//    updated exactly once per sweep, from the same values as the separate
//    dual pass of k_solve, so the results are bit-identical; the dual pass,
//    its grid barrier and its second read of every contact disappear.
//  * The residual partials of each block are written before the last colour's
//    barrier (double-buffered by sweep parity), so the stop decision needs no
//    barrier of its own.
constexpr uint32_t kStageRows = 1024;      // staged contact rows per batch
constexpr uint32_t kBatchBodies = 256;     // bodies per batch
// Staged row record (floats; u32 fields stored as bits).
enum : uint32_t {
    kRJ = 0,          // this body's jacobian rows n, t0, t1 (3 x 6)
    kRSt = 18,        // stiffness: raw penalty x stiffness scale (3)
    kRForce = 21,     // force of each row (3)
    kRLam = 24,       // raw lambda xyz and w (4)
    kRPen = 28,       // raw penalty xyz (3)
    kRPre = 31,       // error terms summed before this body's jacobian product (3)
    kRPost = 34,      // ... and after it (3; first body of the contact only)
    kRFric = 37,      // friction sqrt(mu_a mu_b)
    kRBeta = 38,      // penalty growth factor of the pair
    kRTrial = 39,     // normal trial force at the start of the colour
    kRContact = 40,   // contact index
    kRFlags = 41,     // bit 0: this body is the contact's first body; bit 1: its dual is updated
                      // here; bit 2: the row crosses (crossing safeguard, set by the body's group)
    kRowWords = 43,   // odd: consecutive rows start in different shared-memory banks
};
static_assert(sizeof(GroupRows<32>) <= size_t(kStageRows) * kRowWords * 4, "oversized-body rows fit the stage");
constexpr uint32_t kStagedGroups = 64;  // lane groups per CTA at most (512 threads, 8 lanes)
constexpr size_t kStagedSmem =
    size_t(kStageRows) * kRowWords * 4 + size_t(kBatchBodies) * 10 * 4 + 64 * 4 + kStagedGroups * sizeof(Blk) +
    kStagedGroups * 2 * sizeof(BodyView);

struct StageTables {
    float* rows;       // kStageRows x kRowWords
    uint32_t* body;    // per batch slot: body index
    uint32_t* skip;    // per batch slot: 1 = not solved this sweep (impact phase, finished scene)
    uint32_t* off;     // kBatchBodies + 1 row offsets
    float* dx;         // per batch slot: displacement (6)
    uint32_t* scratch; // 64 words for scans and counts
    Blk* jblk;         // per lane group: the block while joint rows are added
    BodyView* jview;   // per lane group: the visited joint's two bodies
};
__device__ __forceinline__ StageTables stage_tables(uint8_t* raw) {
    StageTables t;
    t.rows = reinterpret_cast<float*>(raw);
    uint32_t* u = reinterpret_cast<uint32_t*>(raw + size_t(kStageRows) * kRowWords * 4);
    t.body = u;
    t.skip = u + kBatchBodies;
    t.off = u + 2 * kBatchBodies;            // kBatchBodies + 1 (one word of slack)
    t.dx = reinterpret_cast<float*>(u + 3 * kBatchBodies + 1);
    t.scratch = reinterpret_cast<uint32_t*>(t.dx + 6 * kBatchBodies);
    t.jblk = reinterpret_cast<Blk*>(t.scratch + 64);
    t.jview = reinterpret_cast<BodyView*>(t.jblk + kStagedGroups);
    return t;
}

// Stage contact row r (flat index t) of batch slot sl into the row table.
__device__ __forceinline__ void stage_row(const Dev& d, const StageTables& tb, uint32_t t, uint32_t sl, uint32_t r,
                                          uint32_t col, uint32_t phase, float dt) {
    const uint32_t i = tb.body[sl];
    const uint32_t ro = d.roff[i] + r;
    const uint32_t code = d.blist[ro], other = d.bother[ro];
    const uint32_t c = code & 0x7fffffffu;
    const bool first = (code >> 31) == 0;
    V6 me;
#pragma unroll
    for (int k = 0; k < 6; ++k) me.v[k] = tb.dx[6 * sl + k];
    const Lite o = load_lite(d, other);
    const uint32_t ocol = d.color[other];
    const float4 lam = d.c_lam[c], pen = d.c_pen[c], e = d.c_e[c];
    V6 ja[3], jb[3];
    load_jac(d, c, ja, jb);
    const float2 mub = d.c_mub[c];
    const float friction = mub.x, beta = mub.y;
    const float e3[3] = {e.x, e.y, e.z};
    float err[3], pre[3], post[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        // err = e + J_a . dx_a + J_b . dx_b, in that order (contact_rows).
        if (first) {
            pre[k] = e3[k];
            post[k] = dot6(jb[k], o.dx);
            err[k] = (pre[k] + dot6(ja[k], me)) + post[k];
        } else {
            pre[k] = e3[k] + dot6(ja[k], o.dx);
            post[k] = 0.0f;
            err[k] = pre[k] + dot6(jb[k], me);
        }
    }
    const F3 trial{lam.x + pen.x * err[0], lam.y + pen.y * err[1], lam.z + pen.z * err[2]};
    F3 f, sc;
    project_with_scales(trial, friction, f, sc);
    float forces[3] = {f.n, f.t0, f.t1};
    if (phase != 0) {
        const float4 fo = d.c_foff[c];
        forces[0] = f.n - fo.x;
        forces[1] = f.t0 - fo.y;
        forces[2] = f.t1 - fo.z;
    }
    float* row = tb.rows + size_t(t) * kRowWords;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        // Selected element by element (no run-time reference into either array).
#pragma unroll
        for (int k = 0; k < 6; ++k) row[kRJ + 6 * x + k] = first ? ja[x].v[k] : jb[x].v[k];
    }
    row[kRSt + 0] = pen.x * sc.n;
    row[kRSt + 1] = pen.y * sc.t0;
    row[kRSt + 2] = pen.z * sc.t1;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        row[kRForce + x] = forces[x];
        row[kRPre + x] = pre[x];
        row[kRPost + x] = post[x];
    }
    row[kRLam + 0] = lam.x;
    row[kRLam + 1] = lam.y;
    row[kRLam + 2] = lam.z;
    row[kRLam + 3] = lam.w;
    row[kRPen + 0] = pen.x;
    row[kRPen + 1] = pen.y;
    row[kRPen + 2] = pen.z;
    row[kRFric] = friction;
    row[kRBeta] = beta;
    row[kRTrial] = trial.n;
    // The dual is updated here when the other body is not dynamic (no
    // colour) or solved in an earlier colour of the sweep.
    const bool owned = ocol == kInvalid || ocol < col;
    row[kRContact] = __uint_as_float(c);
    row[kRFlags] = __uint_as_float((first ? 1u : 0u) | (owned ? 2u : 0u));
}

// The dual update of one staged contact row with the body's displacement
// after its solve (dual_contact's arithmetic, values from the stage).
__device__ __forceinline__ void staged_dual(const Dev& d, const float* row, const V6& me, uint32_t scene,
                                            bool scene_last, Res& res) {
    const uint32_t flags = __float_as_uint(row[kRFlags]);
    const bool first = flags & 1u;
    const uint32_t c = __float_as_uint(row[kRContact]);
    float err[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        V6 j;
#pragma unroll
        for (int q = 0; q < 6; ++q) j.v[q] = row[kRJ + 6 * k + q];
        err[k] = first ? (row[kRPre + k] + dot6(j, me)) + row[kRPost + k] : row[kRPre + k] + dot6(j, me);
    }
    const float friction = row[kRFric], beta = row[kRBeta];
    float4 lam = make_float4(row[kRLam], row[kRLam + 1], row[kRLam + 2], row[kRLam + 3]);
    float4 pen = make_float4(row[kRPen], row[kRPen + 1], row[kRPen + 2], 0.0f);
    F3 f = project_contact(F3{lam.x + pen.x * err[0], lam.y + pen.y * err[1], lam.z + pen.z * err[2]}, friction);
    const float tx = lam.y + pen.y * err[1];
    const float ty = lam.z + pen.z * err[2];
    const float bound = friction * f.n;
    const bool stick = tx * tx + ty * ty <= bound * bound;
    lam.x = f.n;
    lam.y = f.t0;
    lam.z = f.t1;
    if (f.n > 0.0f) pen.x = fmn(kMaxPenalty, pen.x + beta * fab(err[0]));
    if (stick) {
        pen.y = fmn(kMaxPenalty, pen.y + beta * fab(err[1]));
        pen.z = fmn(kMaxPenalty, pen.z + beta * fab(err[2]));
    }
    pen.w = stick ? 1.0f : 0.0f;
    d.c_lam[c] = lam;
    d.c_pen[c] = pen;
    if (f.n > 0.0f || err[0] > 0.0f) {
        const float v = f.n > 0.0f ? fab(err[0]) : err[0];
        res_add(res, v);
        if (scene_last) {
            atomicAdd(&d.scene_res_sq[scene], v * v);
            atomicAdd(&d.scene_res_n[scene], 1u);
            atomicMax(reinterpret_cast<int*>(&d.scene_res_mx[scene]), __float_as_int(v));
        }
    }
}

// Duals of contacts owned by body i (the other body non-dynamic or of an
// earlier colour), read from global memory: the oversized-body path.
__device__ void owned_contact_duals(const Dev& d, uint32_t i, uint32_t col, float dt, uint32_t phase, Res& res,
                                    uint32_t it, int gl, int G) {
    const uint32_t ro = d.roff[i], rn = d.rcount[i];
    for (uint32_t r = gl; r < rn; r += G) {
        const uint32_t other = d.bother[ro + r];
        const uint32_t ocol = d.color[other];
        if (!(ocol == kInvalid || ocol < col)) continue;
        const uint32_t c = d.blist[ro + r] & 0x7fffffffu;
        dual_contact(d, c, d.c_bodies[c], dt, phase, res, it);
    }
}

// Joints owned by body i: dual_joint once the later of its two bodies solved.
__device__ void owned_joint_duals(const Dev& d, uint32_t i, uint32_t col, float dt, uint32_t phase, Res& res,
                                  uint32_t it, int gl, int G) {
    const uint32_t jcnt = d.jdeg[i];
    if (!jcnt) return;
    const uint32_t jlo = d.jinc_off[i];
    for (uint32_t k = gl; k < jcnt; k += G) {
        const uint32_t j = d.jinc_list[jlo + k];
        const JointState js = d.jstate[j];
        const uint32_t other = js.dense_a == i ? js.dense_b : js.dense_a;
        const uint32_t ocol = d.color[other];
        if (!(ocol == kInvalid || ocol < col)) continue;
        dual_joint(d, j, phase, dt, res, it);
    }
}

template <int G>
__device__ __forceinline__ V6 staged_update(const Dev& d, uint32_t i, uint32_t phase, const V6& upd, uint32_t gmask,
                                            int gl);

// One body's primal from the stage (G lanes; lane gl), then its owned duals.
template <int G>
__device__ void staged_body(const Dev& d, const StageTables& tb, uint32_t sl, uint32_t col, uint32_t phase, float dt,
                            uint32_t gmask, int gl, int gbase, Res& res, uint32_t it) {
    const uint32_t i = tb.body[sl];
    const uint32_t r0 = tb.off[sl], r1 = tb.off[sl + 1];
    V6 dx0;
#pragma unroll
    for (int k = 0; k < 6; ++k) dx0.v[k] = tb.dx[6 * sl + k];
    float ent[Owned<G>::E];
    {
        const float4 ia = d.inA[i], ib = d.inB[i];
        float H[21];
#pragma unroll
        for (int k = 0; k < 21; ++k) H[k] = 0.0f;
        H[bidx(0, 0)] = ia.x;
        H[bidx(1, 1)] = ia.x;
        H[bidx(2, 2)] = ia.x;
        H[bidx(3, 3)] = ia.y;
        H[bidx(4, 3)] = ia.z;
        H[bidx(5, 3)] = ib.x;
        H[bidx(4, 4)] = ia.w;
        H[bidx(5, 4)] = ib.y;
        H[bidx(5, 5)] = ib.z;
#pragma unroll
        for (int q = 0; q < Owned<G>::E; ++q) {
            const int e = gl + G * q;
            float v = 0.0f;
#pragma unroll
            for (int k = 0; k < 21; ++k) v = e == k ? H[k] : v;
            if (e >= 21 && e < 27) {
                const int r = e - 21;
                float gs = 0.0f;
#pragma unroll
                for (int c = 0; c < 6; ++c) gs += H[bidx(r, c)] * dx0.v[c];
                v = gs;
            }
            ent[q] = v;
        }
    }
    // Rows in list order, each row's n, t0, t1: the serial loop's additions.
#pragma unroll
    for (int q = 0; q < Owned<G>::E; ++q) {
        const int e = gl + G * q;
        if (e >= 27) continue;
        int ei = 0, ek = 0;
        const bool hess = e < 21;
        if (hess) entry_ik(e, ei, ek);
        else ei = e - 21;
        float acc = ent[q];
        for (uint32_t t = r0; t < r1; ++t) {
            const float* row = tb.rows + size_t(t) * kRowWords;
#pragma unroll
            for (int x = 0; x < 3; ++x) {
                const float* jr = row + kRJ + 6 * x;
                acc += hess ? (row[kRSt + x] * jr[ei]) * jr[ek] : jr[ei] * row[kRForce + x];
            }
        }
        ent[q] = acc;
    }
    Blk blk;
    gather_block<G>(ent, blk, gmask, gbase);
    const uint32_t jcnt = d.jdeg[i];
    if (jcnt) joint_rows_shared<G>(d, i, phase, dt, blk, tb.jblk + threadIdx.x / G, tb.jview + 2 * (threadIdx.x / G),
                                        gmask, gl);
    V6 upd;
    const bool solved = block_solve(blk, upd);
    V6 dxn = dx0;
    if (solved) {
        // Crossing safeguard (geometry_constraints_solve.slang:433-475): each
        // lane flags its share of the staged normal rows, then every lane adds
        // the flagged rows to its entries in list order.
        bool flagged = false;
        for (uint32_t t = r0 + gl; t < r1; t += G) {
            float* row = tb.rows + size_t(t) * kRowWords;
            V6 nr;
#pragma unroll
            for (int k = 0; k < 6; ++k) nr.v[k] = row[kRJ + k];
            const float k0 = row[kRPen], trial = row[kRTrial];
            const bool cross = trial <= 0.0f && trial + k0 * dot6(nr, upd) > k0 * 1.0e-6f;
            uint32_t flags = __float_as_uint(row[kRFlags]);
            flags = cross ? (flags | 4u) : (flags & ~4u);
            row[kRFlags] = __uint_as_float(flags);
            flagged = flagged || cross;
        }
        const bool crossing = __any_sync(gmask, flagged);
        __syncwarp(gmask);
        if (crossing) {
            own_entries<G>(blk, gl, ent);
#pragma unroll
            for (int q = 0; q < Owned<G>::E; ++q) {
                const int e = gl + G * q;
                if (e >= 27) continue;
                int ei = 0, ek = 0;
                if (e < 21) entry_ik(e, ei, ek);
                float acc = ent[q];
                for (uint32_t t = r0; t < r1; ++t) {
                    const float* row = tb.rows + size_t(t) * kRowWords;
                    if (!(__float_as_uint(row[kRFlags]) & 4u)) continue;
                    const float k0 = row[kRPen];
                    acc += e < 21 ? k0 * row[kRJ + ei] * row[kRJ + ek] : row[kRJ + e - 21] * row[kRTrial];
                }
                ent[q] = acc;
            }
            gather_block<G>(ent, blk, gmask, gbase);
            V6 safe;
            if (block_solve(blk, safe)) upd = safe;
        }
        dxn = staged_update<G>(d, i, phase, upd, gmask, gl);
    }
    __syncwarp(gmask);
    // Owned contact duals, one row per lane.
    uint32_t scene = 0;
    bool scene_last = false;
    if (batched(d)) {
        scene = d.scene_of[i];
        scene_last = phase == 0 && it + 1 == d.scene_budget[scene];
    }
    for (uint32_t t = r0 + gl; t < r1; t += G) {
        const float* row = tb.rows + size_t(t) * kRowWords;
        if (__float_as_uint(row[kRFlags]) & 2u) staged_dual(d, row, dxn, scene, scene_last, res);
    }
    // Owned joint duals read both bodies' displacements from global memory.
    __syncwarp(gmask);
    if (jcnt) owned_joint_duals(d, i, col, dt, phase, res, it, gl, G);
}

// The body's update (apply_pose_update, geometry_constraints_solve.slang:
// 374-399, or the impact phase's linear update): lane 0 stores it; every lane
// returns the new displacement. Every lane reads the body's state before
// lane 0 stores.
template <int G>
__device__ __forceinline__ V6 staged_update(const Dev& d, uint32_t i, uint32_t phase, const V6& upd, uint32_t gmask,
                                            int gl) {
    float4 l = d.dxl[i], a = d.dxa[i];
    Q4 rel = q4(d.dq[i]);
    __syncwarp(gmask);
    l.x += upd.v[0];
    l.y += upd.v[1];
    l.z += upd.v[2];
    if (phase == 0) {
        const V3 r{upd.v[3], upd.v[4], upd.v[5]};
        const bool rotates = !(r.x == 0.0f && r.y == 0.0f && r.z == 0.0f);
        if (rotates) {
            Q4 dd = qmul(Q4{r.x, r.y, r.z, 0.0f}, rel);
            rel = qnormalize(Q4{rel.x + 0.5f * dd.x, rel.y + 0.5f * dd.y, rel.z + 0.5f * dd.z, rel.w + 0.5f * dd.w});
            if (rel.w < 0.0f) rel = {-rel.x, -rel.y, -rel.z, -rel.w};
            a = make_float4(2.0f * rel.x, 2.0f * rel.y, 2.0f * rel.z, 0.0f);
        }
        if (gl == 0) {
            d.dxl[i] = l;
            if (rotates) {
                d.dq[i] = f4(rel);
                d.dxa[i] = a;
            }
        }
    } else {
        a.x += upd.v[3];
        a.y += upd.v[4];
        a.z += upd.v[5];
        if (gl == 0) {
            d.dxl[i] = l;
            d.dxa[i] = a;
        }
    }
    return {{l.x, l.y, l.z, a.x, a.y, a.z}};
}

template <int T, bool Timed>
__global__ void __launch_bounds__(T, 1) k_solve_staged(Dev d, StepParams sp, uint32_t phase) {
    Counters* c = d.ctr;
    if (phase != 0 && c->impact == 0) return;
    if (c->status & kStBarrierTimeout) return;  // the tick was abandoned
    extern __shared__ __align__(16) uint8_t stage_raw[];
    const StageTables tb = stage_tables(stage_raw);
    const int lane = threadIdx.x & 31;
    const float dt = sp.dt;
    const uint32_t colors = c->colors;
    uint32_t budget = sp.budget_request;
    if (!sp.realtime && sp.requested == 0) budget = max(budget, c->joint_iters);
    if (phase != 0 && sp.tolerance > 0.0f) budget = c->budget;
    const bool adaptive = phase == 0 && sp.tolerance > 0.0f && !batched(d);
    const uint32_t iters = batched(d) ? min(c->budget_max, kMaxIterations)
                                      : adaptive ? min(max(sp.max_iterations, 1u), kMaxIterations)
                                                 : min(budget, kMaxIterations);
    __shared__ double wsq[T / 32];
    __shared__ uint32_t wn[T / 32], wov[T / 32];
    __shared__ float wmx[T / 32];
    const bool timing = Timed && phase == 0;
    if (timing && blockIdx.x == 0 && threadIdx.x == 0) c->dbg_start = gtimer();
    for (uint32_t it = 0; it < iters; ++it) {
        Res res{0.0, 0u, 0.0f, 0u, sp.tolerance};
        const uint32_t parity = (it & 1u) * 512u;
        for (uint32_t col = 0; col <= colors; ++col) {
            if (col < colors) {
                const uint32_t lo = c->color_off[col * kSortClasses], hi = c->color_off[(col + 1) * kSortClasses];
                const uint32_t span = hi - lo;
                const uint32_t mine = span > blockIdx.x ? (span - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
                for (uint32_t j0 = 0; j0 < mine;) {
                    // Profiling build: phase times of colour 0's batches in
                    // the first sweep (formation, staging, solve) summed
                    // over CTAs into dbg_sum[0..2], batches in dbg_sum[6].
                    const bool phase_clock = timing && it == 0 && col == 0 && threadIdx.x == 0;
                    unsigned long long tp0 = phase_clock ? gtimer() : 0ull;
                    // Batch slots: this CTA's next bodies of the colour.
                    const uint32_t want = min(kBatchBodies, mine - j0);
                    uint32_t cnt = 0;
                    if (threadIdx.x < want) {
                        const uint32_t i = d.corder[lo + blockIdx.x + (j0 + threadIdx.x) * gridDim.x];
                        const bool skip = (phase != 0 && d.impact[i] == 0) ||
                                          (batched(d) && it >= d.scene_budget[d.scene_of[i]]);
                        cnt = skip ? 0u : d.rcount[i];
                        tb.body[threadIdx.x] = i;
                        tb.skip[threadIdx.x] = skip ? 1u : 0u;
                        const float4 l = d.dxl[i], a = d.dxa[i];
                        float* dx = tb.dx + 6 * threadIdx.x;
                        dx[0] = l.x;
                        dx[1] = l.y;
                        dx[2] = l.z;
                        dx[3] = a.x;
                        dx[4] = a.y;
                        dx[5] = a.z;
                    }
                    // Inclusive scan of the slots' row counts (T >= kBatchBodies).
                    uint32_t x = cnt;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                        if (lane >= o) x += y;
                    }
                    if (lane == 31) tb.scratch[threadIdx.x >> 5] = x;
                    __syncthreads();
                    if (threadIdx.x < 32) {
                        uint32_t p = threadIdx.x < T / 32 ? tb.scratch[threadIdx.x] : 0u;
#pragma unroll
                        for (int o = 1; o < 32; o <<= 1) {
                            const uint32_t y = __shfl_up_sync(0xffffffffu, p, o);
                            if (lane >= o) p += y;
                        }
                        tb.scratch[32 + threadIdx.x] = p;
                    }
                    __syncthreads();
                    const uint32_t incl = x + ((threadIdx.x >> 5) ? tb.scratch[32 + (threadIdx.x >> 5) - 1] : 0u);
                    if (threadIdx.x < want) tb.off[threadIdx.x + 1] = incl;
                    if (threadIdx.x == 0) tb.off[0] = 0;
                    const uint32_t fit = __syncthreads_count(threadIdx.x < want && incl <= kStageRows);
                    if (fit == 0) {
                        // The next body alone has more rows than the stage
                        // holds: solve it streaming its rows from global
                        // memory (one warp, 32 lanes), then its duals.
                        if (threadIdx.x < 32) {
                            const uint32_t i = tb.body[0];
                            if (!tb.skip[0]) {
                                GroupRows<32>& sm = *reinterpret_cast<GroupRows<32>*>(tb.rows);
                                Ahead ah{i, d.roff[i], d.rcount[i], 0u, 0u, 0u, 0u, d.impact[i]};
                                fetch_codes<32>(d, ah, lane);
                                solve_body_group<32, true>(d, ah, ~0u, phase, dt, sm, 0xffffffffu, lane, 0, 0u);
                                __syncwarp();
                                owned_contact_duals(d, i, col, dt, phase, res, it, lane, 32);
                                __syncwarp();
                                owned_joint_duals(d, i, col, dt, phase, res, it, lane, 32);
                            }
                        }
                        __syncthreads();
                        j0 += 1;
                        continue;
                    }
                    if (phase_clock) {
                        const unsigned long long t = gtimer();
                        atomicAdd(&c->dbg_sum[0], t - tp0);
                        tp0 = t;
                    }
                    // Stage every row of the batch, one thread per row.
                    const uint32_t rows = tb.off[fit];
                    for (uint32_t t = threadIdx.x; t < rows; t += T) {
                        uint32_t a = 0, b = fit;  // slot: off[a] <= t < off[a + 1]
                        while (b - a > 1) {
                            const uint32_t m = (a + b) >> 1;
                            if (tb.off[m] <= t) a = m;
                            else b = m;
                        }
                        stage_row(d, tb, t, a, t - tb.off[a], col, phase, dt);
                    }
                    __syncthreads();
                    if (phase_clock) {
                        const unsigned long long t = gtimer();
                        atomicAdd(&c->dbg_sum[1], t - tp0);
                        atomicAdd(&c->dbg_sum[7], (unsigned long long)rows);
                        tp0 = t;
                    }
                    // Solve: G lanes per body (wider groups when few bodies).
                    auto solve = [&](auto width) {
                        constexpr int G = decltype(width)::value;
                        const int gl = lane % G, gbase = lane - gl;
                        const uint32_t gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << gbase;
                        for (uint32_t sl = threadIdx.x / G; sl < fit; sl += T / G)
                            if (!tb.skip[sl]) staged_body<G>(d, tb, sl, col, phase, dt, gmask, gl, gbase, res, it);
                    };
                    if (d.solve_policy != 1 && fit * 32u <= T) solve(std::integral_constant<int, 32>{});
                    else if (d.solve_policy != 1 && fit * 16u <= T) solve(std::integral_constant<int, 16>{});
                    else solve(std::integral_constant<int, 8>{});
                    __syncthreads();
                    if (phase_clock) {
                        atomicAdd(&c->dbg_sum[2], gtimer() - tp0);
                        atomicAdd(&c->dbg_sum[6], 1ull);
                    }
                    j0 += fit;
                }
            }
            if (timing && it == 0 && col < 19 && threadIdx.x == 0) atomicMax(&c->dbg_work[col], gtimer());
            if (col + 1 >= colors) {
                // Joints with no dynamic body have no owner above; their
                // duals (applied impulse, breaking) are updated here.
                for (uint32_t j = grid_stride_begin(); j < d.nj; j += grid_stride()) {
                    const JointState js = d.jstate[j];
                    if (js.count == 0 || d.motion[js.dense_a] == kDynamic || d.motion[js.dense_b] == kDynamic) continue;
                    dual_joint(d, j, phase, dt, res, it);
                }
                // The sweep's residual partials (after the last colour's
                // duals), published by the barrier below.
                block_residual<T>(res, wsq, wn, wmx, wov, c, parity + blockIdx.x);
                if (!grid_sync(c, d.barrier_spins)) return;
                if (timing && it == 0 && col < 19 && blockIdx.x == 0 && threadIdx.x == 0) c->dbg_release[col] = gtimer();
                break;
            }
            if (!grid_sync(c, d.barrier_spins)) return;
            if (timing && it == 0 && col < 19 && blockIdx.x == 0 && threadIdx.x == 0) c->dbg_release[col] = gtimer();
        }
        const SweepResidual sw = sweep_residual(c, parity, sp);
        if (phase == 0 && grid_stride_begin() == 0) c->residual_trace[it] = sw.measure;
        bool last = it + 1 == iters;
        if (adaptive && sw.met) last = true;
        if (last) {
            if (grid_stride_begin() == 0) {
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

// The staged solve has one build for every feature set.
template <int T, bool Timed>
static void staged_builds(const void* (&out)[kSolveFeatures]) {
    for (int f = 0; f < kSolveFeatures; ++f) out[f] = reinterpret_cast<const void*>(&k_solve_staged<T, Timed>);
}
template <int T>
static SolveVariant staged_variant() {
    SolveVariant v{};
    staged_builds<T, false>(v.ptr);
    staged_builds<T, true>(v.timed);
    v.threads = T;
    v.smem = kStagedSmem;
    return v;
}

const SolveVariant& solve_variant(uint32_t v) {
    static const SolveVariant table[kSolveVariants] = {solve_group_variant_512(), solve_group_variant_384(),
                                                       solve_group_variant_256(), staged_variant<512>(),
                                                       staged_variant<384>()};
    return table[v < kSolveVariants ? v : 0];
}

// Last-iteration contact work (geometry_constraints_solve.slang:533-561),
// one thread per contact point.
__global__ void k_contact_finalize(Dev d, StepParams sp, uint32_t phase) {
    if (phase != 0 && d.ctr->impact == 0) return;
    const float dt = sp.dt;
    const uint32_t n_con = d.ctr->n_contacts;
    for (uint32_t c = grid_stride_begin(); c < n_con; c += grid_stride()) {
        const uint2 ab = d.c_bodies[c];
        const uint32_t a = ab.x, b = ab.y;
        if (phase != 0 && d.impact[a] == 0 && d.impact[b] == 0) continue;
        const V3 n = v3(d.c_n[c]);
        float4 lam = d.c_lam[c];
        const float stick = d.c_pen[c].w;
        V3 t0, t1;
        basis(n, t0, t1);
        lam.w = lam.x * dt;
        d.c_lam[c] = lam;
        d.c_accf[c] = f4(mul(add(mul(t0, lam.y), mul(t1, lam.z)), dt));
        if (stick == 0.0f) {
            V3 xa, xb;
            Q4 qa, qb;
            if (phase != 0) {
                xa = v3(d.tx[a]);
                qa = q4(d.tq[a]);
                xb = v3(d.tx[b]);
                qb = q4(d.tq[b]);
            } else {
                BodyView A = load_body(d, a), B = load_body(d, b);
                body_pose(A, xa, qa);
                body_pose(B, xb, qb);
            }
            const V3 pt = v3(d.c_p[c]);
            const float4 aa = d.c_aa[c], ab = d.c_ab[c];
            d.c_aa[c] = f4(inv_rotate(qa, sub(pt, xa)), aa.w);
            d.c_ab[c] = f4(inv_rotate(qb, sub(pt, xb)), ab.w);
        }
    }
}

// free_mean (geometry_constraints_solve.slang:617-675): anchored flag per
// island (any member touching a non-dynamic body), then the mass-weighted mean
// of unanchored islands, summed serially in body order from the root.
__global__ void k_free_anchor(Dev d, uint32_t phase) {
    const uint32_t n_act = d.ctr->n_act;
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) d.mean[i] = make_float4(0, 0, 0, 0);
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t a = d.act_a[i], b = d.act_b[i];
        const bool da = d.motion[a] == kDynamic, db = d.motion[b] == kDynamic;
        if (da && !db) d.anchored[d.parent[a]] = 1;
        if (db && !da) d.anchored[d.parent[b]] = 1;
    }
    for (uint32_t j = grid_stride_begin(); j < d.nj; j += grid_stride()) {
        const JointState st = d.jstate[j];
        if (st.count == 0) continue;
        const bool da = d.motion[st.dense_a] == kDynamic, db = d.motion[st.dense_b] == kDynamic;
        if (da && !db) d.anchored[d.parent[st.dense_a]] = 1;
        if (db && !da) d.anchored[d.parent[st.dense_b]] = 1;
    }
}

// One warp per island root: the members, found 32 indices at a time between
// the root (the island's lowest index) and the island's largest index, are
// summed by every lane in ascending index order -- the reference's serial
// root loop (geometry_constraints_solve.slang:617-698) without its scan over
// all bodies.
__global__ void k_free_mean(Dev d, uint32_t phase) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = warp; r < d.n; r += warps) {
        if (d.motion[r] != kDynamic || d.parent[r] != r) continue;
        if ((phase != 0 && d.impact[r] == 0) || (d.deg[r] == 0 && d.jdeg[r] == 0)) continue;
        if (d.anchored[r]) continue;
        const uint32_t end = d.island_end[r];
        V3 weighted{0, 0, 0};
        float total = 0.0f;
        for (uint32_t base = r; base <= end; base += 32u) {
            const uint32_t i = base + lane;
            const bool member = i <= end && d.motion[i] == kDynamic && d.parent[i] == r;
            float mass = 0.0f;
            float4 l = make_float4(0, 0, 0, 0);
            if (member) {
                mass = 1.0f / fmx(d.p0[i].x, 1.0e-12f);
                l = d.dxl[i];
            }
            uint32_t mask = __ballot_sync(0xffffffffu, member);
            while (mask) {
                const int k = __ffs(mask) - 1;
                mask &= mask - 1u;
                const float mk = __shfl_sync(0xffffffffu, mass, k);
                const V3 lk{__shfl_sync(0xffffffffu, l.x, k), __shfl_sync(0xffffffffu, l.y, k),
                            __shfl_sync(0xffffffffu, l.z, k)};
                weighted = add(weighted, mul(lk, mk));
                total += mk;
            }
        }
        if (lane == 0 && total > 0.0f) d.mean[r] = f4(mul(weighted, 1.0f / total));
    }
}

__global__ void k_free_subtract(Dev d, uint32_t phase) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        if (d.motion[i] != kDynamic || (phase != 0 && d.impact[i] == 0)) continue;
        const float4 m = d.mean[d.parent[i]];
        float4 l = d.dxl[i];
        l.x -= m.x;
        l.y -= m.y;
        l.z -= m.z;
        d.dxl[i] = l;
    }
}

// apply_states (geometry_constraints_solve.slang:699-733) into the output
// state arrays (v: solved state; t: the AVBD target stays untouched).
__global__ void k_apply(Dev d, StepParams sp, uint32_t phase, float4* ox, float4* oq, float4* ov, float4* ow) {
    if (phase != 0 && d.ctr->impact == 0) return;
    const float dt = sp.dt;
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        if (d.motion[i] != kDynamic) continue;
        if (phase != 0 && d.impact[i] == 0) continue;
        const float4 l = d.dxl[i], a = d.dxa[i];
        const V3 lin = v3(l), rot = v3(a);
        V3 x = v3(d.tx[i]), v = v3(d.tv[i]), w = v3(d.tw[i]);
        Q4 q = q4(d.tq[i]);
        if (phase != 0) {
            v = add(v, mul(lin, 1.0f / dt));
            w = add(w, mul(rot, 1.0f / dt));
            ox[i] = f4(x);
            oq[i] = f4(q);
            ov[i] = f4(v);
            ow[i] = f4(w);
            continue;
        }
        const Q4 dq = q4(d.dq[i]);
        x = add(x, lin);
        if (dq.x != 0.0f || dq.y != 0.0f || dq.z != 0.0f) q = qnormalize(qmul(dq, q));
        v = add(v, mul(lin, 1.0f / dt));
        w = add(w, mul(rotation_vector(dq), 1.0f / dt));
        if (sp.realtime) {
            v = mul(v, 1.0f - 0.05f);
            w = mul(w, 1.0f - 0.05f);
        }
        ox[i] = f4(x);
        oq[i] = f4(q);
        ov[i] = f4(v);
        ow[i] = f4(w);
    }
}

// rigid_avbd_project_hinge_anchors (geometry_constraints_solve.slang:174-209):
// serial over the hinge joints in index order, as in the reference. One
// thread per scene segment (scenes of a batched world share no bodies).
__global__ void k_project_hinges(Dev d, float4* ox, const float4* oq) {
    const uint32_t seg = blockIdx.x * blockDim.x + threadIdx.x;
    if (seg >= d.n_hinge_segs) return;
    for (uint32_t h = d.hinge_seg[seg]; h < d.hinge_seg[seg + 1]; ++h) {
        const uint32_t j = d.hinge_list[h];
        const JointState st = d.jstate[j];
        if (st.count == 0 || !st.enabled) continue;
        const uint32_t a = st.dense_a, b = st.dense_b;
        const float ima = d.motion[a] == kDynamic ? d.p0[a].x : 0.0f;
        const float imb = d.motion[b] == kDynamic ? d.p0[b].x : 0.0f;
        const float sum = ima + imb;
        if (sum <= kEps) continue;
        const Joint& o = d.joints[j];
        V3 pa = add(v3(ox[a]), rotate(q4(oq[a]), V3{o.anchor_a[0], o.anchor_a[1], o.anchor_a[2]}));
        V3 pb = add(v3(ox[b]), rotate(q4(oq[b]), V3{o.anchor_b[0], o.anchor_b[1], o.anchor_b[2]}));
        V3 e = sub(pb, pa);
        ox[a] = f4(add(v3(ox[a]), mul(e, ima / sum)));
        ox[b] = f4(sub(v3(ox[b]), mul(e, imb / sum)));
    }
}

// Velocity-phase setup (geometry_constraints_solve.slang:238-330).
__global__ void k_impact_setup(Dev d, StepParams sp, const float4* ox, const float4* oq, const float4* ov,
                               const float4* ow) {
    if (d.ctr->impact == 0) return;
    const uint32_t n_act = d.ctr->n_act;
    // impact_gaps (uses the phase-0 displacements)
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t a = d.act_a[i], b = d.act_b[i];
        if (d.impact[a] == 0 && d.impact[b] == 0) continue;
        const Lite A = load_lite(d, a), B = load_lite(d, b);
        for (uint32_t q = d.act_off[i]; q < d.act_off[i] + d.act_cnt[i]; ++q) {
            const float4 n4 = d.c_n[q];
            V6 ja[3], jb[3];
            load_jac(d, q, ja, jb);  // normal rows: the phase-0 targets' arms
            float4 e = d.c_e[q];
            e.x = fmx(0.0f, -(n4.w + dot6(ja[0], A.dx) + dot6(jb[0], B.dx)));
            d.c_e[q] = e;
        }
    }
}
__global__ void k_impact_bodies(Dev d, const float4* ox, const float4* oq, const float4* ov, const float4* ow) {
    if (d.ctr->impact == 0) return;
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        if (d.impact[i] != 0 || d.motion[i] != kDynamic) {
            d.tx[i] = ox[i];
            d.tq[i] = oq[i];
            d.tv[i] = ov[i];
            d.tw[i] = ow[i];
            d.dxl[i] = make_float4(0, 0, 0, 0);
            d.dxa[i] = make_float4(0, 0, 0, 0);
            d.dq[i] = make_float4(0, 0, 0, 1);
        }
    }
}
__global__ void k_impact_constraints(Dev d, StepParams sp, const float4* ov, const float4* ow) {
    if (d.ctr->impact == 0) return;
    const float dt = sp.dt;
    for (uint32_t j = grid_stride_begin(); j < d.nj; j += grid_stride()) {
        const JointState st = d.jstate[j];
        if (st.count == 0 || !st.enabled) continue;
        const uint32_t a = st.dense_a, b = st.dense_b;
        if (d.impact[a] == 0 && d.impact[b] == 0) continue;
        BodyView A = load_body(d, a), B = load_body(d, b);
        Blk scratch;
        visit_joint(d.joints[j], d.jrows + size_t(j) * 18, A, B, v3(d.x[a]), q4(d.q[a]), v3(d.x[b]), q4(d.q[b]),
                    d.p0[a], d.p0[b], dt, &scratch, true, kVisitImpact, nullptr);
    }
    const uint32_t n_act = d.ctr->n_act;
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t a = d.act_a[i], b = d.act_b[i];
        if (d.impact[a] == 0 && d.impact[b] == 0) continue;
        const V6 va = jac(mul(v3(ov[a]), dt), mul(v3(ow[a]), dt));
        const V6 vb = jac(mul(v3(ov[b]), dt), mul(v3(ow[b]), dt));
        const float rest_ab = fmn(d.p1[a].y, d.p1[b].y);
        for (uint32_t q = d.act_off[i]; q < d.act_off[i] + d.act_cnt[i]; ++q) {
            float4 e = d.c_e[q];
            const float gap = e.x;
            V6 ja[3], jb[3];
            load_jac(d, q, ja, jb);  // recomputed from the reset targets
            const bool cached = d.c_aa[q].w != 0.0f;
            const float speed = e.w;
            const float rest = !cached && speed < -1.0f ? rest_ab : 0.0f;
            e.x = dot6(ja[0], va) + dot6(jb[0], vb) - gap - rest * speed * dt;
            e.y = dot6(ja[1], va) + dot6(jb[1], vb);
            e.z = dot6(ja[2], va) + dot6(jb[2], vb);
            d.c_e[q] = e;
        }
    }
}

// pm_clamp_rigid_speeds (geometry.slang:3086-3100), then commit the solved
// states as the next tick's current states.
__global__ void k_clamp_commit(Dev d, const float4* ox, const float4* oq, const float4* ov, const float4* ow) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        V3 v = v3(ov[i]), w = v3(ow[i]);
        if (d.motion[i] == kDynamic) {
            const float4 p2 = d.p2[i];
            v = clamp_length(v, p2.x);
            w = clamp_length(w, p2.y);
        }
        d.x[i] = ox[i];
        d.q[i] = oq[i];
        d.v[i] = f4(v);
        d.w[i] = f4(w);
    }
}

// pm_save_rigid_contact_cache (geometry.slang:3011-3070) into the next tick's
// cache buffers, keyed by pair code (already sorted).
__global__ void k_cache_save(Dev d, StepParams sp) {
    const uint32_t n_act = d.ctr->n_act;
    if (grid_stride_begin() == 0) {
        *d.out_n_pairs = n_act;
        *d.out_dt = sp.dt;
    }
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t a = d.act_a[i];
        const V3 xa = v3(d.x[a]);
        const Q4 qa = q4(d.q[a]);
        const uint32_t off = d.act_off[i], np = d.act_cnt[i];
        d.out_code[i] = d.act_code[i];
        d.out_off[i] = off;
        d.out_cnt[i] = np;
        for (uint32_t q = 0; q < np; ++q) {
            const uint32_t c = off + q;
            d.out_local[c] = f4(inv_rotate(qa, sub(v3(d.c_p[c]), xa)));
            d.out_normal[c] = d.c_n[c];
            const float4 lam = d.c_lam[c];
            d.out_fimp[c] = f4(v3(d.c_accf[c]), lam.w);
            d.out_lam[c] = lam;
            d.out_pen[c] = d.c_pen[c];
            d.out_aa[c] = d.c_aa[c];
            d.out_ab[c] = d.c_ab[c];
        }
    }
}

// Contact events of the tick (geometry.slang:2902-2939 and :3028-3043): one
// per contact point in active-pair order, up to the capacity. Points,
// normals and penetrations are the narrowphase's (unchanged since); the
// impulses are those the cache save stores (convex pairs are persistent).
__global__ void k_contact_events(Dev d) {
    const uint32_t n = min(d.ctr->n_contacts, d.event_capacity);
    if (grid_stride_begin() == 0) d.ctr->n_events = n;
    for (uint32_t c = grid_stride_begin(); c < n; c += grid_stride()) {
        const uint2 ab = d.c_bodies[c];
        const float4 nn = d.c_n[c], p = d.c_p[c], f = d.c_accf[c];
        ContactEvent e;
        e.body = ab.x;
        e.collider = ab.y;
        e.position[0] = p.x;
        e.position[1] = p.y;
        e.position[2] = p.z;
        e.normal[0] = nn.x;
        e.normal[1] = nn.y;
        e.normal[2] = nn.z;
        e.penetration = fmx(0.0f, nn.w);
        e.normal_impulse = d.c_lam[c].w;
        e.friction_impulse[0] = f.x;
        e.friction_impulse[1] = f.y;
        e.friction_impulse[2] = f.z;
        d.events[c] = e;
    }
}

void launch_solve_all(const Dev& d, const StepParams& sp, cudaStream_t s, const int* coop_blocks,
                      const SolveBuffers& o) {
    const SolveVariant& sv = solve_variant(d.solve_variant);
    const int coop = coop_blocks[d.solve_variant < kSolveVariants ? d.solve_variant : 0];
    const int feat = solve_features(d);
    const uint32_t pb = cap_blocks(d.cap_pair > d.nj ? d.cap_pair : d.nj);
    for (uint32_t phase = 0; phase < (sp.realtime ? 1u : 2u); ++phase) {
        if (phase != 0) {
            k_impact_setup<<<cap_blocks(d.cap_pair), kBlock, 0, s>>>(d, sp, o.ox, o.oq, o.ov, o.ow);
            note_launch(cap_blocks(d.cap_pair));
            k_impact_bodies<<<blocks_for(d.n), kBlock, 0, s>>>(d, o.ox, o.oq, o.ov, o.ow);
            note_launch(blocks_for(d.n));
            launch_contact_jacobians(d, 1, sp.dt, s);
            k_impact_constraints<<<pb, kBlock, 0, s>>>(d, sp, o.ov, o.ow);
            note_launch(pb);
            prof_mark(s, "impact setup");
        }
        Dev dd = d;
        uint32_t ph = phase;
        StepParams spp = sp;
        void* args[] = {&dd, &spp, &ph};
        solve_timer_begin(s);
        // The profiling build only for pmb_world_profile_step (it has the
        // same launch shape; the world sized its grid for both).
        cudaLaunchCooperativeKernel(sp.debug_timing ? sv.timed[feat] : sv.ptr[feat], dim3(coop), dim3(sv.threads), args,
                                    sv.smem, s);
        note_launch(coop);
        solve_timer_end(s);
        prof_mark(s, phase ? "solve phase 1" : "solve phase 0");
        k_contact_finalize<<<cap_blocks(d.cap_contact), kBlock, 0, s>>>(d, sp, phase);
        note_launch(cap_blocks(d.cap_contact));
        k_free_anchor<<<cap_blocks(d.cap_pair > d.n ? d.cap_pair : d.n), kBlock, 0, s>>>(d, phase);
        note_launch(cap_blocks(d.cap_pair > d.n ? d.cap_pair : d.n));
        k_free_mean<<<std::min<uint32_t>(blocks_for(32u * d.n, 256), 148u * 8u), 256, 0, s>>>(d, phase);
        note_launch(std::min<uint32_t>(blocks_for(32u * d.n, 256), 148u * 8u));
        k_free_subtract<<<blocks_for(d.n), kBlock, 0, s>>>(d, phase);
        note_launch(blocks_for(d.n));
        k_apply<<<blocks_for(d.n), kBlock, 0, s>>>(d, sp, phase, o.ox, o.oq, o.ov, o.ow);
        note_launch(blocks_for(d.n));
        if (phase == 0 && d.n_hinge_segs) {
            k_project_hinges<<<blocks_for(d.n_hinge_segs), kBlock, 0, s>>>(d, o.ox, o.oq);
            note_launch(blocks_for(d.n_hinge_segs));
        }
        prof_mark(s, phase ? "finish phase 1" : "finish phase 0");
    }
    set_phase(kPhCommit);
    k_clamp_commit<<<blocks_for(d.n), kBlock, 0, s>>>(d, o.ox, o.oq, o.ov, o.ow);
    note_launch(blocks_for(d.n));
    k_cache_save<<<cap_blocks(d.cap_pair), kBlock, 0, s>>>(d, sp);
    note_launch(cap_blocks(d.cap_pair));
    if (sp.collect_events && d.event_capacity) {
        k_contact_events<<<cap_blocks(d.event_capacity), kBlock, 0, s>>>(d);
        note_launch(cap_blocks(d.event_capacity));
    }
    prof_mark(s, "commit+cache save");
}

}  // namespace pmb

// SPDX-License-Identifier: MIT
// Device helpers of the AVBD solve kernels: body displacements, contact
// rows, the group-per-body and body-per-thread primal, the dual updates and
// the residual reduction. Shared by the solve kernels' translation units.
#pragma once
#include <type_traits>

#include "pmb_joint.cuh"

namespace pmb {

struct Lite {  // what a contact row needs of a body during the solve: its displacement
    V6 dx;
};
__device__ __forceinline__ Lite load_lite(const Dev& d, uint32_t i) {
    const float4 l = d.dxl[i], a = d.dxa[i];
    return {{{l.x, l.y, l.z, a.x, a.y, a.z}}};
}

// Contact jacobians (geometry_constraints.slang:508-532). They depend only on
// the contact geometry and the AVBD target poses, both fixed during a solve
// phase, so they are evaluated once per phase (k_contact_jacobians) and
// stored: 36 floats per contact, rows n, t0, t1 for body a then body b.
__device__ __forceinline__ void contact_jacobians(V3 n, V3 pt, V3 anc_a, V3 anc_b, V3 xa, Q4 qa, V3 xb, Q4 qb,
                                                  V6 ja[3], V6 jb[3]) {
    V3 t0, t1;
    basis(n, t0, t1);
    const V3 axes[3] = {n, t0, t1};
    const V3 arm_a = sub(pt, xa), arm_b = sub(pt, xb);
    const V3 ra_t = rotate(qa, anc_a), rb_t = rotate(qb, anc_b);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        V3 ra = k == 0 ? arm_a : ra_t;
        V3 rb = k == 0 ? arm_b : rb_t;
        ja[k] = jac(mul(axes[k], -1.0f), mul(cross(ra, axes[k]), -1.0f));
        jb[k] = jac(axes[k], cross(rb, axes[k]));
    }
}
__device__ __forceinline__ void load_jac(const Dev& d, uint32_t c, V6 ja[3], V6 jb[3]) {
    const float4* p = d.c_jac + size_t(c) * 9;
    float f[36];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const float4 v = p[k];
        f[4 * k] = v.x;
        f[4 * k + 1] = v.y;
        f[4 * k + 2] = v.z;
        f[4 * k + 3] = v.w;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            ja[r].v[k] = f[6 * r + k];
            jb[r].v[k] = f[18 + 6 * r + k];
        }
}
__device__ __forceinline__ void contact_rows(const Dev& d, uint32_t c, float4 e, const Lite& A, const Lite& B,
                                             V6 ja[3], V6 jb[3], float err[3]) {
    load_jac(d, c, ja, jb);
    const float e3[3] = {e.x, e.y, e.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) err[k] = e3[k] + dot6(ja[k], A.dx) + dot6(jb[k], B.dx);
}

__device__ __forceinline__ void apply_pose_update(const Dev& d, uint32_t i, const V6& u, float4 l, float4 dq) {
    l.x += u.v[0];
    l.y += u.v[1];
    l.z += u.v[2];
    d.dxl[i] = l;
    V3 r{u.v[3], u.v[4], u.v[5]};
    if (r.x == 0.0f && r.y == 0.0f && r.z == 0.0f) return;
    Q4 rel = q4(dq);
    Q4 dd = qmul(Q4{r.x, r.y, r.z, 0.0f}, rel);
    rel = qnormalize(Q4{rel.x + 0.5f * dd.x, rel.y + 0.5f * dd.y, rel.z + 0.5f * dd.z, rel.w + 0.5f * dd.w});
    if (rel.w < 0.0f) rel = {-rel.x, -rel.y, -rel.z, -rel.w};
    d.dq[i] = f4(rel);
    d.dxa[i] = make_float4(2.0f * rel.x, 2.0f * rel.y, 2.0f * rel.z, 0.0f);
}
__device__ __forceinline__ void apply_pose_update(const Dev& d, uint32_t i, const V6& u) {
    apply_pose_update(d, i, u, d.dxl[i], d.dq[i]);
}

// Group-per-body primal: G lanes (G = 8, 16 or 32) solve one body. Lanes
// evaluate the body's contact rows G at a time (coalesced SoA loads) and
// stage them in shared memory; each lane owns ceil(27/G) of the 27 entries of
// the packed 6x6 block (21 Hessian, 6 gradient) and adds the staged rows to
// them in list order. Every entry thus sees exactly the additions, in exactly
// the order, of the serial per-body loop of
// geometry_constraints_solve.slang:339-400, whatever G is, and the block is
// bit-identical to it; the LDL^T solve then runs in registers. The crossing
// safeguard reuses the staged normal rows: its error term is the same
// expression at the same displacements.
//
// G is chosen per colour: 8 lanes when the colour has more bodies than the
// grid has 16-lane groups, else 16, or 32 when even 32-lane groups cover it.
// The tail colours of a pile hold few but heavily loaded bodies (tens of
// rows), and a colour ends when its slowest body does, so wider groups
// there shorten the critical path.
//
// Shared-memory banks: the groups of a warp run in step, so their accesses
// share instructions. A lane's slot is 43 words (odd) and a normal row 9, so
// the lanes of a group write to distinct banks modulo 8; groups start 8, 16
// or 24 banks apart, so the four 8-lane (two 16-lane) groups of a warp
// neither collide on those writes nor on the row reads of the accumulation
// (each group reads within a 14-word row).
constexpr int kRowStride = 14;  // words of one staged row
constexpr int kSlotWords = 43;  // a lane's three rows (42 words) and a pad word
template <int G> struct GroupRowsData {
    // Normal rows kept for the crossing safeguard (rows past them are
    // evaluated again there): 32 for 8-lane groups, 64 for the 16- and
    // 32-lane groups of the heavy bodies (which fit the same staging area).
    static constexpr uint32_t kSlots = G >= 16 ? 64u : 32u;
    // Chunk being accumulated: per lane slot 3 rows of (jacobian[6],
    // stiffness, force, stiffness x jacobian[6]); the last six are the
    // Hessian products' first factors, formed once per row instead of once
    // per entry.
    float r[G][kSlotWords];
    float nrow[kSlots][9];  // normal row: jacobian[6], raw penalty, trial force (and a pad word)
    Blk jblk;            // the block while joint rows are added (joint_rows_shared)
    BodyView jview[2];   // the joint's two bodies during its visit
};
template <int G> struct GroupRows : GroupRowsData<G> {
    // Pads the group to 24 banks mod 32 (8 lanes: bases 0, 24, 16, 8) or 16
    // (16 lanes: bases 0, 16).
    static constexpr int kWords = int(sizeof(GroupRowsData<G>) / 4);
    static constexpr int kTarget = G == 8 ? 24 : G == 16 ? 16 : kWords % 32;
    static constexpr int kPad = (kTarget - kWords % 32 + 32) % 32;
    float pad[kPad == 0 ? 32 : kPad];
    __device__ __forceinline__ float* row(int slot, int x) { return &this->r[slot][kRowStride * x]; }
    __device__ __forceinline__ const float* row(int slot, int x) const { return &this->r[slot][kRowStride * x]; }
};
static_assert(sizeof(GroupRows<8>) / 4 % 32 == 24 && sizeof(GroupRows<16>) / 4 % 32 == 16, "group bank offsets");
// Per-warp staging area: four 8-lane groups, two 16-lane groups or one
// 32-lane group.
constexpr size_t kWarpStage = 4 * sizeof(GroupRows<8>);
static_assert(2 * sizeof(GroupRows<16>) <= kWarpStage && sizeof(GroupRows<32>) <= kWarpStage, "staging area");
// Per-thread slots of the body-per-thread sweep and the dual pass: a block,
// a joint's two body views and its residual contributions, in shared memory
// so the joint visit (a call) reads them there rather than from local memory.
constexpr size_t kThreadViews = 32 * sizeof(Blk);
constexpr size_t kThreadJointRes = kThreadViews + 64 * sizeof(BodyView);
static_assert(kThreadViews % 8 == 0 && kThreadJointRes % 8 == 0, "slot alignment");
static_assert(kThreadJointRes + 32 * sizeof(JointRes) <= kWarpStage, "per-thread joint slots");

__device__ __forceinline__ void entry_ik(int e, int& i, int& k) {
    i = e >= 15 ? 5 : e >= 10 ? 4 : e >= 6 ? 3 : e >= 3 ? 2 : e >= 1 ? 1 : 0;
    k = e - i * (i + 1) / 2;
}

// Lane gl owns entries gl, gl+G, gl+2G, ... (those below 27).
template <int G> struct Owned {
    static constexpr int E = (27 + G - 1) / G;
};
template <int G>
__device__ __forceinline__ void gather_block(const float* ent, Blk& blk, uint32_t gmask, int gbase) {
#pragma unroll
    for (int e = 0; e < 21; ++e) blk.h[e] = __shfl_sync(gmask, ent[e / G], gbase + (e % G));
#pragma unroll
    for (int r = 0; r < 6; ++r) blk.g[r] = __shfl_sync(gmask, ent[(21 + r) / G], gbase + ((21 + r) % G));
}
template <int G> __device__ __forceinline__ void own_entries(const Blk& blk, int gl, float* ent) {
#pragma unroll
    for (int m = 0; m < Owned<G>::E; ++m) {
        const int e = gl + G * m;
        float v = 0.0f;
#pragma unroll
        for (int q = 0; q < 21; ++q) v = e == q ? blk.h[q] : v;
#pragma unroll
        for (int r = 0; r < 6; ++r) v = e == 21 + r ? blk.g[r] : v;
        ent[m] = v;
    }
}

template <int G>
__device__ __forceinline__ void accumulate_chunk(float* ent, int gl, const GroupRows<G>& sm, uint32_t m) {
    static_assert(G <= 8 || G % 4 == 0, "wide groups take rows four at a time");
    // Products first (independent, pipelined loads), then the ordered adds.
#pragma unroll
    for (int q = 0; q < Owned<G>::E; ++q) {
        const int e = gl + G * q;
        if (e >= 27) continue;
        int ei = 0, ek = 0;
        const bool hess = e < 21;
        if (hess) entry_ik(e, ei, ek);
        else ei = e - 21;
        if (G <= 8) {
            float prod[G][3];
#pragma unroll
            for (int t = 0; t < G; ++t)
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    const float* row = sm.row(t, x);
                    prod[t][x] = hess ? row[8 + ei] * row[ek] : row[ei] * row[7];
                }
#pragma unroll
            for (int t = 0; t < G; ++t)
#pragma unroll
                for (int x = 0; x < 3; ++x)
                    if (t < int(m)) ent[q] += prod[t][x];
        } else {
            // Four rows' products at a time (their loads in flight together),
            // then their adds in row order; products of rows past m are
            // formed from the slot's stale values and dropped.
            for (int t0 = 0; t0 < int(m); t0 += 4) {
                float prod[4][3];
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int x = 0; x < 3; ++x) {
                        const float* row = sm.row(t0 + u, x);
                        prod[u][x] = hess ? row[8 + ei] * row[ek] : row[ei] * row[7];
                    }
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int x = 0; x < 3; ++x)
                        if (t0 + u < int(m)) ent[q] += prod[u][x];
            }
        }
    }
}

// Whether a staged normal row's trial force crosses zero under the update
// (geometry_constraints_solve.slang:433-475).
__device__ __forceinline__ bool crosses(const float* row, const V6& upd) {
    V6 nr;
#pragma unroll
    for (int k = 0; k < 6; ++k) nr.v[k] = row[k];
    const float k0 = row[6], trial = row[7];
    return trial <= 0.0f && trial + k0 * dot6(nr, upd) > k0 * 1.0e-6f;
}
// Adds the crossing rows of a chunk (bit t of `mask`: row s0 + t) to the
// lane's entries, rows in list order.
template <int G>
__device__ __forceinline__ void accumulate_crossing(float* ent, int gl, const GroupRows<G>& sm, uint32_t s0,
                                                    uint32_t m, uint32_t mask) {
#pragma unroll
    for (int q = 0; q < Owned<G>::E; ++q) {
        const int e = gl + G * q;
        if (e >= 27) continue;
        int ei = 0, ek = 0;
        if (e < 21) entry_ik(e, ei, ek);
        for (uint32_t t = 0; t < m; ++t) {
            if (!((mask >> t) & 1u)) continue;
            const float* row = sm.nrow[(s0 + t) % GroupRows<G>::kSlots];
            if (e < 21) ent[q] += row[6] * row[ei] * row[ek];
            else ent[q] += row[e - 21] * row[7];
        }
    }
}

// What a body's solve reads of one of its contact rows: the contact (code:
// index, bit 31 set when the body is the contact's second body) and the other
// body. Loaded apart from the arithmetic so a body's first rows can be in
// flight while its own state arrives.
struct RawContact {
    uint32_t c;
    bool first;
    Lite other;
    float2 mub;  // the pair's friction and penalty growth factor
    float4 lam, pen, e;
    V6 ja[3], jb[3];
};
__device__ __forceinline__ RawContact load_contact(const Dev& d, uint32_t code, uint32_t other_body) {
    RawContact r;
    r.c = code & 0x7fffffffu;
    r.first = (code >> 31) == 0;
    r.other = load_lite(d, other_body);
    r.mub = d.c_mub[r.c];
    r.lam = d.c_lam[r.c];
    r.pen = d.c_pen[r.c];
    r.e = d.c_e[r.c];
    load_jac(d, r.c, r.ja, r.jb);
    return r;
}

// Rows of one contact for body i into chunk slot `slot`; its normal row,
// raw penalty and normal trial also go to nrow[nslot].
template <int G>
__device__ __forceinline__ void stage_loaded(const Dev& d, const Lite& me, const RawContact& rc,
                                             uint32_t phase, float dt, GroupRows<G>& sm, int slot, int nslot) {
    const uint32_t c = rc.c;
    const bool first = rc.first;
    const Lite A = first ? me : rc.other;  // values, not run-time references (no local copies)
    const Lite B = first ? rc.other : me;
    const float friction = rc.mub.x;
    const float4 lam = rc.lam, pen = rc.pen;
    V6 ja[3], jb[3];
    float err[3];
    {
        // contact_rows' error terms, from the loaded jacobians
        const float e3[3] = {rc.e.x, rc.e.y, rc.e.z};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            ja[k] = rc.ja[k];
            jb[k] = rc.jb[k];
            err[k] = e3[k] + dot6(ja[k], A.dx) + dot6(jb[k], B.dx);
        }
    }
    F3 trial{lam.x + pen.x * err[0], lam.y + pen.y * err[1], lam.z + pen.z * err[2]};
    if (nslot >= 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) sm.nrow[nslot][k] = first ? ja[0].v[k] : jb[0].v[k];
        sm.nrow[nslot][6] = pen.x;
        sm.nrow[nslot][7] = trial.n;
    }
    if (slot < 0) return;
    F3 f, sc;
    project_with_scales(trial, friction, f, sc);
    float forces[3] = {f.n, f.t0, f.t1};
    if (phase != 0) {
        const float4 fo = d.c_foff[c];
        forces[0] = f.n - fo.x;
        forces[1] = f.t0 - fo.y;
        forces[2] = f.t1 - fo.z;
    }
    const float st[3] = {pen.x * sc.n, pen.y * sc.t0, pen.z * sc.t1};
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        // Values selected element by element: a reference chosen at run time
        // between the two arrays would give them addresses (local memory).
        V6 row;
#pragma unroll
        for (int k = 0; k < 6; ++k) row.v[k] = first ? ja[x].v[k] : jb[x].v[k];
        float* out = sm.row(slot, x);
#pragma unroll
        for (int k = 0; k < 6; ++k) out[k] = row.v[k];
        out[6] = st[x];
        out[7] = forces[x];
#pragma unroll
        for (int k = 0; k < 6; ++k) out[8 + k] = st[x] * row.v[k];  // = (stiffness x J_i), as before
    }
}
template <int G>
__device__ __forceinline__ void stage_contact(const Dev& d, const Lite& me, uint32_t code,
                                              uint32_t other_body, uint32_t phase, float dt, GroupRows<G>& sm,
                                              int slot, int nslot) {
    stage_loaded<G>(d, me, load_contact(d, code, other_body), phase, dt, sm, slot, nslot);
}

// The body a lane group solves next in its colour, fetched while the current
// one solves (bodies of one colour share no contact, so nothing the current
// body writes is read here): its record and this lane's row codes of its
// first two chunks.
struct Ahead {
    uint32_t i, ro, rn;
    uint32_t code0, other0, code1, other1;
    uint32_t impact;  // the body's impact flag (the velocity phase solves impacted bodies only)
};
template <int G>
__device__ __forceinline__ void fetch_codes(const Dev& d, Ahead& a, int gl) {
    const uint32_t s0 = uint32_t(gl), s1 = uint32_t(gl) + uint32_t(G);
    a.code0 = s0 < a.rn ? d.blist[a.ro + s0] : 0u;
    a.other0 = s0 < a.rn ? d.bother[a.ro + s0] : 0u;
    a.code1 = s1 < a.rn ? d.blist[a.ro + s1] : 0u;
    a.other1 = s1 < a.rn ? d.bother[a.ro + s1] : 0u;
}
template <int G>
__device__ __forceinline__ Ahead fetch_ahead(const Dev& d, uint32_t k, int gl) {
    const uint4 r = d.crec[k];
    Ahead a{r.x, r.y, r.z, 0u, 0u, 0u, 0u, r.w};
    fetch_codes<G>(d, a, gl);
    return a;
}

// Joint rows of body i added to its block (geometry_constraints_solve.slang:
// 381-400, the serial loop's order). The joint visit takes the block's
// address, so lane 0 works on a copy in the group's shared-memory slot `sb`
// and the group reads the result back: the register block never needs an
// address (which would put it in local memory for every body).
template <int G>
__device__ __forceinline__ void joint_rows_shared(const Dev& d, uint32_t i, uint32_t phase, float dt, Blk& blk,
                                                  Blk* sb, BodyView* views, uint32_t gmask, int gl) {
    if (gl == 0) {
        *sb = blk;
        const uint32_t jcnt = d.jdeg[i], jlo = d.jinc_off[i];
        for (uint32_t k = 0; k < jcnt; ++k) {
            const uint32_t j = d.jinc_list[jlo + k];
            const JointState js = d.jstate[j];
            if (!js.enabled) continue;
            const uint32_t a = js.dense_a, b = js.dense_b;
            const bool first = i == a;
            if (phase == 0) {
                views[0] = load_body(d, a);
                views[1] = load_body(d, b);
                visit_joint(d.joints[j], d.jrows + size_t(j) * 18, views[0], views[1], v3(d.x[a]), q4(d.q[a]),
                            v3(d.x[b]), q4(d.q[b]), d.p0[a], d.p0[b], dt, sb, first, kVisitAccumulate, nullptr);
            } else {
                const Lite A = load_lite(d, a), B = load_lite(d, b);
                for (uint32_t r = 0; r < js.count; ++r) {
                    Row row = load_row(d.jrows[size_t(j) * 18 + r]);
                    if (row.stiffness >= kMaxPenalty) row_accumulate(*sb, row, first, A.dx, B.dx, dt);
                }
            }
        }
    }
    __syncwarp(gmask);
    blk = *sb;
    __syncwarp(gmask);
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Joints: the world has joints (a world without them gets a build with no
// joint code, which needs fewer registers).
// ah: the body (its record and this lane's first row codes, fetched ahead);
// on return it holds the same for slot kn of the colour order (~0u: none).
template <int G, bool Joints>
__device__ void solve_body_group(const Dev& d, Ahead& ah, uint32_t kn, uint32_t phase, float dt, GroupRows<G>& sm,
                                 uint32_t gmask, int gl, int gbase, uint32_t trace = 0) {
    // trace 1: slowest body of the colour per stage; 2: stage times summed
    // over the colour's bodies (profiling only).
    const unsigned long long t0 = trace ? gtimer() : 0ull;
    auto mark = [&](int k) {
        if (trace == 1 && gl == 0) atomicMax(&d.ctr->dbg_body[k], gtimer() - t0);
        if (trace == 2 && gl == 0) atomicAdd(&d.ctr->dbg_sum[k], gtimer() - t0);
    };
    const uint32_t i = ah.i, ro = ah.ro, rn = ah.rn;
    const uint32_t code0 = ah.code0, other0 = ah.other0, code1 = ah.code1, other1 = ah.other1;
    uint4 nrec = make_uint4(0u, 0u, 0u, 0u);
    if (kn != ~0u) nrec = d.crec[kn];
    const Lite me = load_lite(d, i);
    float ent[Owned<G>::E];
    const float4 ia = d.inA[i], ib = d.inB[i];
    // The block's starting entries: inertia and its gradient. Formed after
    // the first chunk's rows are requested, so those loads and this body's
    // own state are in flight together.
    // The inertia block H is zero outside the linear diagonal and the
    // angular 3x3. Its gradient H dx is the serial sum over c = 0..5 from +0;
    // with dx finite, the sum's zero terms (0 x dx[c], exact zeros) leave
    // every partial sum unchanged (it is never -0), so each sum reduces to
    // its nonzero terms in order, bit for bit; a non-finite dx (0 x inf is
    // NaN) takes the full sums. All indices are compile-time (a lane's entry
    // picks its value by comparison), so nothing goes to local memory.
    auto init_entries = [&] {
        const V6& x = me.dx;
        bool finite = true;
#pragma unroll
        for (int c = 0; c < 6; ++c) finite = finite && fab(x.v[c]) < kFltMax;
        float gr[6];
        if (finite) {
            gr[0] = 0.0f + ia.x * x.v[0];
            gr[1] = 0.0f + ia.x * x.v[1];
            gr[2] = 0.0f + ia.x * x.v[2];
            gr[3] = ((0.0f + ia.y * x.v[3]) + ia.z * x.v[4]) + ib.x * x.v[5];
            gr[4] = ((0.0f + ia.z * x.v[3]) + ia.w * x.v[4]) + ib.y * x.v[5];
            gr[5] = ((0.0f + ib.x * x.v[3]) + ib.y * x.v[4]) + ib.z * x.v[5];
        } else {
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
            for (int r = 0; r < 6; ++r) {
                float gs = 0.0f;
#pragma unroll
                for (int c = 0; c < 6; ++c) gs += H[bidx(r, c)] * x.v[c];
                gr[r] = gs;
            }
        }
#pragma unroll
        for (int q = 0; q < Owned<G>::E; ++q) {
            const int e = gl + G * q;
            float v = 0.0f;
            v = (e == int(bidx(0, 0)) || e == int(bidx(1, 1)) || e == int(bidx(2, 2))) ? ia.x : v;
            v = e == int(bidx(3, 3)) ? ia.y : v;
            v = e == int(bidx(4, 3)) ? ia.z : v;
            v = e == int(bidx(5, 3)) ? ib.x : v;
            v = e == int(bidx(4, 4)) ? ia.w : v;
            v = e == int(bidx(5, 4)) ? ib.y : v;
            v = e == int(bidx(5, 5)) ? ib.z : v;
#pragma unroll
            for (int r = 0; r < 6; ++r) v = e == 21 + r ? gr[r] : v;
            ent[q] = v;
        }
    };
    if (rn == 0) init_entries();
    for (uint32_t base = 0; base < rn; base += G) {
        const uint32_t sidx = base + gl;
        if (sidx < rn) {
            const int nslot = sidx < GroupRows<G>::kSlots ? int(sidx) : -1;
            const uint32_t code = base == 0 ? code0 : base == uint32_t(G) ? code1 : d.blist[ro + sidx];
            const uint32_t other = base == 0 ? other0 : base == uint32_t(G) ? other1 : d.bother[ro + sidx];
            stage_contact<G>(d, me, code, other, phase, dt, sm, gl, nslot);
        }
        if (base == 0) init_entries();
        __syncwarp(gmask);
        accumulate_chunk<G>(ent, gl, sm, min(uint32_t(G), rn - base));
        __syncwarp(gmask);
    }
    // The next body's record and row codes, in flight while this one solves.
    if (kn != ~0u) {
        ah.i = nrec.x;
        ah.ro = nrec.y;
        ah.rn = nrec.z;
        ah.impact = nrec.w;
        fetch_codes<G>(d, ah, gl);
    }
    mark(0);
    Blk blk;
    gather_block<G>(ent, blk, gmask, gbase);
    mark(1);
    if constexpr (Joints) {
        if (d.jdeg[i]) joint_rows_shared<G>(d, i, phase, dt, blk, &sm.jblk, sm.jview, gmask, gl);
    }
    V6 upd;
    if (!block_solve(blk, upd)) return;
    mark(2);
    // The body's rotation offset, read while the safeguard runs (only this
    // group writes it in the colour), so the update at the end waits on no
    // load; its displacement is `me` (read at the start; both w are 0).
    const float4 dq_start = phase == 0 ? d.dq[i] : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    // Crossing safeguard (geometry_constraints_solve.slang:433-475): a
    // ballot per chunk flags the rows; rows past the kept normal rows are
    // evaluated again into the slots. (Reloading the entries from the block
    // keeps them out of registers during the factorisation: keeping them
    // live instead, when no joint rows changed the block, was slower.)
    own_entries<G>(blk, gl, ent);
    constexpr uint32_t kSlots = GroupRows<G>::kSlots;
    constexpr uint32_t kLanes = G == 32 ? 0xffffffffu : (1u << G) - 1u;
    bool crossing = false;
    for (uint32_t base = 0; base < rn; base += G) {
        const uint32_t sidx = base + gl;
        if (base >= kSlots) {
            __syncwarp(gmask);  // the slots' previous rows are read
            if (sidx < rn)
                stage_contact<G>(d, me, d.blist[ro + sidx], d.bother[ro + sidx], phase, dt, sm, -1,
                                 int(sidx % kSlots));
            __syncwarp(gmask);
        }
        const bool f = sidx < rn && crosses(sm.nrow[sidx % kSlots], upd);
        const uint32_t m = (__ballot_sync(gmask, f) >> gbase) & kLanes;
        if (m) {
            crossing = true;
            accumulate_crossing<G>(ent, gl, sm, base % kSlots, min(uint32_t(G), rn - base), m);
        }
    }
    mark(3);
    if (crossing) {
        gather_block<G>(ent, blk, gmask, gbase);
        V6 safe;
        if (block_solve(blk, safe)) upd = safe;
    }
    mark(4);
    if (trace == 1 && gl == 0) atomicMax(&d.ctr->dbg_rn, rn);
    if (trace == 2 && gl == 0) {
        atomicAdd(&d.ctr->dbg_sum[6], 1ull);
        atomicAdd(&d.ctr->dbg_sum[7], (unsigned long long)rn);
    }
    if (gl == 0) {
        float4 l = make_float4(me.dx.v[0], me.dx.v[1], me.dx.v[2], 0.0f);
        if (phase == 0) {
            apply_pose_update(d, i, upd, l, dq_start);
        } else {
            float4 a = make_float4(me.dx.v[3], me.dx.v[4], me.dx.v[5], 0.0f);
            l.x += upd.v[0];
            l.y += upd.v[1];
            l.z += upd.v[2];
            a.x += upd.v[3];
            a.y += upd.v[4];
            a.z += upd.v[5];
            d.dxl[i] = l;
            d.dxa[i] = a;
        }
    }
}

// One thread solves body i: the serial loop of geometry_constraints_solve.
// slang:339-475 as written -- add_row per contact row in list order, the
// joints' rows, LDL^T, then the crossing safeguard over the normal rows --
// for colours with far more bodies than the grid has lane groups, where a
// body per thread finishes the colour in fewer rounds than wider groups.
// `sb`: this thread's shared-memory block slot for the joint visit.
__device__ __forceinline__ void load_normal_rows(const Dev& d, uint32_t c, V6& ja, V6& jb) {
    const float4* p = d.c_jac + size_t(c) * 9;
    const float4 a0 = p[0], a1 = p[1], b4 = p[4], b5 = p[5];  // floats 0-7 and 16-23
    ja = {{a0.x, a0.y, a0.z, a0.w, a1.x, a1.y}};
    jb = {{b4.z, b4.w, b5.x, b5.y, b5.z, b5.w}};
}
template <bool Joints>
__device__ void solve_body_thread(const Dev& d, uint32_t i, uint32_t phase, float dt, Blk* sb, BodyView* views) {
    const Lite me = load_lite(d, i);
    const uint32_t ro = d.roff[i], rn = d.rcount[i];
    Blk blk;
    {
        const float4 ia = d.inA[i], ib = d.inB[i];
#pragma unroll
        for (int k = 0; k < 21; ++k) blk.h[k] = 0.0f;
        blk.h[bidx(0, 0)] = ia.x;
        blk.h[bidx(1, 1)] = ia.x;
        blk.h[bidx(2, 2)] = ia.x;
        blk.h[bidx(3, 3)] = ia.y;
        blk.h[bidx(4, 3)] = ia.z;
        blk.h[bidx(5, 3)] = ib.x;
        blk.h[bidx(4, 4)] = ia.w;
        blk.h[bidx(5, 4)] = ib.y;
        blk.h[bidx(5, 5)] = ib.z;
#pragma unroll
        for (int r = 0; r < 6; ++r) {
            float gs = 0.0f;
#pragma unroll
            for (int c = 0; c < 6; ++c) gs += blk.h[bidx(r, c)] * me.dx.v[c];
            blk.g[r] = gs;
        }
    }
    for (uint32_t r = 0; r < rn; ++r) {
        const uint32_t code = d.blist[ro + r], other_body = d.bother[ro + r];
        const uint32_t c = code & 0x7fffffffu;
        const bool first = (code >> 31) == 0;
        const Lite other = load_lite(d, other_body);
        const Lite A = first ? me : other, B = first ? other : me;
        const float friction = d.c_mub[c].x;
        const float4 lam = d.c_lam[c], pen = d.c_pen[c];
        V6 ja[3], jb[3];
        float err[3];
        contact_rows(d, c, d.c_e[c], A, B, ja, jb, err);
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
        const float st[3] = {pen.x * sc.n, pen.y * sc.t0, pen.z * sc.t1};
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            V6 row;
#pragma unroll
            for (int k = 0; k < 6; ++k) row.v[k] = first ? ja[x].v[k] : jb[x].v[k];
            add_row(blk, row, st[x], forces[x]);
        }
    }
    if constexpr (Joints) {
        if (d.jdeg[i]) {
            // The joint visit takes the block's address: work on this thread's
            // shared-memory copy so the register block never needs one.
            *sb = blk;
            const uint32_t jcnt = d.jdeg[i], jlo = d.jinc_off[i];
            for (uint32_t k = 0; k < jcnt; ++k) {
                const uint32_t j = d.jinc_list[jlo + k];
                const JointState js = d.jstate[j];
                if (!js.enabled) continue;
                const uint32_t a = js.dense_a, b = js.dense_b;
                const bool first = i == a;
                if (phase == 0) {
                    views[0] = load_body(d, a);
                    views[1] = load_body(d, b);
                    visit_joint(d.joints[j], d.jrows + size_t(j) * 18, views[0], views[1], v3(d.x[a]), q4(d.q[a]),
                                v3(d.x[b]), q4(d.q[b]), d.p0[a], d.p0[b], dt, sb, first, kVisitAccumulate, nullptr);
                } else {
                    const Lite A = load_lite(d, a), B = load_lite(d, b);
                    for (uint32_t r = 0; r < js.count; ++r) {
                        Row row = load_row(d.jrows[size_t(j) * 18 + r]);
                        if (row.stiffness >= kMaxPenalty) row_accumulate(*sb, row, first, A.dx, B.dx, dt);
                    }
                }
            }
            blk = *sb;
        }
    }
    V6 upd;
    if (!block_solve(blk, upd)) return;
    // Crossing safeguard: the normal rows again, at the same displacements.
    bool crossing = false;
    for (uint32_t r = 0; r < rn; ++r) {
        const uint32_t code = d.blist[ro + r], other_body = d.bother[ro + r];
        const uint32_t c = code & 0x7fffffffu;
        const bool first = (code >> 31) == 0;
        const Lite other = load_lite(d, other_body);
        const Lite A = first ? me : other, B = first ? other : me;
        V6 ja, jb;
        load_normal_rows(d, c, ja, jb);
        const float err0 = d.c_e[c].x + dot6(ja, A.dx) + dot6(jb, B.dx);
        const float k0 = d.c_pen[c].x;
        const float trial = d.c_lam[c].x + k0 * err0;
        V6 nr;
#pragma unroll
        for (int k = 0; k < 6; ++k) nr.v[k] = first ? ja.v[k] : jb.v[k];
        if (trial <= 0.0f && trial + k0 * dot6(nr, upd) > k0 * 1.0e-6f) {
            add_row(blk, nr, k0, trial);
            crossing = true;
        }
    }
    if (crossing) {
        V6 safe;
        if (block_solve(blk, safe)) upd = safe;
    }
    if (phase == 0) {
        apply_pose_update(d, i, upd);
    } else {
        float4 l = d.dxl[i], a = d.dxa[i];
        l.x += upd.v[0];
        l.y += upd.v[1];
        l.z += upd.v[2];
        a.x += upd.v[3];
        a.y += upd.v[4];
        a.z += upd.v[5];
        d.dxl[i] = l;
        d.dxa[i] = a;
    }
}

// Residual accumulator of one dual pass (this build's addition): rows that
// carry force or penetrate contribute |C_n| (force > 0) or C_n (penetration
// only); hard joint rows contribute |C|. Reported as the RMS, the largest
// value, and the number of rows above the schedule's tolerance.
struct Res {
    double sq;
    uint32_t n;
    float mx;
    uint32_t over;
    float tol;
};
__device__ __forceinline__ void res_add(Res& r, float v) {
    r.sq += double(v) * double(v);
    r.n += 1;
    r.mx = fmx(r.mx, v);
    if (v > r.tol) r.over += 1;
}

// advance_duals for one contact point (geometry_constraints_solve.slang:
// 494-532; the last-iteration block runs in k_contact_finalize). ab: the
// contact's bodies (c_bodies[c]), loaded by the caller ahead of time.
static __device__ void dual_contact(const Dev& d, uint32_t c, uint2 ab, float dt, uint32_t phase, Res& res,
                                    uint32_t it) {
    const uint32_t a = ab.x, b = ab.y;
    if (phase != 0 && d.impact[a] == 0 && d.impact[b] == 0) return;
    // Batched worlds: a scene past its budget is finished; its last sweep
    // feeds the scene's residual.
    uint32_t scene = 0;
    bool scene_last = false;
    if (batched(d)) {
        scene = d.scene_of[a];
        const uint32_t budget = d.scene_budget[scene];
        if (it >= budget) return;
        scene_last = phase == 0 && it + 1 == budget;  // the tick's residual is the pose phase's
    }
    const Lite A = load_lite(d, a), B = load_lite(d, b);
    const float2 mub = d.c_mub[c];
    const float friction = mub.x, beta = mub.y;
    float4 lam = d.c_lam[c], pen = d.c_pen[c];
    V6 ja[3], jb[3];
    float err[3];
    contact_rows(d, c, d.c_e[c], A, B, ja, jb, err);
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

// slots: this thread's two body views and joint residual in shared memory
// (nullptr: local ones, for kernels without the per-thread slots).
static __device__ void dual_joint(const Dev& d, uint32_t j, uint32_t phase, float dt, Res& res, uint32_t it,
                                  BodyView* views = nullptr, JointRes* jres = nullptr) {
    JointState js = d.jstate[j];
    if (js.count == 0 || !js.enabled) return;
    const uint32_t a = js.dense_a, b = js.dense_b;
    if (phase != 0 && d.impact[a] == 0 && d.impact[b] == 0) return;
    uint32_t scene = 0;
    bool scene_last = false;
    if (batched(d)) {
        scene = d.scene_of[a];
        const uint32_t budget = d.scene_budget[scene];
        if (it >= budget) return;
        scene_last = it + 1 == budget;
    }
    float impulse = 0.0f;
    if (phase == 0) {
        BodyView local_views[2];
        JointRes local_res;
        BodyView* v = views ? views : local_views;
        JointRes* out = jres ? jres : &local_res;
        v[0] = load_body(d, a);
        v[1] = load_body(d, b);
        *out = JointRes{0.0, 0u, 0.0f, 0u};
        // An advance visit leaves the block alone (no block pointer).
        impulse = visit_joint(d.joints[j], d.jrows + size_t(j) * 18, v[0], v[1], v3(d.x[a]), q4(d.q[a]), v3(d.x[b]),
                              q4(d.q[b]), d.p0[a], d.p0[b], dt, nullptr, true, kVisitAdvance, nullptr, out, res.tol);
        // The joint's own residual (a batched world also needs it per scene),
        // added in the same order as a running sum would.
        const JointRes jr = *out;
        res.sq += jr.sq;
        res.n += jr.n;
        res.mx = fmx(res.mx, jr.mx);
        res.over += jr.over;
        if (scene_last && jr.n) {
            atomicAdd(&d.scene_res_sq[scene], float(jr.sq));
            atomicAdd(&d.scene_res_n[scene], jr.n);
            atomicMax(reinterpret_cast<int*>(&d.scene_res_mx[scene]), __float_as_int(fmx(jr.mx, 0.0f)));
        }
    } else {
        const Lite A = load_lite(d, a), B = load_lite(d, b);
        for (uint32_t r = 0; r < js.count; ++r) {
            JointRow& s = d.jrows[size_t(j) * 18 + r];
            Row row = load_row(s);
            impulse += fab(row.stiffness < kMaxPenalty ? row.reference_force : row_force(row, A.dx, B.dx, dt)) * dt;
            if (row.stiffness >= kMaxPenalty) store_row(s, row_advance(row, A.dx, B.dx));
        }
    }
    js.applied = impulse;
    const float thr = d.joints[j].breaking_threshold;
    if (thr > 0.0f && impulse > thr) {
        js.broken = 1;
        js.enabled = 0;
    }
    d.jstate[j] = js;
}

// One block's residual partials into slot `slot` of the counters: warp
// trees, then warps in order (deterministic).
template <int T>
__device__ __forceinline__ void block_residual(Res res, double* wsq, uint32_t* wn, float* wmx, uint32_t* wov,
                                               Counters* c, uint32_t slot) {
    for (int o = 16; o > 0; o >>= 1) {
        res.sq += __shfl_xor_sync(0xffffffffu, res.sq, o);
        res.n += __shfl_xor_sync(0xffffffffu, res.n, o);
        res.mx = fmx(res.mx, __shfl_xor_sync(0xffffffffu, res.mx, o));
        res.over += __shfl_xor_sync(0xffffffffu, res.over, o);
    }
    if ((threadIdx.x & 31) == 0) {
        wsq[threadIdx.x >> 5] = res.sq;
        wn[threadIdx.x >> 5] = res.n;
        wmx[threadIdx.x >> 5] = res.mx;
        wov[threadIdx.x >> 5] = res.over;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double bs = 0.0;
        uint32_t bn = 0, bo = 0;
        float bm = 0.0f;
        for (int k = 0; k < T / 32; ++k) {
            bs += wsq[k];
            bn += wn[k];
            bm = fmx(bm, wmx[k]);
            bo += wov[k];
        }
        c->res_sum[slot] = bs;
        c->res_cnt[slot] = bn;
        c->res_mx[slot] = bm;
        c->res_over[slot] = bo;
    }
}

// The sweep's residual from every block's partials (slots base .. base +
// gridDim.x): RMS, largest row violation, fraction of rows above the
// tolerance, and whether the schedule's measure meets the tolerance
// (residual_norm 0: every row within it; 1: the RMS; 2: at most one row in a
// thousand above it).
struct SweepResidual {
    float rms, mx, over, measure;
    bool met;
};
// Every block needs the same decision, so every block sums the partials in
// slot order. One warp per block reads them -- each lane a slot of every 32,
// all loads in flight at once -- and the block shares the result: when every
// thread walked the slots itself, the whole grid's uncached reads of the same
// few L2 lines kept each sweep's start waiting tens of microseconds.
__device__ __forceinline__ SweepResidual sweep_residual(Counters* c, uint32_t base, const StepParams& sp) {
    __shared__ SweepResidual shared_result;
    if (threadIdx.x < 32) {
        const uint32_t lane = threadIdx.x;
        double tsq = 0.0;
        uint32_t tn = 0, to = 0;
        float tmx = 0.0f;
        constexpr uint32_t kAhead = 5;  // slots per lane loaded together (160 blocks)
        for (uint32_t k0 = 0; k0 < gridDim.x; k0 += 32u * kAhead) {
            double sq[kAhead];
            uint32_t cn[kAhead], ov[kAhead];
            float mx[kAhead];
#pragma unroll
            for (uint32_t j = 0; j < kAhead; ++j) {
                const uint32_t k = k0 + 32u * j + lane;
                const bool in = k < gridDim.x;
                sq[j] = in ? ((volatile double*)c->res_sum)[base + k] : 0.0;
                cn[j] = in ? ((volatile uint32_t*)c->res_cnt)[base + k] : 0u;
                mx[j] = in ? ((volatile float*)c->res_mx)[base + k] : 0.0f;
                ov[j] = in ? ((volatile uint32_t*)c->res_over)[base + k] : 0u;
            }
            // Slot order: chunk j, then lanes in order (the same additions
            // as a serial walk over the slots).
#pragma unroll
            for (uint32_t j = 0; j < kAhead; ++j)
                for (uint32_t l = 0; l < 32u; ++l) {
                    if (k0 + 32u * j + l >= gridDim.x) break;
                    tsq += __shfl_sync(0xffffffffu, sq[j], int(l));
                    tn += __shfl_sync(0xffffffffu, cn[j], int(l));
                    tmx = fmx(tmx, __shfl_sync(0xffffffffu, mx[j], int(l)));
                    to += __shfl_sync(0xffffffffu, ov[j], int(l));
                }
        }
        if (lane == 0) {
            SweepResidual r;
            r.rms = tn ? float(sqrt(tsq / double(tn))) : 0.0f;
            r.mx = tmx;
            r.over = tn ? float(to) / float(tn) : 0.0f;
            if (sp.residual_norm == 1) {
                r.measure = r.rms;
                r.met = r.rms <= sp.tolerance;
            } else if (sp.residual_norm == 2) {
                r.measure = r.over;
                r.met = uint64_t(to) * 1000u <= uint64_t(tn);
            } else {
                r.measure = tmx;
                r.met = tmx <= sp.tolerance;
            }
            shared_result = r;
        }
    }
    __syncthreads();
    return shared_result;
}

__device__ __forceinline__ void atomic_max_pos(float* addr, float v) {
    atomicMax(reinterpret_cast<int*>(addr), __float_as_int(fmx(v, 0.0f)));
}

}  // namespace pmb

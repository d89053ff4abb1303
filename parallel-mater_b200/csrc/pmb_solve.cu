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
#include "pmb_joint.cuh"

namespace pmb {

struct Lite {  // what a contact row needs of a body
    V3 x;
    Q4 q;
    V6 dx;
};
__device__ __forceinline__ Lite load_lite(const Dev& d, uint32_t i) {
    float4 l = d.dxl[i], a = d.dxa[i];
    return {v3(d.tx[i]), q4(d.tq[i]), {{l.x, l.y, l.z, a.x, a.y, a.z}}};
}

// geometry_constraints.slang:508-532
__device__ __forceinline__ void contact_rows(V3 n, V3 pt, V3 anc_a, V3 anc_b, float4 e, const Lite& A, const Lite& B,
                                             V6 ja[3], V6 jb[3], float err[3]) {
    V3 t0, t1;
    basis(n, t0, t1);
    const V3 axes[3] = {n, t0, t1};
    const V3 arm_a = sub(pt, A.x), arm_b = sub(pt, B.x);
    const V3 ra_t = rotate(A.q, anc_a), rb_t = rotate(B.q, anc_b);
    const float e3[3] = {e.x, e.y, e.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        V3 ra = k == 0 ? arm_a : ra_t;
        V3 rb = k == 0 ? arm_b : rb_t;
        ja[k] = jac(mul(axes[k], -1.0f), mul(cross(ra, axes[k]), -1.0f));
        jb[k] = jac(axes[k], cross(rb, axes[k]));
        err[k] = e3[k] + dot6(ja[k], A.dx) + dot6(jb[k], B.dx);
    }
}

__device__ __forceinline__ void apply_pose_update(const Dev& d, uint32_t i, const V6& u) {
    float4 l = d.dxl[i];
    l.x += u.v[0];
    l.y += u.v[1];
    l.z += u.v[2];
    d.dxl[i] = l;
    V3 r{u.v[3], u.v[4], u.v[5]};
    if (r.x == 0.0f && r.y == 0.0f && r.z == 0.0f) return;
    Q4 rel = q4(d.dq[i]);
    Q4 dd = qmul(Q4{r.x, r.y, r.z, 0.0f}, rel);
    rel = qnormalize(Q4{rel.x + 0.5f * dd.x, rel.y + 0.5f * dd.y, rel.z + 0.5f * dd.z, rel.w + 0.5f * dd.w});
    if (rel.w < 0.0f) rel = {-rel.x, -rel.y, -rel.z, -rel.w};
    d.dq[i] = f4(rel);
    d.dxa[i] = make_float4(2.0f * rel.x, 2.0f * rel.y, 2.0f * rel.z, 0.0f);
}

// geometry_constraints_solve.slang:331-491 for one body.
__device__ void solve_body(const Dev& d, uint32_t i, uint32_t phase, float dt) {
    const Lite me = load_lite(d, i);
    const float4 ia = d.inA[i], ib = d.inB[i];
    Blk blk;
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
        blk.g[r] = 0.0f;
#pragma unroll
        for (int c = 0; c < 6; ++c) blk.g[r] += blk.h[bidx(r, c)] * me.dx.v[c];
    }
    const uint32_t lo = d.inc_off[i], cnt = d.deg[i];
    for (uint32_t k = 0; k < cnt; ++k) {
        const uint32_t p = d.inc_list[lo + k];
        const uint32_t a = d.act_a[p], b = d.act_b[p];
        const bool first = i == a;
        const Lite other = load_lite(d, first ? b : a);
        const Lite& A = first ? me : other;
        const Lite& B = first ? other : me;
        const float friction = sqrtf(d.p1[a].x * d.p1[b].x);
        const uint32_t off = d.act_off[p], np = d.act_cnt[p];
        for (uint32_t q = 0; q < np; ++q) {
            const uint32_t c = off + q;
            const float4 n4 = d.c_n[c], lam = d.c_lam[c], pen = d.c_pen[c];
            V6 ja[3], jb[3];
            float err[3];
            contact_rows(v3(n4), v3(d.c_p[c]), v3(d.c_aa[c]), v3(d.c_ab[c]), d.c_e[c], A, B, ja, jb, err);
            F3 trial{lam.x + pen.x * err[0], lam.y + pen.y * err[1], lam.z + pen.z * err[2]};
            F3 f = project_contact(trial, friction);
            F3 s = stiffness_scales(trial, friction);
            float forces[3] = {f.n, f.t0, f.t1};
            if (phase != 0) {
                V3 t0, t1;
                basis(v3(n4), t0, t1);
                const V3 af = v3(d.c_accf[c]);
                forces[0] = f.n - lam.w / dt;
                forces[1] = f.t0 - dot(af, t0) / dt;
                forces[2] = f.t1 - dot(af, t1) / dt;
            }
            const float st[3] = {s.n, s.t0, s.t1};
            const float pk[3] = {pen.x, pen.y, pen.z};
#pragma unroll
            for (int x = 0; x < 3; ++x) add_row(blk, first ? ja[x] : jb[x], pk[x] * st[x], forces[x]);
        }
    }
    const uint32_t jlo = d.jinc_off[i], jcnt = d.jdeg[i];
    for (uint32_t k = 0; k < jcnt; ++k) {
        const uint32_t j = d.jinc_list[jlo + k];
        const JointState js = d.jstate[j];
        if (!js.enabled) continue;
        const uint32_t a = js.dense_a, b = js.dense_b;
        const bool first = i == a;
        if (phase == 0) {
            BodyView A = load_body(d, a), B = load_body(d, b);
            visit_joint(d.joints[j], d.jrows + size_t(j) * 18, A, B, v3(d.x[a]), q4(d.q[a]), v3(d.x[b]), q4(d.q[b]),
                        d.p0[a], d.p0[b], dt, &blk, first, kVisitAccumulate, nullptr, nullptr);
        } else {
            const Lite A = load_lite(d, a), B = load_lite(d, b);
            for (uint32_t r = 0; r < js.count; ++r) {
                Row row = load_row(d.jrows[size_t(j) * 18 + r]);
                if (row.stiffness >= kMaxPenalty) row_accumulate(blk, row, first, A.dx, B.dx, dt);
            }
        }
    }
    V6 upd;
    if (!block_solve(blk, upd)) return;
    bool crossing = false;
    for (uint32_t k = 0; k < cnt; ++k) {
        const uint32_t p = d.inc_list[lo + k];
        const uint32_t a = d.act_a[p], b = d.act_b[p];
        const bool first = i == a;
        const Lite other = load_lite(d, first ? b : a);
        const Lite& A = first ? me : other;
        const Lite& B = first ? other : me;
        const uint32_t off = d.act_off[p], np = d.act_cnt[p];
        for (uint32_t q = 0; q < np; ++q) {
            const uint32_t c = off + q;
            const V3 n = v3(d.c_n[c]), pt = v3(d.c_p[c]);
            const V3 arm_a = sub(pt, A.x), arm_b = sub(pt, B.x);
            V6 ja = jac(mul(n, -1.0f), mul(cross(arm_a, n), -1.0f));
            V6 jb = jac(n, cross(arm_b, n));
            float e = d.c_e[c].x + dot6(ja, A.dx) + dot6(jb, B.dx);
            const V6& nr = first ? ja : jb;
            const float lam0 = d.c_lam[c].x, k0 = d.c_pen[c].x;
            float trial = lam0 + k0 * e;
            if (trial <= 0.0f && trial + k0 * dot6(nr, upd) > k0 * 1.0e-6f) {
                add_row(blk, nr, k0, trial);
                crossing = true;
            }
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

// advance_duals for one pair (geometry_constraints_solve.slang:494-565 without
// the last-iteration block); returns max(0, C_n) over its points.
__device__ float dual_pair(const Dev& d, uint32_t i, float dt) {
    const uint32_t a = d.act_a[i], b = d.act_b[i];
    const Lite A = load_lite(d, a), B = load_lite(d, b);
    const float friction = sqrtf(d.p1[a].x * d.p1[b].x);
    const float beta = (1.0f / (fmx(d.p0[a].x + d.p0[b].x, 1.0e-6f) * dt * dt)) * 100.0f;
    const uint32_t off = d.act_off[i], np = d.act_cnt[i];
    float res = 0.0f;
    for (uint32_t q = 0; q < np; ++q) {
        const uint32_t c = off + q;
        const float4 n4 = d.c_n[c];
        float4 lam = d.c_lam[c], pen = d.c_pen[c];
        V6 ja[3], jb[3];
        float err[3];
        contact_rows(v3(n4), v3(d.c_p[c]), v3(d.c_aa[c]), v3(d.c_ab[c]), d.c_e[c], A, B, ja, jb, err);
        res = fmx(res, err[0]);
        F3 f = project_contact(F3{lam.x + pen.x * err[0], lam.y + pen.y * err[1], lam.z + pen.z * err[2]}, friction);
        float tx = lam.y + pen.y * err[1];
        float ty = lam.z + pen.z * err[2];
        float bound = friction * f.n;
        bool stick = tx * tx + ty * ty <= bound * bound;
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
    }
    return res;
}

__device__ float dual_joint(const Dev& d, uint32_t j, uint32_t phase, float dt) {
    JointState js = d.jstate[j];
    if (js.count == 0 || !js.enabled) return 0.0f;
    const uint32_t a = js.dense_a, b = js.dense_b;
    if (phase != 0 && d.impact[a] == 0 && d.impact[b] == 0) return 0.0f;
    float impulse = 0.0f, res = 0.0f;
    if (phase == 0) {
        BodyView A = load_body(d, a), B = load_body(d, b);
        Blk scratch;
        impulse = visit_joint(d.joints[j], d.jrows + size_t(j) * 18, A, B, v3(d.x[a]), q4(d.q[a]), v3(d.x[b]),
                              q4(d.q[b]), d.p0[a], d.p0[b], dt, &scratch, true, kVisitAdvance, nullptr, &res);
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
    return res;
}

__device__ __forceinline__ void atomic_max_pos(float* addr, float v) {
    atomicMax(reinterpret_cast<int*>(addr), __float_as_int(fmx(v, 0.0f)));
}

__global__ void __launch_bounds__(kBlock) k_solve(Dev d, StepParams sp, uint32_t phase) {
    Counters* c = d.ctr;
    if (phase != 0 && c->impact == 0) return;
    const float dt = sp.dt;
    const uint32_t colors = c->colors;
    uint32_t budget = sp.budget_request;
    if (!sp.realtime && sp.requested == 0) budget = max(budget, c->joint_iters);
    const bool adaptive = phase == 0 && sp.tolerance > 0.0f;
    const uint32_t iters = adaptive ? min(max(sp.max_iterations, 1u), kMaxIterations) : min(budget, kMaxIterations);
    const uint32_t n_act = c->n_act;
    __shared__ float block_res;
    for (uint32_t it = 0; it < iters; ++it) {
        for (uint32_t col = 0; col < colors; ++col) {
            const uint32_t b0 = c->color_off[col], b1 = c->color_off[col + 1];
            for (uint32_t k = b0 + grid_stride_begin(); k < b1; k += grid_stride()) {
                const uint32_t i = d.corder[k];
                if (phase != 0 && d.impact[i] == 0) continue;
                solve_body(d, i, phase, dt);
            }
            if (!grid_sync(c)) return;
        }
        if (threadIdx.x == 0) block_res = 0.0f;
        __syncthreads();
        float res = 0.0f;
        for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
            if (phase != 0 && d.impact[d.act_a[i]] == 0 && d.impact[d.act_b[i]] == 0) continue;
            res = fmx(res, dual_pair(d, i, dt));
        }
        for (uint32_t j = grid_stride_begin(); j < d.nj; j += grid_stride()) res = fmx(res, dual_joint(d, j, phase, dt));
        for (int o = 16; o > 0; o >>= 1) res = fmx(res, __shfl_xor_sync(0xffffffffu, res, o));
        if ((threadIdx.x & 31) == 0) atomic_max_pos(&block_res, res);
        __syncthreads();
        if (threadIdx.x == 0 && phase == 0) atomic_max_pos(&c->residual_trace[it], block_res);
        if (!grid_sync(c)) return;
        bool last = it + 1 == iters;
        if (adaptive && ((volatile float*)c->residual_trace)[it] <= sp.tolerance) last = true;
        if (last) {
            if (grid_stride_begin() == 0) {
                if (phase == 0) {
                    c->iterations = it + 1;
                    c->residual = ((volatile float*)c->residual_trace)[it];
                }
                c->budget = it + 1;
            }
            return;
        }
    }
}

const void* solve_kernel_ptr = reinterpret_cast<const void*>(&k_solve);

// Last-iteration contact work (geometry_constraints_solve.slang:533-561).
__global__ void k_contact_finalize(Dev d, StepParams sp, uint32_t phase) {
    if (phase != 0 && d.ctr->impact == 0) return;
    const float dt = sp.dt;
    const uint32_t n_act = d.ctr->n_act;
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t a = d.act_a[i], b = d.act_b[i];
        if (phase != 0 && d.impact[a] == 0 && d.impact[b] == 0) continue;
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
        const uint32_t off = d.act_off[i], np = d.act_cnt[i];
        for (uint32_t q = 0; q < np; ++q) {
            const uint32_t c = off + q;
            const V3 n = v3(d.c_n[c]);
            float4 lam = d.c_lam[c];
            const float stick = d.c_pen[c].w;
            V3 t0, t1;
            basis(n, t0, t1);
            lam.w = lam.x * dt;
            d.c_lam[c] = lam;
            d.c_accf[c] = f4(mul(add(mul(t0, lam.y), mul(t1, lam.z)), dt));
            if (stick == 0.0f) {
                const V3 pt = v3(d.c_p[c]);
                float4 aa = d.c_aa[c], ab = d.c_ab[c];
                d.c_aa[c] = f4(inv_rotate(qa, sub(pt, xa)), aa.w);
                d.c_ab[c] = f4(inv_rotate(qb, sub(pt, xb)), ab.w);
            }
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

__global__ void k_free_mean(Dev d, uint32_t phase) {
    for (uint32_t r = grid_stride_begin(); r < d.n; r += grid_stride()) {
        if (d.motion[r] != kDynamic || d.parent[r] != r) continue;
        if ((phase != 0 && d.impact[r] == 0) || (d.deg[r] == 0 && d.jdeg[r] == 0)) continue;
        if (d.anchored[r]) continue;
        V3 weighted{0, 0, 0};
        float total = 0.0f;
        for (uint32_t i = r; i < d.n; ++i) {
            if (d.motion[i] != kDynamic || d.parent[i] != r) continue;
            const float mass = 1.0f / fmx(d.p0[i].x, 1.0e-12f);
            weighted = add(weighted, mul(v3(d.dxl[i]), mass));
            total += mass;
        }
        if (total > 0.0f) d.mean[r] = f4(mul(weighted, 1.0f / total));
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

// rigid_avbd_project_hinge_anchors (geometry_constraints_solve.slang:174-209),
// serial over joints as in the reference.
__global__ void k_project_hinges(Dev d, float4* ox, const float4* oq) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (uint32_t j = 0; j < d.nj; ++j) {
        const JointState st = d.jstate[j];
        if (st.count == 0 || !st.enabled || d.joints[j].type != kHinge) continue;
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
    const float dt = sp.dt;
    const uint32_t n_act = d.ctr->n_act;
    // impact_gaps (uses the phase-0 displacements)
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t a = d.act_a[i], b = d.act_b[i];
        if (d.impact[a] == 0 && d.impact[b] == 0) continue;
        const Lite A = load_lite(d, a), B = load_lite(d, b);
        for (uint32_t q = d.act_off[i]; q < d.act_off[i] + d.act_cnt[i]; ++q) {
            const float4 n4 = d.c_n[q];
            const V3 n = v3(n4), pt = v3(d.c_p[q]);
            V6 ja = jac(mul(n, -1.0f), mul(cross(sub(pt, A.x), n), -1.0f));
            V6 jb = jac(n, cross(sub(pt, B.x), n));
            float4 e = d.c_e[q];
            e.x = fmx(0.0f, -(n4.w + dot6(ja, A.dx) + dot6(jb, B.dx)));
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
                    d.p0[a], d.p0[b], dt, &scratch, true, kVisitImpact, nullptr, nullptr);
    }
    const uint32_t n_act = d.ctr->n_act;
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t a = d.act_a[i], b = d.act_b[i];
        if (d.impact[a] == 0 && d.impact[b] == 0) continue;
        const Lite A = load_lite(d, a), B = load_lite(d, b);
        const V6 va = jac(mul(v3(ov[a]), dt), mul(v3(ow[a]), dt));
        const V6 vb = jac(mul(v3(ov[b]), dt), mul(v3(ow[b]), dt));
        const float rest_ab = fmn(d.p1[a].y, d.p1[b].y);
        for (uint32_t q = d.act_off[i]; q < d.act_off[i] + d.act_cnt[i]; ++q) {
            float4 e = d.c_e[q];
            const float gap = e.x;
            V6 ja[3], jb[3];
            float err[3];
            contact_rows(v3(d.c_n[q]), v3(d.c_p[q]), v3(d.c_aa[q]), v3(d.c_ab[q]), e, A, B, ja, jb, err);
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

void launch_solve_all(const Dev& d, const StepParams& sp, cudaStream_t s, int coop_blocks, const SolveBuffers& o) {
    const uint32_t pb = blocks_for(d.cap_pair > d.nj ? d.cap_pair : d.nj);
    for (uint32_t phase = 0; phase < (sp.realtime ? 1u : 2u); ++phase) {
        if (phase != 0) {
            k_impact_setup<<<blocks_for(d.cap_pair), kBlock, 0, s>>>(d, sp, o.ox, o.oq, o.ov, o.ow);
            k_impact_bodies<<<blocks_for(d.n), kBlock, 0, s>>>(d, o.ox, o.oq, o.ov, o.ow);
            k_impact_constraints<<<pb, kBlock, 0, s>>>(d, sp, o.ov, o.ow);
        }
        Dev dd = d;
        uint32_t ph = phase;
        StepParams spp = sp;
        void* args[] = {&dd, &spp, &ph};
        cudaLaunchCooperativeKernel(solve_kernel_ptr, dim3(coop_blocks), dim3(kBlock), args, 0, s);
        k_contact_finalize<<<blocks_for(d.cap_pair), kBlock, 0, s>>>(d, sp, phase);
        k_free_anchor<<<blocks_for(d.cap_pair > d.n ? d.cap_pair : d.n), kBlock, 0, s>>>(d, phase);
        k_free_mean<<<blocks_for(d.n), kBlock, 0, s>>>(d, phase);
        k_free_subtract<<<blocks_for(d.n), kBlock, 0, s>>>(d, phase);
        k_apply<<<blocks_for(d.n), kBlock, 0, s>>>(d, sp, phase, o.ox, o.oq, o.ov, o.ow);
        if (phase == 0 && d.nj) k_project_hinges<<<1, 32, 0, s>>>(d, o.ox, o.oq);
    }
    k_clamp_commit<<<blocks_for(d.n), kBlock, 0, s>>>(d, o.ox, o.oq, o.ov, o.ow);
    k_cache_save<<<blocks_for(d.cap_pair), kBlock, 0, s>>>(d, sp);
}

}  // namespace pmb

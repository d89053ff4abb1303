// SPDX-License-Identifier: MIT
// Joint rows on the device: the reference's rigid_avbd_visit_joint and
// rigid_avbd_visit_joint_row (geometry_constraints.slang:626-926) for all
// eight joint types. One visit re-linearises every row of a joint from the
// current poses; init warm-starts the stored rows, accumulate adds them to a
// body's 6x6 block, advance updates their duals, impact prepares the
// velocity phase.
#pragma once
#include "pmb_world.cuh"

namespace pmb {

enum : unsigned { kVisitInit = 0, kVisitAccumulate = 1, kVisitAdvance = 2, kVisitImpact = 3 };

struct BodyView {
    V3 x;
    Q4 q;
    V6 dx;
    Q4 dq;
    V3 v, w;
};

__device__ __forceinline__ BodyView load_body(const Dev& d, uint32_t i) {
    BodyView b;
    b.x = v3(d.tx[i]);
    b.q = q4(d.tq[i]);
    float4 l = d.dxl[i], a = d.dxa[i];
    b.dx = {{l.x, l.y, l.z, a.x, a.y, a.z}};
    b.dq = q4(d.dq[i]);
    b.v = v3(d.tv[i]);
    b.w = v3(d.tw[i]);
    return b;
}

// geometry_constraints.slang:362-372
__device__ __forceinline__ void body_pose(const BodyView& b, V3& x, Q4& q) {
    x = add(b.x, V3{b.dx.v[0], b.dx.v[1], b.dx.v[2]});
    q = b.q;
    if (b.dq.x != 0.0f || b.dq.y != 0.0f || b.dq.z != 0.0f) q = qnormalize(qmul(b.dq, b.q));
}

// geometry_constraints.slang:401-422
__device__ __forceinline__ V3 log_axis(Q4 frame, V3 lg, unsigned axis) {
    float s = len2(lg);
    float coef = 1.0f / 12.0f + s * (1.0f / 720.0f + s * (1.0f / 30240.0f + s * (1.0f / 1209600.0f + s / 47900160.0f)));
    if (s > 1.0f) {
        float ang = sqrtf(s);
        float half = 0.5f * ang;
        coef = (1.0f - x_cot(half)) / s;
    }
    V3 u = unit_axis(axis);
    V3 l = add(add(u, mul(cross(lg, u), 0.5f)), mul(cross(lg, cross(lg, u)), coef));
    return rotate(frame, l);
}

__device__ __forceinline__ Row load_row(const JointRow& s) {
    Row r;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        r.a.v[k] = s.a[k];
        r.b.v[k] = s.b[k];
    }
    r.dual = {s.lambda, s.penalty};
    r.error = s.error;
    r.velocity = s.velocity;
    r.lower = s.lower;
    r.upper = s.upper;
    r.stiffness = s.stiffness;
    r.damping = s.damping;
    r.beta = s.beta;
    r.reference_force = s.reference_force;
    return r;
}
__device__ __forceinline__ void store_row(JointRow& s, const Row& r) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        s.a[k] = r.a.v[k];
        s.b[k] = r.b.v[k];
    }
    s.lambda = r.dual.lambda;
    s.penalty = r.dual.penalty;
    s.error = r.error;
    s.velocity = r.velocity;
    s.lower = r.lower;
    s.upper = r.upper;
    s.stiffness = r.stiffness;
    s.damping = r.damping;
    s.beta = r.beta;
    s.reference_force = r.reference_force;
}

// Residual contributions of a joint's hard rows in an advance visit: the
// sum of squares, count, largest |C| and count above the tolerance, added
// to the target's fields.
struct JointRes {
    double sq;
    uint32_t n;
    float mx;
    uint32_t over;
};

struct JointCtx {
    JointRow* rows;
    const BodyView* A;
    const BodyView* B;
    Blk* blk;
    uint32_t index;
    float impulse;
    bool first;
    unsigned visit;
    float dt;
    double res_sq;
    uint32_t res_n;
    float res_max;
    uint32_t res_over;  // hard rows whose |C| exceeds res_tol
    float res_tol;
};

// geometry_constraints.slang:626-713
static __device__ void joint_row(JointCtx& c, const V6& ja, const V6& jb, float current, float previous, float penalty,
                          bool angular, float stiffness, float damping, float lower, float upper, bool motor,
                          float motor_speed, V3 curv_a, V3 curv_b, float stabilization) {
    if (c.index >= 18) return;  // a joint stores at most 18 rows
    uint32_t ri = c.index++;
    Row row = load_row(c.rows[ri]);
    const float dt = c.dt;
    float lin = dot6(ja, c.A->dx) + dot6(jb, c.B->dx);
    row.a = ja;
    row.b = jb;
    row.stiffness = stiffness;
    row.damping = damping;
    if (c.visit == kVisitInit) {
        if (!(row.dual.penalty > kMinPenalty)) row.dual.penalty = penalty;
        row.dual = warm_start(row.dual, stiffness);
        if (stiffness < kMaxPenalty) row.dual.lambda = 0.0f;
        row.beta = penalty * (angular ? 10.0f : 100.0f);
        row.reference_force = 0.0f;
    }
    row.error = current - (stiffness < kMaxPenalty ? 0.0f : stabilization * previous) - lin;
    row.velocity = motor ? motor_speed : (current - previous - lin) / dt;
    row.lower = lower;
    row.upper = upper;
    if (c.visit == kVisitAccumulate) {
        row_accumulate(*c.blk, row, c.first, c.A->dx, c.B->dx, dt);
        if (!angular) {
            V3 axis{jb.v[0], jb.v[1], jb.v[2]};
            V3 arm = c.first ? curv_a : curv_b;
            float force = row_force(row, c.A->dx, c.B->dx, dt);
            for (unsigned col = 0; col < 3; ++col) {
                V3 val = sub(mul(add(mul(axis, comp(arm, col)), mul(arm, comp(axis, col))), 0.5f),
                             mul(unit_axis(col), dot(axis, arm)));
                c.blk->h[bidx(3 + col, 3 + col)] += fab(force) * sqrtf(len2(val));
            }
        }
    } else if (c.visit == kVisitAdvance) {
        c.impulse += fab(row_force(row, c.A->dx, c.B->dx, dt)) * dt;
        if (stiffness >= kMaxPenalty) {
            const float v = fab(row_error(row, c.A->dx, c.B->dx));
            c.res_sq += double(v) * double(v);
            c.res_n += 1;
            c.res_max = fmx(c.res_max, v);
            if (v > c.res_tol) c.res_over += 1;
        }
        store_row(c.rows[ri], row_advance(row, c.A->dx, c.B->dx));
    } else if (c.visit == kVisitImpact) {
        if (stiffness < kMaxPenalty) {
            row.reference_force = row_force(row, c.A->dx, c.B->dx, dt);
        } else {
            float gap = lower == 0.0f ? fmn(0.0f, current) : (upper == 0.0f ? fmx(0.0f, current) : 0.0f);
            V6 va = jac(mul(c.A->v, dt), mul(c.A->w, dt));
            V6 vb = jac(mul(c.B->v, dt), mul(c.B->w, dt));
            row.reference_force = row.dual.lambda;
            row.error = dot6(ja, va) + dot6(jb, vb) + gap - (motor ? motor_speed * dt : 0.0f);
        }
        store_row(c.rows[ri], row);
    } else {
        store_row(c.rows[ri], row);
    }
}

// geometry_constraints.slang:715-926. prevA/prevB: start-of-tick poses.
static __device__ float visit_joint(const Joint& o, JointRow* rows, const BodyView& A, const BodyView& B, V3 prev_xa,
                             Q4 prev_qa, V3 prev_xb, Q4 prev_qb, float4 pa0, float4 pb0, float dt, Blk* blk,
                             bool first, unsigned visit, uint32_t* count_out, JointRes* res_out = nullptr,
                             float res_tol = 0.0f) {
    JointCtx c{rows, &A, &B, blk, 0u, 0.0f, first, visit, dt, 0.0, 0u, 0.0f, 0u, res_tol};
    V3 xa, xb;
    Q4 qa, qb;
    body_pose(A, xa, qa);
    body_pose(B, xb, qb);
    const V3 la{o.anchor_a[0], o.anchor_a[1], o.anchor_a[2]}, lb{o.anchor_b[0], o.anchor_b[1], o.anchor_b[2]};
    const Q4 fa_l{o.frame_a[0], o.frame_a[1], o.frame_a[2], o.frame_a[3]};
    const Q4 fb_l{o.frame_b[0], o.frame_b[1], o.frame_b[2], o.frame_b[3]};
    V3 arm_a = rotate(qa, la), arm_b = rotate(qb, lb);
    V3 error = sub(add(xb, arm_b), add(xa, arm_a));
    V3 old_error = sub(add(prev_xb, rotate(prev_qb, lb)), add(prev_xa, rotate(prev_qa, la)));
    const Q4 frame_a = qnormalize(qmul(qa, fa_l)), old_a = qnormalize(qmul(prev_qa, fa_l));
    const uint32_t t = o.type;
    // A point joint has three linear lock rows and no angular row, so its
    // visit skips the relative-rotation terms (same values for every row it
    // does emit).
    const bool angular_rows = t != kPoint;
    const bool swing = t == kHinge || t == kPiston || (t == kMotor && o.motor_angular != 0);
    const V3 free_axis = t == kHinge ? V3{0, 0, 1} : V3{1, 0, 0};
    V3 twist{0, 0, 0}, old_twist{0, 0, 0}, swing_axis{0, 0, 0}, rotation{0, 0, 0}, old_rotation{0, 0, 0};
    Q4 frame_b{0, 0, 0, 1}, old_b{0, 0, 0, 1};
    if (angular_rows) {
        frame_b = qnormalize(qmul(qb, fb_l));
        old_b = qnormalize(qmul(prev_qb, fb_l));
        twist = rotation_vector(qrelative(frame_a, frame_b, true));
        old_twist = rotation_vector(qrelative(old_a, old_b, true));
        swing_axis = inv_rotate(frame_a, rotate(frame_b, free_axis));
        const V3 old_swing = inv_rotate(old_a, rotate(old_b, free_axis));
        rotation = swing ? cross(free_axis, swing_axis) : twist;
        old_rotation = swing ? cross(free_axis, old_swing) : old_twist;
    }
    float lin_pen = 1.0f / (fmx(pa0.x + pb0.x, 1.0e-6f) * dt * dt);
    const bool generic = t == kGeneric || t == kGenericSpring;
    const bool motor_type = t == kMotor;
    for (unsigned axis = 0; axis < 3; ++axis) {
        V3 dir = rotate(frame_a, unit_axis(axis));
        V3 old_dir = rotate(old_a, unit_axis(axis));
        for (unsigned av = 0; av < (angular_rows ? 2u : 1u); ++av) {
            bool angular = av != 0;
            bool lock = angular ? (t == kFixed || t == kSlider || (t == kHinge && axis != 2) ||
                                   (t == kPiston && axis != 0) ||
                                   (motor_type && (axis != 0 || o.motor_angular == 0)))
                                : (t == kFixed || t == kPoint || t == kHinge ||
                                   ((t == kSlider || t == kPiston) && axis != 0) ||
                                   (motor_type && (axis != 0 || o.motor_linear == 0)));
            uint32_t lim_axes = angular ? o.ang_limit_axes : o.lin_limit_axes;
            const float* lim_lo = angular ? o.ang_lower : o.lin_lower;
            const float* lim_hi = angular ? o.ang_upper : o.lin_upper;
            uint32_t spr_axes = angular ? o.ang_spring_axes : o.lin_spring_axes;
            const float* spr_k = angular ? o.ang_stiffness : o.lin_stiffness;
            const float* spr_c = angular ? o.ang_damping : o.lin_damping;
            float current = angular ? comp(rotation, axis) : dot(error, dir);
            float old_current = angular ? comp(old_rotation, axis) : dot(old_error, old_dir);
            V3 ang_axis{0, 0, 0};
            if (angular)
                ang_axis = swing ? rotate(frame_a, sub(mul(unit_axis(axis), dot(free_axis, swing_axis)),
                                                       mul(free_axis, comp(swing_axis, axis))))
                                 : log_axis(frame_a, twist, axis);
            V6 ja = angular ? jac(V3{0, 0, 0}, mul(ang_axis, -1.0f))
                            : jac(mul(dir, -1.0f), add(mul(cross(arm_a, dir), -1.0f), cross(dir, error)));
            V6 jb = angular ? jac(V3{0, 0, 0}, ang_axis) : jac(dir, cross(arm_b, dir));
            float penalty = angular ? 1.0f / (fmx(dot(dir, add(inv_inertia_world(pa0, qa, dir),
                                                               inv_inertia_world(pb0, qb, dir))),
                                                  1.0e-6f) *
                                              dt * dt)
                                    : lin_pen;
            float lock_pen =
                angular ? fmx(penalty, 2.0f * lin_pen * fmx(len2(cross(dir, arm_a)), len2(cross(dir, arm_b)))) : penalty;
            V3 curv_a = add(error, arm_a);
            if (lock) {
                if (visit == kVisitInit && angular && c.index < 18)
                    rows[c.index].penalty = fmx(rows[c.index].penalty, lock_pen / kGamma);
                joint_row(c, ja, jb, current, old_current, lock_pen, angular, kMaxPenalty, 0.0f, -kMaxPenalty,
                          kMaxPenalty, false, 0.0f, curv_a, arm_b, kAlpha);
            }
            bool free_limit = angular ? ((t == kHinge && axis == 2) || (t == kPiston && axis == 0))
                                      : ((t == kSlider || t == kPiston) && axis == 0);
            if ((generic || free_limit) && (lim_axes & (1u << axis)) != 0) {
                float lc = angular ? comp(twist, axis) : current;
                float olc = angular ? comp(old_twist, axis) : old_current;
                V3 lax = log_axis(frame_a, twist, axis);
                V6 la6 = angular ? jac(V3{0, 0, 0}, mul(lax, -1.0f)) : ja;
                V6 lb6 = angular ? jac(V3{0, 0, 0}, lax) : jb;
                float lower = lim_lo[axis], upper = lim_hi[axis];
                if (lower == upper) {
                    float eq_pen = angular && generic ? lock_pen : penalty;
                    if (visit == kVisitInit && angular && generic && c.index < 18)
                        rows[c.index].penalty = fmx(rows[c.index].penalty, eq_pen / kGamma);
                    joint_row(c, la6, lb6, lc - lower, olc - lower, eq_pen, angular, kMaxPenalty, 0.0f, -kMaxPenalty,
                              kMaxPenalty, false, 0.0f, curv_a, arm_b, kAlpha);
                } else if (lower < upper) {
                    joint_row(c, la6, lb6, lc - upper, fmx(olc - upper, 0.0f), penalty, angular, kMaxPenalty, 0.0f,
                              0.0f, kMaxPenalty, false, 0.0f, curv_a, arm_b, 0.8f);
                    joint_row(c, la6, lb6, lc - lower, fmn(olc - lower, 0.0f), penalty, angular, kMaxPenalty, 0.0f,
                              -kMaxPenalty, 0.0f, false, 0.0f, curv_a, arm_b, 0.8f);
                }
            }
            if (t == kGenericSpring && (spr_axes & (1u << axis)) != 0)
                joint_row(c, ja, jb, current, old_current, penalty, angular, spr_k[axis], spr_c[axis], -kMaxPenalty,
                          kMaxPenalty, false, 0.0f, curv_a, arm_b, kAlpha);
            if (motor_type && axis == 0 && (angular ? o.motor_angular != 0 : o.motor_linear != 0)) {
                float speed = angular ? o.motor_angular_velocity : o.motor_linear_velocity;
                float bound = (angular ? o.motor_angular_max_impulse : o.motor_linear_max_impulse) / dt;
                Q4 rel = qrelative(frame_a, frame_b, true);
                Q4 old_rel = qrelative(old_a, old_b, true);
                V3 mrot = rotation_vector(qrelative(Q4{0, 0, 0, 1}, qrelative(old_rel, rel, false), true));
                V3 max_ = log_axis(frame_a, mrot, axis);
                V6 ma = angular ? jac(V3{0, 0, 0}, mul(max_, -1.0f)) : ja;
                V6 mb = angular ? jac(V3{0, 0, 0}, max_) : jb;
                float travel = angular ? comp(mrot, axis) : current - old_current;
                joint_row(c, ma, mb, travel - speed * dt, 0.0f, penalty, angular, kMaxPenalty, 0.0f, -bound, bound,
                          true, speed, curv_a, arm_b, kAlpha);
            }
        }
    }
    if (count_out) *count_out = c.index;
    if (res_out) {
        res_out->sq += c.res_sq;
        res_out->n += c.res_n;
        res_out->mx = fmx(res_out->mx, c.res_max);
        res_out->over += c.res_over;
    }
    return c.impulse;
}

}  // namespace pmb

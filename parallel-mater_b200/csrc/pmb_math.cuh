// SPDX-License-Identifier: MIT
// Device math for the rigid AVBD step. The formulas are the reference's
// (src/slang/math.slang:6-248, src/slang/constraint_math.slang:8-345) written
// for registers: float4-packed vectors, packed 21-entry symmetric blocks.
// The library is compiled with --fmad=false and IEEE division/square root
// (the reference compiles with --fmad=false, CMakeLists.txt:421), and every
// expression keeps the reference's evaluation order, so results track the
// serial FP32 restatement to the last bit except where a libm function
// would round differently on the host and the device: arctangent and
// cotangent are evaluated by atan2_q1 / x_cot below from basic operations.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define PMB_HD __host__ __device__ __forceinline__

namespace pmb {

constexpr uint32_t kInvalid = 0xffffffffu;
constexpr float kEps = 1.0e-6f;
constexpr float kAlpha = 0.99f;
constexpr float kGamma = 0.999f;
constexpr float kMinPenalty = 1.0f;
constexpr float kMaxPenalty = 1.0e10f;
constexpr float kFltMax = 3.402823466e38f;

struct V3 { float x, y, z; };
struct Q4 { float x, y, z, w; };

PMB_HD float rsq(float v) { return 1.0f / sqrtf(v); }
PMB_HD float fmn(float a, float b) { return a < b ? a : b; }
PMB_HD float fmx(float a, float b) { return a > b ? a : b; }
PMB_HD float fab(float a) { return a < 0.0f ? -a : a; }
PMB_HD float fclamp(float v, float lo, float hi) { return fmn(fmx(v, lo), hi); }

PMB_HD V3 v3(float x, float y, float z) { return {x, y, z}; }
PMB_HD V3 v3(float4 a) { return {a.x, a.y, a.z}; }
PMB_HD float4 f4(V3 a, float w = 0.0f) { return make_float4(a.x, a.y, a.z, w); }
PMB_HD Q4 q4(float4 a) { return {a.x, a.y, a.z, a.w}; }
PMB_HD float4 f4(Q4 a) { return make_float4(a.x, a.y, a.z, a.w); }
PMB_HD V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
PMB_HD V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
PMB_HD V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
PMB_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PMB_HD V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
PMB_HD V3 vmin(V3 a, V3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
PMB_HD V3 vmax(V3 a, V3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
PMB_HD float len2(V3 a) { return dot(a, a); }
PMB_HD float len(V3 a) { return sqrtf(len2(a)); }
PMB_HD V3 normalized_or(V3 v, V3 fb) {
    float s = len2(v);
    return s <= kEps * kEps ? fb : mul(v, rsq(s));
}
PMB_HD float comp(V3 v, unsigned k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
PMB_HD V3 unit_axis(unsigned k) { return k == 0 ? V3{1, 0, 0} : (k == 1 ? V3{0, 1, 0} : V3{0, 0, 1}); }

PMB_HD Q4 conj(Q4 q) { return {-q.x, -q.y, -q.z, q.w}; }
PMB_HD Q4 qmul(Q4 a, Q4 b) {
    return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
PMB_HD Q4 qnormalize(Q4 q) {
    float s = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (s <= kEps * kEps) return {0, 0, 0, 0};
    float inv = rsq(s);
    return {q.x * inv, q.y * inv, q.z * inv, q.w * inv};
}
PMB_HD Q4 qrelative(Q4 from, Q4 to, bool local) {
    float c = from.x * to.x + from.y * to.y + from.z * to.z + from.w * to.w;
    if (c < 0.0f) to = {-to.x, -to.y, -to.z, -to.w};
    Q4 d{to.x - from.x, to.y - from.y, to.z - from.z, to.w - from.w};
    Q4 r = local ? qmul(conj(from), d) : qmul(d, conj(from));
    r.w = fab(c);
    return qnormalize(r);
}
PMB_HD V3 rotate(Q4 q, V3 v) {
    V3 u{q.x, q.y, q.z};
    V3 t = mul(cross(u, v), 2.0f);
    return add(v, add(mul(t, q.w), cross(u, t)));
}
PMB_HD V3 inv_rotate(Q4 q, V3 v) { return rotate(conj(q), v); }
PMB_HD V3 rotation_displacement(Q4 from, Q4 to, V3 v) {
    if (from.x * to.x + from.y * to.y + from.z * to.z + from.w * to.w < 0.0f) to = {-to.x, -to.y, -to.z, -to.w};
    V3 o{from.x, from.y, from.z}, n{to.x, to.y, to.z};
    V3 d = sub(n, o);
    V3 oc = cross(o, v), dc = cross(d, v);
    return mul(add(add(mul(oc, to.w - from.w), mul(dc, to.w)), add(cross(d, oc), cross(n, dc))), 2.0f);
}
// Arctangent and cotangent from IEEE-exact basic operations only (+ - * /
// and sqrt, no contraction), so this library and a serial FP32 restatement
// compiled without contraction evaluate them to the same bits; libm atan2f,
// sinf and cosf round differently on the host and on the device.
//
// atan2 for the first quadrant (y >= 0, x >= 0, not both zero): with
// t = min/max in [0, 1], the addition formula atan(t) = pi/6 +
// atan((sqrt(3) t - 1) / (t + sqrt(3))) when t > tan(pi/12) leaves
// |u| <= tan(pi/12), where the Maclaurin series u - u^3/3 + u^5/5 - ... is
// summed to u^15 (truncation below 1e-10 relative); pi/2 - atan(x/y) when
// y > x. A few ulp from the correctly rounded value.
PMB_HD float atan2_q1(float y, float x) {
    const bool swap = y > x;
    const float t = swap ? x / y : y / x;
    const bool shift = t > 0.26794919f;  // tan(pi/12)
    const float u = shift ? (t * 1.7320508f - 1.0f) / (t + 1.7320508f) : t;
    const float u2 = u * u;
    float p = -1.0f / 15.0f;
    p = 1.0f / 13.0f + u2 * p;
    p = -1.0f / 11.0f + u2 * p;
    p = 1.0f / 9.0f + u2 * p;
    p = -1.0f / 7.0f + u2 * p;
    p = 1.0f / 5.0f + u2 * p;
    p = -1.0f / 3.0f + u2 * p;
    p = 1.0f + u2 * p;
    float r = u * p;
    if (shift) r = 0.52359878f + r;  // pi/6
    return swap ? 1.5707964f - r : r;
}
// x cos(x) / sin(x) for x in [0, pi/2]: Maclaurin series of sin to x^15
// and of cos to x^16 (truncation below 1e-9 on that interval).
PMB_HD float x_cot(float x) {
    const float x2 = x * x;
    float s = -1.0f / 1307674368000.0f;            // -1/15!
    s = 1.0f / 6227020800.0f + x2 * s;             //  1/13!
    s = -1.0f / 39916800.0f + x2 * s;              // -1/11!
    s = 1.0f / 362880.0f + x2 * s;                 //  1/9!
    s = -1.0f / 5040.0f + x2 * s;                  // -1/7!
    s = 1.0f / 120.0f + x2 * s;                    //  1/5!
    s = -1.0f / 6.0f + x2 * s;                     // -1/3!
    s = 1.0f + x2 * s;                             // sin(x) / x
    float c = 1.0f / 20922789888000.0f;            //  1/16!
    c = -1.0f / 87178291200.0f + x2 * c;           // -1/14!
    c = 1.0f / 479001600.0f + x2 * c;              //  1/12!
    c = -1.0f / 3628800.0f + x2 * c;               // -1/10!
    c = 1.0f / 40320.0f + x2 * c;                  //  1/8!
    c = -1.0f / 720.0f + x2 * c;                   // -1/6!
    c = 1.0f / 24.0f + x2 * c;                     //  1/4!
    c = -0.5f + x2 * c;                            // -1/2!
    c = 1.0f + x2 * c;                             // cos(x)
    return c / s;                                  // x cos(x) / sin(x)
}
PMB_HD V3 rotation_vector(Q4 d) {
    float s = d.x * d.x + d.y * d.y + d.z * d.z;
    float scale = 2.0f + s * (1.0f / 3.0f + s * (3.0f / 20.0f + s * (5.0f / 56.0f + s * (35.0f / 576.0f))));
    if (s > 0.01f) {
        float vs = sqrtf(s);
        scale = 2.0f * atan2_q1(vs, fclamp(d.w, 0.0f, 1.0f)) / vs;
    }
    return {d.x * scale, d.y * scale, d.z * scale};
}
PMB_HD V3 delta_velocity(Q4 from, Q4 to, float dt) {
    if (dt <= 0.0f) return {0, 0, 0};
    return mul(rotation_vector(qrelative(from, to, false)), 1.0f / dt);
}
PMB_HD V3 clamp_length(V3 v, float m) {
    float s = len2(v);
    if (s <= m * m || s <= kEps * kEps) return v;
    return mul(v, m * rsq(s));
}
PMB_HD V3 inv_inertia_world(float4 inv, Q4 q, V3 v) {
    V3 l = inv_rotate(q, v);
    return rotate(q, V3{l.x * inv.y, l.y * inv.z, l.z * inv.w});
}

// ------------------------------------------------------------------ AVBD
struct Dual { float lambda, penalty; };
PMB_HD Dual warm_start(Dual d, float stiffness) {
    d.lambda *= kAlpha * kGamma;
    d.penalty = fmn(stiffness, fclamp(d.penalty * kGamma, kMinPenalty, kMaxPenalty));
    return d;
}
PMB_HD float dual_force(Dual d, float e, float lo, float hi) { return fclamp(d.lambda + d.penalty * e, lo, hi); }
PMB_HD Dual update_dual(Dual d, float e, float beta, float lo, float hi, float stiffness) {
    float u = d.lambda + d.penalty * e;
    d.lambda = stiffness < kMaxPenalty ? 0.0f : fclamp(u, lo, hi);
    if (u > lo && u < hi) d.penalty = fmn(stiffness, fmn(kMaxPenalty, d.penalty + beta * fab(e)));
    return d;
}
struct F3 { float n, t0, t1; };
PMB_HD float friction_scale(float t0, float t1, float bound) {
    if (bound <= 0.0f) return 0.0f;
    float s = t0 * t0 + t1 * t1;
    return s <= bound * bound ? 1.0f : fmn(1.0f, bound * rsq(s));
}
PMB_HD F3 project_contact(F3 f, float mu) {
    f.n = fmx(f.n, 0.0f);
    float s = friction_scale(f.t0, f.t1, mu * f.n);
    f.t0 *= s;
    f.t1 *= s;
    return f;
}
PMB_HD F3 stiffness_scales(F3 t, float mu) {
    float n = fmx(t.n, 0.0f);
    float s = friction_scale(t.t0, t.t1, mu * n);
    return {t.n > 0.0f ? 1.0f : 0.0f, s, s};
}

// project_contact and stiffness_scales of one trial force: they share the
// friction scale (same inputs), evaluated once.
PMB_HD void project_with_scales(F3 t, float mu, F3& f, F3& sc) {
    const float n = fmx(t.n, 0.0f);
    const float s = friction_scale(t.t0, t.t1, mu * n);
    f = {n, t.t0 * s, t.t1 * s};
    sc = {t.n > 0.0f ? 1.0f : 0.0f, s, s};
}

struct V6 { float v[6]; };
PMB_HD float dot6(const V6& a, const V6& b) {
    float r = 0.0f;
#pragma unroll
    for (int i = 0; i < 6; ++i) r += a.v[i] * b.v[i];
    return r;
}
PMB_HD V6 jac(V3 l, V3 a) { return {{l.x, l.y, l.z, a.x, a.y, a.z}}; }
PMB_HD constexpr unsigned bidx(unsigned r, unsigned c) { return r >= c ? r * (r + 1u) / 2u + c : c * (c + 1u) / 2u + r; }
struct Blk { float h[21]; float g[6]; };

PMB_HD void add_row(Blk& b, const V6& j, float stiffness, float force) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        b.g[i] += j.v[i] * force;
#pragma unroll
        for (int k = 0; k <= i; ++k) b.h[bidx(i, k)] += stiffness * j.v[i] * j.v[k];
    }
}

// LDL^T with one equilibrated retry (constraint_math.slang:165-276).
PMB_HD bool block_solve(const Blk& in, V6& delta) {
    const float eps = 1.1920928955078125e-7f;
    const float pivot_floor = 8.0f * eps;
    const float roundoff = 64.0f * eps;
#pragma unroll
    for (int i = 0; i < 6; ++i) delta.v[i] = 0.0f;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        float d = in.h[bidx(i, i)];
        if (!(d > 0.0f) || !(d < kFltMax) || !(fab(in.g[i]) < kFltMax)) return false;
#pragma unroll
        for (int j = 0; j < i; ++j)
            if (!(fab(in.h[bidx(i, j)]) < kFltMax)) return false;
    }
#pragma unroll 1
    for (int attempt = 0; attempt < 2; ++attempt) {
        Blk b = in;
        float scale[6], dg[6], fw[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            scale[i] = attempt ? rsq(b.h[bidx(i, i)]) : 1.0f;
            dg[i] = 0.0f;
            fw[i] = 0.0f;
        }
        if (attempt) {
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                b.g[i] *= scale[i];
                if (!(fab(b.g[i]) < kFltMax)) return false;
#pragma unroll
                for (int j = 0; j < i; ++j) {
                    b.h[bidx(i, j)] *= scale[i] * scale[j];
                    if (!(fab(b.h[bidx(i, j)]) <= 1.0f + roundoff)) return false;
                }
                b.h[bidx(i, i)] = 1.0f;
            }
        }
        bool retry = false;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            if (!retry) {
#pragma unroll
                for (int j = 0; j < i; ++j) {
                    float sum = b.h[bidx(i, j)];
#pragma unroll
                    for (int k = 0; k < j; ++k) sum -= b.h[bidx(i, k)] * dg[k] * b.h[bidx(j, k)];
                    b.h[bidx(i, j)] = sum / dg[j];
                }
                float diag = b.h[bidx(i, i)];
#pragma unroll
                for (int k = 0; k < i; ++k) diag -= b.h[bidx(i, k)] * b.h[bidx(i, k)] * dg[k];
                if (attempt == 0) {
                    if (!(diag > pivot_floor * in.h[bidx(i, i)]) || !(diag < kFltMax)) retry = true;
                    else dg[i] = diag;
                } else {
                    if (!(diag >= -roundoff) || !(diag < kFltMax)) return false;
                    dg[i] = fmx(diag, pivot_floor);
                }
                if (!retry) {
                    fw[i] = -b.g[i];
#pragma unroll
                    for (int k = 0; k < i; ++k) fw[i] -= b.h[bidx(i, k)] * fw[k];
                }
            }
        }
        if (retry) continue;
#pragma unroll
        for (int i = 5; i >= 0; --i) {
            delta.v[i] = fw[i] / dg[i];
#pragma unroll
            for (int k = i + 1; k < 6; ++k) delta.v[i] -= b.h[bidx(k, i)] * delta.v[k];
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            delta.v[i] *= scale[i];
            if (!(fab(delta.v[i]) < kFltMax)) return false;
        }
        return true;
    }
    return false;
}

struct Row {
    V6 a, b;
    Dual dual;
    float error, velocity, lower, upper, stiffness, damping, beta, reference_force;
};
PMB_HD float row_error(const Row& r, const V6& a, const V6& b) { return r.error + dot6(r.a, a) + dot6(r.b, b); }
PMB_HD float row_trial(const Row& r, const V6& a, const V6& b, float dt) {
    float disp = dot6(r.a, a) + dot6(r.b, b);
    return r.dual.lambda + r.dual.penalty * (r.error + disp) + r.damping * (r.velocity + disp / dt);
}
PMB_HD float row_force(const Row& r, const V6& a, const V6& b, float dt) {
    return fclamp(row_trial(r, a, b, dt), r.lower, r.upper);
}
PMB_HD void row_accumulate(Blk& blk, const Row& r, bool first, const V6& a, const V6& b, float dt) {
    float trial = row_trial(r, a, b, dt);
    bool two_sided = r.lower < 0.0f && r.upper > 0.0f;
    float stiff = two_sided || (trial > r.lower && trial < r.upper) ? r.dual.penalty + r.damping / dt : 0.0f;
    add_row(blk, first ? r.a : r.b, stiff, fclamp(trial, r.lower, r.upper) - r.reference_force);
}
PMB_HD Row row_advance(Row r, const V6& a, const V6& b) {
    r.dual = update_dual(r.dual, row_error(r, a, b), r.beta, r.lower, r.upper, r.stiffness);
    return r;
}

PMB_HD void basis(V3 n, V3& t0, V3& t1) {
    t0 = normalized_or(cross(n, fab(n.x) < 0.57735f ? V3{1, 0, 0} : V3{0, 1, 0}), V3{0, 0, 1});
    t1 = cross(n, t0);
}

}  // namespace pmb

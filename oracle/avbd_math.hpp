// SPDX-License-Identifier: MIT
// ORACLE — test infrastructure only. CPU restatement of the reference's AVBD
// numerical core, used by tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg as the checker. Nothing in the product links this file.
//
// Vector/quaternion helpers follow src/slang/math.slang:6-248 and the block,
// dual and row math follows src/slang/constraint_math.slang:8-345 of the
// reference (tabutyn/parallel-mater). Templated on the scalar so the same
// steps run in FP32 (the reference's arithmetic) and FP64 (error replay).
// Built with -ffp-contract=off: the reference compiles its kernels with
// --fmad=false / -fp-mode precise. rsqrt(x) is evaluated as 1/sqrt(x).
#pragma once
#include <cmath>
#include <cstdint>

namespace oracle {

template <class R> struct V3 { R x{}, y{}, z{}; };
template <class R> struct Q4 { R x{}, y{}, z{}, w{}; };

template <class R> inline R rsq(R v) { return R(1) / std::sqrt(v); }
template <class R> inline R mn(R a, R b) { return a < b ? a : b; }
template <class R> inline R mx(R a, R b) { return a > b ? a : b; }
template <class R> inline R ab(R a) { return a < R(0) ? -a : a; }
template <class R> inline R clampv(R v, R lo, R hi) { return mn(mx(v, lo), hi); }

// math.slang:6-64
template <class R> inline V3<R> add(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> sub(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> mul(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline V3<R> vmin(V3<R> a, V3<R> b) {
    return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)};
}
template <class R> inline V3<R> vmax(V3<R> a, V3<R> b) {
    return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)};
}
template <class R> inline R len2(V3<R> a) { return dot(a, a); }
template <class R> inline R len(V3<R> a) { return std::sqrt(len2(a)); }
template <class R> constexpr R kEps() { return R(1.0e-6); }
template <class R> inline V3<R> normalized_or(V3<R> v, V3<R> fallback) {
    R s = len2(v);
    return s <= kEps<R>() * kEps<R>() ? fallback : mul(v, rsq(s));
}
template <class R> inline R comp(V3<R> v, unsigned axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }
template <class R> inline V3<R> unit_axis(unsigned axis) {
    return axis == 0 ? V3<R>{1, 0, 0} : (axis == 1 ? V3<R>{0, 1, 0} : V3<R>{0, 0, 1});
}

// math.slang:66-135
template <class R> inline Q4<R> conj(Q4<R> q) { return {-q.x, -q.y, -q.z, q.w}; }
template <class R> inline Q4<R> qmul(Q4<R> a, Q4<R> b) {
    return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
            a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
template <class R> inline Q4<R> qnormalize(Q4<R> q) {
    R s = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (s <= kEps<R>() * kEps<R>()) return {};
    R inv = rsq(s);
    return {q.x * inv, q.y * inv, q.z * inv, q.w * inv};
}
template <class R> inline Q4<R> qrelative(Q4<R> from, Q4<R> to, bool local) {
    R c = from.x * to.x + from.y * to.y + from.z * to.z + from.w * to.w;
    if (c < R(0)) to = {-to.x, -to.y, -to.z, -to.w};
    Q4<R> d{to.x - from.x, to.y - from.y, to.z - from.z, to.w - from.w};
    Q4<R> r = local ? qmul(conj(from), d) : qmul(d, conj(from));
    r.w = ab(c);
    return qnormalize(r);
}
template <class R> inline V3<R> rotate(Q4<R> q, V3<R> v) {
    V3<R> u{q.x, q.y, q.z};
    V3<R> t = mul(cross(u, v), R(2));
    return add(v, add(mul(t, q.w), cross(u, t)));
}
template <class R> inline V3<R> inv_rotate(Q4<R> q, V3<R> v) { return rotate(conj(q), v); }
template <class R> inline V3<R> rotation_displacement(Q4<R> from, Q4<R> to, V3<R> v) {
    if (from.x * to.x + from.y * to.y + from.z * to.z + from.w * to.w < R(0))
        to = {-to.x, -to.y, -to.z, -to.w};
    V3<R> o{from.x, from.y, from.z}, n{to.x, to.y, to.z};
    V3<R> d = sub(n, o);
    V3<R> oc = cross(o, v), dc = cross(d, v);
    return mul(add(add(mul(oc, to.w - from.w), mul(dc, to.w)), add(cross(d, oc), cross(n, dc))), R(2));
}
// Arctangent (first quadrant) and x cot(x) on [0, pi/2]. In FP32 they are
// evaluated from basic operations -- the addition formula with pi/6 and the
// Maclaurin series of atan to u^15, and of sin to x^15 and cos to x^16 --
// the same steps as the CUDA library, so both round identically; the libm
// functions would round differently on the host and on the device. The FP64
// replay uses libm (the exact functions to double precision).
template <class R> inline R atan2_q1(R y, R x) {
    if constexpr (sizeof(R) == 8) {
        return std::atan2(y, x);
    } else {
        const bool swap = y > x;
        const float t = swap ? x / y : y / x;
        const bool shift = t > 0.26794919f;  // tan(pi/12)
        const float u = shift ? (t * 1.7320508f - 1.0f) / (t + 1.7320508f) : t;
        const float u2 = u * u;
        const float coef[8] = {1.0f, -1.0f / 3.0f, 1.0f / 5.0f, -1.0f / 7.0f,
                               1.0f / 9.0f, -1.0f / 11.0f, 1.0f / 13.0f, -1.0f / 15.0f};
        float p = coef[7];
        for (int k = 6; k >= 0; --k) p = coef[k] + u2 * p;
        float r = u * p;
        if (shift) r = 0.52359878f + r;  // pi/6
        return swap ? 1.5707964f - r : r;
    }
}
template <class R> inline R x_cot(R x) {
    if constexpr (sizeof(R) == 8) {
        return x * std::cos(x) / std::sin(x);
    } else {
        const float x2 = x * x;
        const float sc[8] = {1.0f, -1.0f / 6.0f, 1.0f / 120.0f, -1.0f / 5040.0f, 1.0f / 362880.0f,
                             -1.0f / 39916800.0f, 1.0f / 6227020800.0f, -1.0f / 1307674368000.0f};
        const float cc[9] = {1.0f, -0.5f, 1.0f / 24.0f, -1.0f / 720.0f, 1.0f / 40320.0f, -1.0f / 3628800.0f,
                             1.0f / 479001600.0f, -1.0f / 87178291200.0f, 1.0f / 20922789888000.0f};
        float s = sc[7];
        for (int k = 6; k >= 0; --k) s = sc[k] + x2 * s;
        float c = cc[8];
        for (int k = 7; k >= 0; --k) c = cc[k] + x2 * c;
        return c / s;
    }
}
// math.slang:221-240
template <class R> inline V3<R> rotation_vector(Q4<R> d) {
    R s = d.x * d.x + d.y * d.y + d.z * d.z;
    R scale = R(2) + s * (R(1) / R(3) + s * (R(3) / R(20) + s * (R(5) / R(56) + s * (R(35) / R(576)))));
    if (s > R(0.01)) {
        R vs = std::sqrt(s);
        scale = R(2) * atan2_q1(vs, clampv(d.w, R(0), R(1))) / vs;
    }
    return {d.x * scale, d.y * scale, d.z * scale};
}
template <class R> inline V3<R> delta_velocity(Q4<R> from, Q4<R> to, R dt) {
    if (dt <= R(0)) return {};
    return mul(rotation_vector(qrelative(from, to, false)), R(1) / dt);
}
template <class R> inline V3<R> clamp_length(V3<R> v, R maximum) {
    R s = len2(v);
    if (s <= maximum * maximum || s <= kEps<R>() * kEps<R>()) return v;
    return mul(v, maximum * rsq(s));
}

// ---------------------------------------------------------------- AVBD core
// constraint_math.slang:8-14
template <class R> struct K {
    static constexpr R alpha = R(0.99);
    static constexpr R gamma = R(0.999);
    static constexpr R kmin = R(1.0);
    static constexpr R kmax = R(1.0e10);
};

template <class R> struct Dual { R lambda{}, penalty{}; };

// constraint_math.slang:30-37
template <class R> inline Dual<R> warm_start(Dual<R> d, R stiffness) {
    d.lambda *= K<R>::alpha * K<R>::gamma;
    d.penalty = mn(stiffness, clampv(d.penalty * K<R>::gamma, K<R>::kmin, K<R>::kmax));
    return d;
}
// constraint_math.slang:39-42
template <class R> inline R dual_force(Dual<R> d, R error, R lo, R hi) {
    return clampv(d.lambda + d.penalty * error, lo, hi);
}
// constraint_math.slang:44-56
template <class R> inline Dual<R> update_dual(Dual<R> d, R error, R beta, R lo, R hi, R stiffness) {
    R u = d.lambda + d.penalty * error;
    d.lambda = stiffness < K<R>::kmax ? R(0) : clampv(u, lo, hi);
    if (u > lo && u < hi) d.penalty = mn(stiffness, mn(K<R>::kmax, d.penalty + beta * ab(error)));
    return d;
}

template <class R> struct Force3 { R n{}, t0{}, t1{}; };
// constraint_math.slang:65-96
template <class R> inline R friction_scale(R t0, R t1, R bound) {
    if (bound <= R(0)) return R(0);
    R s = t0 * t0 + t1 * t1;
    return s <= bound * bound ? R(1) : mn(R(1), bound * rsq(s));
}
template <class R> inline Force3<R> project_contact(Force3<R> f, R friction) {
    f.n = mx(f.n, R(0));
    R bound = friction * f.n;
    R s = friction_scale(f.t0, f.t1, bound);
    f.t0 *= s;
    f.t1 *= s;
    return f;
}
template <class R> inline Force3<R> stiffness_scales(Force3<R> trial, R friction) {
    R n = mx(trial.n, R(0));
    R s = friction_scale(trial.t0, trial.t1, friction * n);
    return {trial.n > R(0) ? R(1) : R(0), s, s};
}

template <class R> struct Vec6 { R v[6]{}; };
template <class R> inline R dot6(const Vec6<R>& a, const Vec6<R>& b) {
    R r = R(0);
    for (unsigned i = 0; i < 6; ++i) r += a.v[i] * b.v[i];
    return r;
}
inline unsigned bidx(unsigned r, unsigned c) {
    unsigned hi = r > c ? r : c, lo = r > c ? c : r;
    return hi * (hi + 1u) / 2u + lo;
}
// Packed symmetric lower triangle (constraint_math.slang:125-132).
template <class R> struct Block { R h[21]{}; R g[6]{}; };

// constraint_math.slang:151-163
template <class R> inline void add_row(Block<R>& b, const Vec6<R>& j, R stiffness, R force) {
    for (unsigned i = 0; i < 6; ++i) {
        b.g[i] += j.v[i] * force;
        for (unsigned k = 0; k <= i; ++k) b.h[bidx(i, k)] += stiffness * j.v[i] * j.v[k];
    }
}

// constraint_math.slang:165-276: LDL^T with one equilibrated retry.
template <class R> inline bool block_solve(const Block<R>& in, Vec6<R>& delta) {
    const R largest = R(3.402823466e38);
    const R eps = R(1.1920928955078125e-7);
    const R pivot_floor = R(8) * eps;
    const R roundoff = R(64) * eps;
    delta = Vec6<R>{};
    for (unsigned i = 0; i < 6; ++i) {
        R d = in.h[bidx(i, i)];
        if (!(d > R(0)) || !(d < largest) || !(ab(in.g[i]) < largest)) return false;
        for (unsigned j = 0; j < i; ++j)
            if (!(ab(in.h[bidx(i, j)]) < largest)) return false;
    }
    for (unsigned attempt = 0; attempt < 2; ++attempt) {
        Block<R> b = in;
        R scale[6], dg[6], fw[6];
        for (unsigned i = 0; i < 6; ++i) {
            scale[i] = attempt ? rsq(b.h[bidx(i, i)]) : R(1);
            dg[i] = R(0);
            fw[i] = R(0);
        }
        if (attempt) {
            for (unsigned i = 0; i < 6; ++i) {
                b.g[i] *= scale[i];
                if (!(ab(b.g[i]) < largest)) return false;
                for (unsigned j = 0; j < i; ++j) {
                    b.h[bidx(i, j)] *= scale[i] * scale[j];
                    if (!(ab(b.h[bidx(i, j)]) <= R(1) + roundoff)) return false;
                }
                b.h[bidx(i, i)] = R(1);
            }
        }
        bool retry = false;
        for (unsigned i = 0; i < 6; ++i) {
            for (unsigned j = 0; j < i; ++j) {
                R sum = b.h[bidx(i, j)];
                for (unsigned k = 0; k < j; ++k) sum -= b.h[bidx(i, k)] * dg[k] * b.h[bidx(j, k)];
                b.h[bidx(i, j)] = sum / dg[j];
            }
            R diag = b.h[bidx(i, i)];
            for (unsigned k = 0; k < i; ++k) diag -= b.h[bidx(i, k)] * b.h[bidx(i, k)] * dg[k];
            if (attempt == 0) {
                if (!(diag > pivot_floor * in.h[bidx(i, i)]) || !(diag < largest)) {
                    retry = true;
                    break;
                }
                dg[i] = diag;
            } else {
                if (!(diag >= -roundoff) || !(diag < largest)) return false;
                dg[i] = mx(diag, pivot_floor);
            }
            fw[i] = -b.g[i];
            for (unsigned k = 0; k < i; ++k) fw[i] -= b.h[bidx(i, k)] * fw[k];
        }
        if (retry) continue;
        for (int i = 5; i >= 0; --i) {
            delta.v[i] = fw[i] / dg[i];
            for (unsigned k = unsigned(i) + 1; k < 6; ++k) delta.v[i] -= b.h[bidx(k, unsigned(i))] * delta.v[k];
        }
        for (unsigned i = 0; i < 6; ++i) {
            delta.v[i] *= scale[i];
            if (!(ab(delta.v[i]) < largest)) return false;
        }
        return true;
    }
    return false;
}

// constraint_math.slang:278-345
template <class R> struct Row {
    Vec6<R> a, b;
    Dual<R> dual;
    R error{}, velocity{}, lower{}, upper{}, stiffness{}, damping{}, beta{}, reference_force{};
};
template <class R> inline R row_error(const Row<R>& r, const Vec6<R>& a, const Vec6<R>& b) {
    return r.error + dot6(r.a, a) + dot6(r.b, b);
}
template <class R> inline R row_trial(const Row<R>& r, const Vec6<R>& a, const Vec6<R>& b, R dt) {
    R disp = dot6(r.a, a) + dot6(r.b, b);
    return r.dual.lambda + r.dual.penalty * (r.error + disp) + r.damping * (r.velocity + disp / dt);
}
template <class R> inline R row_force(const Row<R>& r, const Vec6<R>& a, const Vec6<R>& b, R dt) {
    return clampv(row_trial(r, a, b, dt), r.lower, r.upper);
}
template <class R> inline void row_accumulate(Block<R>& blk, const Row<R>& r, bool first, const Vec6<R>& a,
                                              const Vec6<R>& b, R dt) {
    R trial = row_trial(r, a, b, dt);
    bool two_sided = r.lower < R(0) && r.upper > R(0);
    R stiff = two_sided || (trial > r.lower && trial < r.upper) ? r.dual.penalty + r.damping / dt : R(0);
    add_row(blk, first ? r.a : r.b, stiff, clampv(trial, r.lower, r.upper) - r.reference_force);
}
template <class R> inline Row<R> row_advance(Row<R> r, const Vec6<R>& a, const Vec6<R>& b) {
    r.dual = update_dual(r.dual, row_error(r, a, b), r.beta, r.lower, r.upper, r.stiffness);
    return r;
}

}  // namespace oracle

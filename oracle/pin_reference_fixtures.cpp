// SPDX-License-Identifier: MIT
// ORACLE PIN — test infrastructure only. Runs the reference's own AVBD
// numerical fixtures (tests/solver/geometry_constraint_cases.hpp, validated by
// its own avbd_cases::validate) with every AVBD math call routed to the
// oracle's restatement instead of the reference's C++ mirror.
//
// Mechanism: the mirror header (tests/solver/reference/geometry_constraints.hpp)
// is included first with its function names macro-renamed, so its
// `#pragma once` is consumed; shims with the original names then forward to
// oracle:: functions, and the fixture header binds to the shims. Half-space
// projection fixtures (scalar cases 56-75) exercise the reference's triangle
// correction code (reference/halfspace.hpp), which is not part of the convex
// face-contact path restated here; they run unmodified and are reported apart.
//
// Built by oracle/Makefile target `pin` into oracle/_ref/ from the sources
// where they lie under the reference checkout (REF=... on the make line).
#define warm_start ref_warm_start
#define force ref_force
#define update_dual ref_update_dual
#define project_contact ref_project_contact
#define contact_stiffness_scales ref_contact_stiffness_scales
#define add_row ref_add_row
#define solve ref_solve
#define row_error ref_row_error
#define row_trial ref_row_trial
#define row_force ref_row_force
#define accumulate ref_accumulate
#define advance ref_advance
#include "reference/geometry_constraints.hpp"
#undef warm_start
#undef force
#undef update_dual
#undef project_contact
#undef contact_stiffness_scales
#undef add_row
#undef solve
#undef row_error
#undef row_trial
#undef row_force
#undef accumulate
#undef advance

#include <cstdio>

#include "avbd_math.hpp"

namespace parallel_mater {
namespace avbd {

inline oracle::Block<float> to_o(const Block& b) {
    oracle::Block<float> o{};
    for (int i = 0; i < 21; ++i) o.h[i] = b.h.values[i];
    for (int i = 0; i < 6; ++i) o.g[i] = b.g[i];
    return o;
}
inline void from_o(const oracle::Block<float>& o, Block& b) {
    for (int i = 0; i < 21; ++i) b.h.values[i] = o.h[i];
    for (int i = 0; i < 6; ++i) b.g[i] = o.g[i];
}
inline oracle::Vec6<float> to_o(const Vector6& v) {
    oracle::Vec6<float> o{};
    for (int i = 0; i < 6; ++i) o.v[i] = v.v[i];
    return o;
}
inline oracle::Row<float> to_o(const Row& r) {
    oracle::Row<float> o{};
    o.a = to_o(r.a);
    o.b = to_o(r.b);
    o.dual = {r.dual.lambda, r.dual.penalty};
    o.error = r.error;
    o.velocity = r.velocity;
    o.lower = r.lower;
    o.upper = r.upper;
    o.stiffness = r.stiffness;
    o.damping = r.damping;
    o.beta = r.beta;
    o.reference_force = r.reference_force;
    return o;
}
inline Row from_o(const oracle::Row<float>& o, Row r) {
    r.dual = {o.dual.lambda, o.dual.penalty};
    return r;
}

inline Dual warm_start(Dual v, float stiffness = maximum_penalty) {
    auto d = oracle::warm_start(oracle::Dual<float>{v.lambda, v.penalty}, stiffness);
    return {d.lambda, d.penalty};
}
inline float force(Dual v, float error, float lower = -maximum_penalty, float upper = maximum_penalty) {
    return oracle::dual_force(oracle::Dual<float>{v.lambda, v.penalty}, error, lower, upper);
}
inline Dual update_dual(Dual v, float error, float beta, float lower = -maximum_penalty,
                        float upper = maximum_penalty, float stiffness = maximum_penalty) {
    auto d = oracle::update_dual(oracle::Dual<float>{v.lambda, v.penalty}, error, beta, lower, upper, stiffness);
    return {d.lambda, d.penalty};
}
inline ContactForce project_contact(ContactForce v, float friction) {
    auto f = oracle::project_contact(oracle::Force3<float>{v.normal, v.tangent0, v.tangent1}, friction);
    return {f.n, f.t0, f.t1};
}
inline ContactForce contact_stiffness_scales(ContactForce v, float friction) {
    auto f = oracle::stiffness_scales(oracle::Force3<float>{v.normal, v.tangent0, v.tangent1}, friction);
    return {f.n, f.t0, f.t1};
}
inline void add_row(Block& b, Vector6 j, float stiffness, float row_force_value) {
    auto o = to_o(b);
    oracle::add_row(o, to_o(j), stiffness, row_force_value);
    from_o(o, b);
}
inline bool solve(Block in, Vector6& delta) {
    oracle::Vec6<float> d{};
    bool ok = oracle::block_solve(to_o(in), d);
    for (int i = 0; i < 6; ++i) delta.v[i] = d.v[i];
    return ok;
}
inline float row_error(Row r, Vector6 a, Vector6 b) { return oracle::row_error(to_o(r), to_o(a), to_o(b)); }
inline float row_trial(Row r, Vector6 a, Vector6 b, float dt) {
    return oracle::row_trial(to_o(r), to_o(a), to_o(b), dt);
}
inline float row_force(Row r, Vector6 a, Vector6 b, float dt) {
    return oracle::row_force(to_o(r), to_o(a), to_o(b), dt);
}
inline void accumulate(Block& blk, Row r, bool first, Vector6 a, Vector6 b, float dt) {
    auto o = to_o(blk);
    oracle::row_accumulate(o, to_o(r), first, to_o(a), to_o(b), dt);
    from_o(o, blk);
}
inline Row advance(Row r, Vector6 a, Vector6 b) { return from_o(oracle::row_advance(to_o(r), to_o(a), to_o(b)), r); }

}  // namespace avbd
}  // namespace parallel_mater

#include "geometry_constraint_cases.hpp"

int main() {
    unsigned on_path = 0, on_path_passed = 0, other = 0, other_passed = 0;
    for (unsigned index = 0; index < avbd_cases::count; ++index) {
        const auto result = avbd_cases::evaluate(index);
        const bool ok = avbd_cases::validate(index, result);
        const unsigned scalar = index >= avbd_cases::block_count ? index - avbd_cases::block_count : 0u;
        const bool halfspace = index >= avbd_cases::block_count && scalar >= 56;
        if (halfspace) {
            ++other;
            other_passed += ok;
        } else {
            ++on_path;
            on_path_passed += ok;
        }
        std::printf("%s %3u %s %s\n", ok ? "PASS" : "FAIL", index, halfspace ? "halfspace" : "oracle",
                    avbd_cases::name(index));
    }
    std::printf("oracle fixtures: %u/%u passed; half-space fixtures (reference code): %u/%u passed\n",
                on_path_passed, on_path, other_passed, other);
    return on_path_passed == on_path ? 0 : 1;
}

// SPDX-License-Identifier: MIT
// Golden-vector generator (run by tests/golden/make_golden.py in a checkout
// that has the reference). Inputs come from the reference's own block
// fixtures (tests/solver/geometry_constraint_cases.hpp make_block) plus
// seeded random and edge-case inputs; every output is computed by the
// reference's C++ mirror of constraint_math.slang
// (tests/solver/reference/geometry_constraints.hpp). Writes JSON to stdout.
#include <cinttypes>
#include <cmath>
#include <cstdint>
#include <cstdio>

#include "geometry_constraint_cases.hpp"

using namespace parallel_mater::avbd;

static uint64_t rng_state = 0x9E3779B97F4A7C15ull;
static uint64_t next_u64() {
    uint64_t z = (rng_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static float uni(float lo, float hi) { return lo + (hi - lo) * float(double(next_u64() >> 11) * 0x1.0p-53); }
static float logu(float lo, float hi) { return std::exp(uni(std::log(lo), std::log(hi))); }

static void pf(float v) {
    if (std::isnan(v)) std::printf("\"nan\"");
    else if (std::isinf(v)) std::printf(v > 0 ? "\"inf\"" : "\"-inf\"");
    else std::printf("%.9g", double(v));
}
static void arr(const float* v, int n) {
    std::printf("[");
    for (int i = 0; i < n; ++i) { if (i) std::printf(","); pf(v[i]); }
    std::printf("]");
}

static void block_entry(const Block& b, bool first) {
    Vector6 d{};
    bool ok = solve(b, d);
    std::printf("%s{\"h\":", first ? "" : ",\n");
    arr(b.h.values, 21);
    std::printf(",\"g\":");
    arr(b.g, 6);
    std::printf(",\"solved\":%d,\"delta\":", ok ? 1 : 0);
    arr(d.v, 6);
    std::printf("}");
}

int main() {
    std::printf("{\"source\":\"reference tests/solver/reference/geometry_constraints.hpp\",\n\"blocks\":[\n");
    bool first = true;
    for (unsigned i = 0; i < avbd_cases::block_count; ++i) { block_entry(avbd_cases::make_block(i), first); first = false; }
    // Seeded contact-like blocks: body inertia plus 1-24 contact rows.
    for (int c = 0; c < 200; ++c) {
        Block b{};
        float m = logu(0.1f, 1e4f) / (1.f / 3600.f);
        float I = m * logu(0.01f, 1.f);
        for (unsigned i = 0; i < 6; ++i) b.h[i][i] = i < 3 ? m : I * uni(0.5f, 2.f);
        int rows = 1 + int(next_u64() % 24);
        for (int r = 0; r < rows; ++r) {
            Vector6 j{};
            for (int k = 0; k < 3; ++k) j.v[k] = uni(-1.f, 1.f);
            for (int k = 3; k < 6; ++k) j.v[k] = uni(-0.8f, 0.8f);
            float k = logu(1.f, c % 5 == 0 ? 1e10f : 1e8f);
            add_row(b, j, (next_u64() & 3) ? k : 0.f, uni(-1e5f, 1e5f));
        }
        for (unsigned i = 0; i < 6; ++i) b.g[i] += uni(-1e3f, 1e3f);
        block_entry(b, false);
    }
    std::printf("\n],\n\"duals\":[\n");
    for (int c = 0; c < 400; ++c) {
        float lam = uni(-50.f, 50.f), pen = logu(0.01f, 2e10f), err = uni(-0.5f, 0.5f), beta = logu(1.f, 1e8f);
        float lo = (c % 3 == 0) ? 0.f : -maximum_penalty, hi = (c % 7 == 0) ? uni(0.f, 20.f) : maximum_penalty;
        if (c % 11 == 0) lo = -hi;
        float stiff = (c % 4 == 0) ? logu(0.1f, 1e6f) : maximum_penalty;
        Dual d{lam, pen};
        Dual w = warm_start(d, stiff), u = update_dual(d, err, beta, lo, hi, stiff);
        float f = force(d, err, lo, hi);
        float in[7] = {lam, pen, err, beta, lo, hi, stiff}, out[5] = {w.lambda, w.penalty, f, u.lambda, u.penalty};
        std::printf("%s{\"in\":", c ? ",\n" : "");
        arr(in, 7);
        std::printf(",\"out\":");
        arr(out, 5);
        std::printf("}");
    }
    std::printf("\n],\n\"contacts\":[\n");
    for (int c = 0; c < 400; ++c) {
        float t[3] = {uni(-10.f, 40.f), uni(-30.f, 30.f), uni(-30.f, 30.f)};
        if (c % 13 == 0) t[1] = t[2] = 0.f;
        float mu = (c % 9 == 0) ? 0.f : uni(0.f, 1.2f);
        ContactForce in{t[0], t[1], t[2]};
        ContactForce p = project_contact(in, mu), s = contact_stiffness_scales(in, mu);
        float iv[4] = {t[0], t[1], t[2], mu}, out[6] = {p.normal, p.tangent0, p.tangent1, s.normal, s.tangent0, s.tangent1};
        std::printf("%s{\"in\":", c ? ",\n" : "");
        arr(iv, 4);
        std::printf(",\"out\":");
        arr(out, 6);
        std::printf("}");
    }
    std::printf("\n],\n\"rows\":[\n");
    for (int c = 0; c < 400; ++c) {
        float v[42] = {};
        for (int k = 0; k < 12; ++k) v[k] = uni(-1.f, 1.f);
        v[12] = uni(-100.f, 100.f);
        v[13] = logu(1.f, 1e9f);
        v[14] = uni(-0.2f, 0.2f);
        v[15] = uni(-2.f, 2.f);
        v[16] = (c % 3 == 0) ? 0.f : -maximum_penalty;
        v[17] = (c % 5 == 0) ? uni(0.f, 50.f) : maximum_penalty;
        if (c % 10 == 0) v[16] = -v[17];
        v[18] = (c % 4 == 0) ? logu(1.f, 1e5f) : maximum_penalty;
        v[19] = (c % 6 == 0) ? uni(0.f, 50.f) : 0.f;
        v[20] = logu(1.f, 1e6f);
        v[21] = (c % 8 == 0) ? uni(-20.f, 20.f) : 0.f;
        for (int k = 22; k < 34; ++k) v[k] = uni(-0.05f, 0.05f);
        v[34] = 1.f / 60.f;
        for (int k = 35; k < 41; ++k) v[k] = logu(1.f, 1e6f);
        v[41] = float(c & 1);
        Row row{};
        for (int k = 0; k < 6; ++k) { row.a.v[k] = v[k]; row.b.v[k] = v[6 + k]; }
        row.dual = {v[12], v[13]};
        row.error = v[14]; row.velocity = v[15]; row.lower = v[16]; row.upper = v[17];
        row.stiffness = v[18]; row.damping = v[19]; row.beta = v[20]; row.reference_force = v[21];
        Vector6 a{}, b{};
        for (int k = 0; k < 6; ++k) { a.v[k] = v[22 + k]; b.v[k] = v[28 + k]; }
        Block blk{};
        for (int k = 0; k < 6; ++k) blk.h[k][k] = v[35 + k];
        accumulate(blk, row, v[41] != 0.f, a, b, v[34]);
        Row adv = advance(row, a, b);
        float gs = 0, ds = 0;
        for (int k = 0; k < 6; ++k) { gs += blk.g[k]; ds += blk.h[k][k]; }
        float out[7] = {row_error(row, a, b), row_trial(row, a, b, v[34]), row_force(row, a, b, v[34]),
                        adv.dual.lambda, adv.dual.penalty, gs, ds};
        std::printf("%s{\"in\":", c ? ",\n" : "");
        arr(v, 42);
        std::printf(",\"out\":");
        arr(out, 7);
        std::printf("}");
    }
    std::printf("\n]}\n");
    return 0;
}

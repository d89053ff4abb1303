// SPDX-License-Identifier: MIT
// ORACLE PIN — test infrastructure only. The oracle's broadphase pair
// predicate (oracle::broadphase_boxes, the candidate pairs of its tick) on the
// reference's own spatial fixtures, with the reference's spatial headers
// compiled from the checkout (src/simulation/rigid_spatial.hpp and the
// spatial_service.hpp / spatial_build.hpp it includes):
//
// 1. The shared-query scenario of tests/solver/rigid_spatial_tests.cpp:180-290:
//    ten bodies whose bounds come from the reference's own
//    rigid_spatial_proxy_envelope (a fast sweep, a rotation about an offset
//    centre, two margins that just reach, a collision-disabled pair, a fixed
//    group). Expected: the reference's spatial_query_aabb over a median-split
//    tree of the same leaves, filtered by the scenario's pair rules (dynamic
//    query, identity order, fixed root, disabled owners), and the scenario's
//    named facts (0-1, 2-3, 4-5 in; 6-7, 8-9 out).
// 2. The leaves of tests/solver/spatial_build_primitives_tests.cpp:245-339:
//    257 seeded 0.2 m boxes (mt19937 0xF806, every third inactive, three
//    coincident), 128 seeded 2 m query boxes, the inclusive touching pair and
//    the 30,065-leaf lattice tier. Expected: every active leaf overlapping the
//    query, inclusively (the fixture's brute force). The oracle answers a
//    query by taking the query box as the only dynamic box; the same leaves
//    also run as dynamic bodies against a sort-and-sweep brute force.
//
// Built by oracle/Makefile target `pin` into oracle/_ref/ (REF=... on the
// make line); run by tests/test_oracle_cpu.py.
#include "simulation/rigid_spatial.hpp"

#include <algorithm>
#include <array>
#include <cstdio>
#include <limits>
#include <random>
#include <set>
#include <utility>
#include <vector>

#include "avbd_step.hpp"

namespace {
namespace sim = parallel_mater::simulation;
using V = oracle::V3<float>;

int failures = 0;
#define PIN_CHECK(cond)                                                              \
    do {                                                                             \
        if (!(cond)) {                                                               \
            std::printf("%s:%d pin check failed: %s\n", __FILE__, __LINE__, #cond); \
            ++failures;                                                              \
        }                                                                            \
    } while (false)

sim::SpatialAabb make_box(float x0, float y0, float z0, float x1, float y1, float z1) {
    sim::SpatialAabb b{};
    b.minimum[0] = x0, b.minimum[1] = y0, b.minimum[2] = z0;
    b.maximum[0] = x1, b.maximum[1] = y1, b.maximum[2] = z1;
    return b;
}
V lo_of(const sim::SpatialAabb& b) { return {b.minimum[0], b.minimum[1], b.minimum[2]}; }
V hi_of(const sim::SpatialAabb& b) { return {b.maximum[0], b.maximum[1], b.maximum[2]}; }

std::set<uint64_t> oracle_pairs(const std::vector<sim::SpatialAabb>& boxes, const std::vector<uint8_t>& dyn,
                                const std::vector<uint32_t>& group, const std::vector<uint64_t>& disabled) {
    std::vector<V> lo, hi;
    for (const auto& b : boxes) lo.push_back(lo_of(b)), hi.push_back(hi_of(b));
    const auto codes = oracle::broadphase_boxes<float>(uint32_t(boxes.size()), lo.data(), hi.data(), dyn.data(),
                                                       group, disabled);
    PIN_CHECK(std::is_sorted(codes.begin(), codes.end()));
    return std::set<uint64_t>(codes.begin(), codes.end());
}

// ---- 1. the shared-query scenario
void shared_queries() {
    const float zero[3]{};
    const uint32_t n = 10;
    std::vector<sim::SpatialAabb> b(n);
    std::vector<uint8_t> dyn(n, 0);
    std::vector<uint32_t> fixed_root(n, std::numeric_limits<uint32_t>::max());
    const float fast_start[3]{-5.0f, 0.0f, 0.0f}, fast_end[3]{5.0f, 0.0f, 0.0f};
    PIN_CHECK(sim::rigid_spatial_proxy_envelope(fast_start, fast_end, zero, 0.2f, 0.0f, zero, zero, 1.0e-5f, b[0]) ==
              PM_SUCCESS);
    dyn[0] = 1;
    b[1] = make_box(-0.2f, -0.2f, -0.2f, 0.2f, 0.2f, 0.2f);
    const float rotation_center[3]{2.0f, 0.0f, 0.0f};
    PIN_CHECK(sim::rigid_spatial_proxy_envelope(zero, zero, rotation_center, 0.1f, 0.0f, zero, zero, 1.0e-5f, b[2]) ==
              PM_SUCCESS);
    dyn[2] = 1;
    b[3] = make_box(-0.1f, 1.9f, -0.1f, 0.1f, 2.1f, 0.1f);
    const float margin_a[3]{10.0f, 0.0f, 0.0f}, margin_b[3]{10.6f, 0.0f, 0.0f};
    PIN_CHECK(sim::rigid_spatial_proxy_envelope(margin_a, margin_a, zero, 0.2f, 0.11f, zero, zero, 1.0e-5f, b[4]) ==
              PM_SUCCESS);
    PIN_CHECK(sim::rigid_spatial_proxy_envelope(margin_b, margin_b, zero, 0.2f, 0.11f, zero, zero, 1.0e-5f, b[5]) ==
              PM_SUCCESS);
    dyn[4] = 1;
    b[6] = b[7] = make_box(20, 0, 0, 21, 1, 1);
    dyn[6] = 1;
    b[8] = b[9] = make_box(30, 0, 0, 31, 1, 1);
    dyn[8] = 1;
    fixed_root[8] = fixed_root[9] = 55;
    const std::pair<uint32_t, uint32_t> disabled_pair{6, 7};

    // The reference's tree query over a median split of the leaves, then the
    // scenario's pair rules; identities increase with the index, as there.
    std::vector<sim::SpatialLeafMetadata> meta(n);
    std::vector<uint8_t> admitted(n, 1);
    for (uint32_t i = 0; i < n; ++i) {
        meta[i].identity = {sim::rigid_spatial_family, 100 + i, 7 + i, 1, sim::rigid_spatial_body_primitive, 20 + i,
                            30 + i};
        meta[i].sort_key = i + 1;
        meta[i].payload_ref = i;
        meta[i].query_mask = sim::rigid_spatial_query_mask;
        meta[i].admission_mask = sim::rigid_spatial_query_mask;
        meta[i].flags = sim::spatial_leaf_retained;
    }
    std::vector<uint32_t> left(n - 1), right(n - 1), sources(n);
    std::vector<sim::SpatialAabb> nodes(2 * n - 1);
    uint32_t next_internal = 0;
    auto build = [&](auto&& self, uint32_t begin, uint32_t end) -> uint32_t {
        if (end - begin == 1) {
            sources[begin] = begin;
            nodes[n - 1 + begin] = b[begin];
            return n - 1 + begin;
        }
        const uint32_t node = next_internal++;
        const uint32_t middle = begin + (end - begin) / 2;
        left[node] = self(self, begin, middle);
        right[node] = self(self, middle, end);
        nodes[node] = sim::spatial_union(nodes[left[node]], nodes[right[node]]);
        return node;
    };
    PIN_CHECK(build(build, 0, n) == 0);
    sim::SpatialTreeView tree{left, right, sources, nodes, meta, admitted, n};
    std::array<uint32_t, 64> traversal{};
    std::vector<uint32_t> candidates(n);
    std::set<uint64_t> expected;
    for (uint32_t q = 0; q < n; ++q) {
        if (!dyn[q]) continue;
        uint32_t written = 0, visited = 0;
        PIN_CHECK(sim::spatial_query_aabb(tree, b[q], sim::rigid_spatial_query_mask, meta[q].sort_key, traversal,
                                          candidates, written, visited) == PM_SUCCESS);
        for (uint32_t k = 0; k < written; ++k) {
            const uint32_t t = meta[candidates[k]].payload_ref;
            if (dyn[t] && !(meta[q].identity < meta[t].identity)) continue;
            if (fixed_root[q] != std::numeric_limits<uint32_t>::max() && fixed_root[q] == fixed_root[t]) continue;
            if (std::min(q, t) == disabled_pair.first && std::max(q, t) == disabled_pair.second) continue;
            expected.insert(uint64_t(q) * n + t);
        }
    }
    std::vector<uint32_t> group(n);
    for (uint32_t i = 0; i < n; ++i) group[i] = fixed_root[i] != std::numeric_limits<uint32_t>::max() ? n + fixed_root[i] : i;
    const std::vector<uint64_t> disabled{uint64_t(6) << 32 | 7};
    const auto actual = oracle_pairs(b, dyn, group, disabled);
    PIN_CHECK(actual == expected);
    PIN_CHECK(actual.count(0 * n + 1) && actual.count(2 * n + 3) && actual.count(4 * n + 5));
    PIN_CHECK(!actual.count(6 * n + 7) && !actual.count(8 * n + 9));
    std::printf("shared-query scenario: %zu pairs, reference query %zu\n", actual.size(), expected.size());
}

// ---- 2. the primitives fixture's leaves and queries
std::set<uint64_t> brute_pairs(const std::vector<sim::SpatialAabb>& b, const std::vector<uint8_t>& dyn) {
    // sort-and-sweep on x, inclusive overlap, a dynamic and (b static or a < b)
    const uint32_t n = uint32_t(b.size());
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return b[x].minimum[0] < b[y].minimum[0]; });
    std::set<uint64_t> out;
    for (uint32_t k = 0; k < n; ++k)
        for (uint32_t m = k + 1; m < n && b[order[m]].minimum[0] <= b[order[k]].maximum[0]; ++m) {
            const uint32_t p = order[k], q = order[m];
            if (!sim::spatial_overlaps(b[p], b[q])) continue;
            for (auto [a, c] : {std::pair{p, q}, std::pair{q, p}})
                if (dyn[a] && (!dyn[c] || a < c)) out.insert(uint64_t(a) * n + c);
        }
    return out;
}

void primitives_leaves() {
    std::mt19937 random(0xF806U);
    std::uniform_real_distribution<float> coordinate(-10.0f, 10.0f);
    constexpr uint32_t capacity = 257;
    std::vector<sim::SpatialAabb> input(capacity);
    std::vector<uint8_t> active(capacity);
    for (uint32_t i = 0; i < capacity; ++i) {
        const float x = coordinate(random), y = coordinate(random), z = coordinate(random);
        input[i] = make_box(x, y, z, x + 0.2f, y + 0.2f, z + 0.2f);
        active[i] = i % 3 != 0;
    }
    input[7] = input[8] = input[11] = make_box(1, 2, 3, 1, 2, 3);
    active[7] = active[8] = active[11] = 1;
    std::vector<uint32_t> sources;
    for (uint32_t i = 0; i < capacity; ++i)
        if (active[i]) sources.push_back(i);
    // Queries: the query box is box 0 and the only dynamic one.
    uint32_t checked = 0;
    for (unsigned sample = 0; sample < 128; ++sample) {
        const float x = coordinate(random), y = coordinate(random), z = coordinate(random);
        const sim::SpatialAabb query = make_box(x, y, z, x + 2, y + 2, z + 2);
        std::vector<sim::SpatialAabb> boxes{query};
        for (uint32_t s : sources) boxes.push_back(input[s]);
        std::vector<uint8_t> dyn(boxes.size(), 0);
        dyn[0] = 1;
        std::vector<uint32_t> group;
        const auto got = oracle_pairs(boxes, dyn, group, {});
        std::set<uint64_t> expected;
        for (uint32_t k = 0; k < sources.size(); ++k)
            if (sim::spatial_overlaps(input[sources[k]], query)) expected.insert(k + 1);
        PIN_CHECK(got == expected);
        checked += uint32_t(expected.size());
    }
    // The same active leaves as dynamic bodies (grid path, coincident leaves).
    {
        std::vector<sim::SpatialAabb> boxes;
        for (uint32_t s : sources) boxes.push_back(input[s]);
        std::vector<uint8_t> dyn(boxes.size(), 1);
        PIN_CHECK(oracle_pairs(boxes, dyn, {}, {}) == brute_pairs(boxes, dyn));
    }
    // Inclusive overlap keeps touching boxes.
    {
        std::vector<sim::SpatialAabb> boxes{make_box(1, 0, 0, 1, 1, 1), make_box(0, 0, 0, 1, 1, 1),
                                            make_box(1, 0, 0, 2, 1, 1)};
        std::vector<uint8_t> dyn{1, 0, 0};
        PIN_CHECK((oracle_pairs(boxes, dyn, {}, {}) == std::set<uint64_t>{1, 2}));
    }
    // The 30,065-leaf lattice tier: coincident copies overlap, neighbours do not.
    {
        constexpr uint32_t count = 30065;
        std::vector<sim::SpatialAabb> boxes(count);
        for (uint32_t i = 0; i < count; ++i) {
            const float x = float(i % 17u) * 0.25f, y = float((i / 17u) % 19u) * 0.2f,
                        z = float((i / (17u * 19u)) % 23u) * 0.15f;
            boxes[i] = make_box(x, y, z, x + 0.1f, y + 0.1f, z + 0.1f);
        }
        std::vector<uint8_t> dyn(count, 1);
        const auto got = oracle_pairs(boxes, dyn, {}, {});
        PIN_CHECK(got == brute_pairs(boxes, dyn));
        std::printf("lattice tier: %zu pairs\n", got.size());
    }
    std::printf("primitives leaves: 128 queries (%u hits) and the leaf sets match\n", checked);
}
}  // namespace

int main() {
    shared_queries();
    primitives_leaves();
    std::printf("spatial pins: %s\n", failures == 0 ? "passed" : "FAILED");
    return failures == 0 ? 0 : 1;
}

// SPDX-License-Identifier: MIT
// Host mesh preparation (see pmb_mesh.cpp).
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace pmb {

struct BvhNodeHost {
    float lo[3], hi[3];
    uint32_t first, count, left, right;  // count != 0: a leaf of triangles [first, first + count)
};

struct PreparedMesh {
    std::vector<uint32_t> indices;                // triangles in BVH leaf order
    std::vector<std::array<float, 4>> planes;     // outward (n, d) per triangle when convex
    std::vector<BvhNodeHost> bvh;                 // build (pre-)order, root first
    std::vector<std::array<float, 3>> shell;      // certified outward normal per triangle, or empty
    bool convex{};
    std::array<float, 3> lo{}, hi{}, center{};
    float radius{};
};

PreparedMesh prepare_mesh(const float* verts, uint32_t nv, const uint32_t* idx, uint32_t ni);

}  // namespace pmb

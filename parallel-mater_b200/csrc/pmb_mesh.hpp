// SPDX-License-Identifier: MIT
// Host mesh preparation (see pmb_mesh.cpp).
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace pmb {

struct PreparedMesh {
    std::vector<uint32_t> indices;                // triangles in BVH leaf order
    std::vector<std::array<float, 4>> planes;     // outward (n, d) per triangle when convex
    bool convex{};
    std::array<float, 3> lo{}, hi{}, center{};
    float radius{};
};

PreparedMesh prepare_mesh(const float* verts, uint32_t nv, const uint32_t* idx, uint32_t ni);

}  // namespace pmb

// SPDX-License-Identifier: MIT
// Host mesh preparation for rigid triangle meshes, as the reference does at
// upload (src/simulation/runtime_deformables.cu.inc:103-270): a median-split
// BVH (<= 4 triangles per leaf, split axis = longest extent, stable sort of
// triangle centroids) whose leaf order becomes the stored triangle order; the
// closed-convex-plane certificate of runtime_domains.cu.inc:1061-1108 (weld
// exact duplicate positions, every welded edge used twice, one outward plane
// per triangle, every vertex within tolerance behind it); AABB and bounding
// sphere about the AABB centre. Compiled with -ffp-contract=off so the plane
// arithmetic is the reference's FP32 sequence.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <functional>
#include <map>
#include <numeric>
#include <vector>

#include "pmb_mesh.hpp"

namespace pmb {
namespace {

struct F3 { float x, y, z; };
F3 add(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
F3 mul(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
F3 cross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float len(F3 a) { return std::sqrt(dot(a, a)); }
F3 normalized_or(F3 v, F3 fb) {
    float s = dot(v, v);
    return s <= 1.0e-6f * 1.0e-6f ? fb : mul(v, 1.0f / std::sqrt(s));
}
float comp(F3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

bool convex_planes(const std::vector<F3>& v, const std::vector<uint32_t>& idx, std::vector<std::array<float, 4>>& out) {
    out.clear();
    std::map<std::array<float, 3>, uint32_t> weld;
    std::vector<uint32_t> remap(v.size());
    F3 center{0, 0, 0};
    for (uint32_t i = 0; i < v.size(); ++i) {
        auto e = weld.emplace(std::array<float, 3>{v[i].x, v[i].y, v[i].z}, uint32_t(weld.size()));
        remap[i] = e.first->second;
        if (e.second) center = add(center, v[i]);
    }
    if (weld.size() < 4) return false;
    center = mul(center, 1.0f / float(weld.size()));
    std::map<uint64_t, uint32_t> edges;
    for (size_t t = 0; t < idx.size(); t += 3)
        for (size_t e = 0; e < 3; ++e) {
            uint64_t a = remap[idx[t + e]], b = remap[idx[t + (e + 1) % 3]];
            ++edges[(std::min(a, b) << 32) | std::max(a, b)];
        }
    for (auto& e : edges)
        if (e.second != 2) return false;
    float scale = 0;
    for (auto& p : v) scale = std::max(scale, len(sub(p, center)));
    const float tol = std::max(1.0e-7f, scale * 1.0e-5f);
    for (size_t t = 0; t < idx.size(); t += 3) {
        F3 a = v[idx[t]];
        F3 n = normalized_or(cross(sub(v[idx[t + 1]], a), sub(v[idx[t + 2]], a)), F3{0, 0, 0});
        float side = dot(n, sub(a, center));
        if (std::fabs(side) <= tol) { out.clear(); return false; }
        if (side < 0.0f) n = mul(n, -1.0f);
        float d = dot(n, a);
        for (auto& p : v)
            if (dot(n, p) - d > tol) { out.clear(); return false; }
        out.push_back({n.x, n.y, n.z, d});
    }
    return true;
}

}  // namespace

PreparedMesh prepare_mesh(const float* verts, uint32_t nv, const uint32_t* idx, uint32_t ni) {
    PreparedMesh m;
    std::vector<F3> v(nv);
    for (uint32_t i = 0; i < nv; ++i) v[i] = {verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]};
    F3 lo = v[0], hi = v[0];
    for (uint32_t i = 1; i < nv; ++i) {
        lo = {std::fmin(lo.x, v[i].x), std::fmin(lo.y, v[i].y), std::fmin(lo.z, v[i].z)};
        hi = {std::fmax(hi.x, v[i].x), std::fmax(hi.y, v[i].y), std::fmax(hi.z, v[i].z)};
    }
    const uint32_t nt = ni / 3;
    std::vector<uint32_t> order(nt);
    std::iota(order.begin(), order.end(), 0u);
    auto centroid = [&](uint32_t t) {
        return mul(add(add(v[idx[3 * t]], v[idx[3 * t + 1]]), v[idx[3 * t + 2]]), 1.0f / 3.0f);
    };
    std::function<void(uint32_t, uint32_t)> build = [&](uint32_t b, uint32_t e) {
        F3 nlo{3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
        F3 nhi = mul(nlo, -1.0f);
        for (uint32_t i = b; i < e; ++i)
            for (uint32_t c = 0; c < 3; ++c) {
                F3 p = v[idx[3 * order[i] + c]];
                nlo = {std::fmin(nlo.x, p.x), std::fmin(nlo.y, p.y), std::fmin(nlo.z, p.z)};
                nhi = {std::fmax(nhi.x, p.x), std::fmax(nhi.y, p.y), std::fmax(nhi.z, p.z)};
            }
        if (e - b <= 4) return;
        F3 ext = sub(nhi, nlo);
        int axis = ext.x >= ext.y && ext.x >= ext.z ? 0 : (ext.y >= ext.z ? 1 : 2);
        std::stable_sort(order.begin() + b, order.begin() + e, [&](uint32_t p, uint32_t q) {
            float fp = comp(centroid(p), axis), fq = comp(centroid(q), axis);
            return fp < fq || (fp == fq && p < q);
        });
        uint32_t mid = b + (e - b) / 2;
        build(b, mid);
        build(mid, e);
    };
    build(0, nt);
    std::vector<uint32_t> re(ni);
    for (uint32_t t = 0; t < nt; ++t)
        for (uint32_t c = 0; c < 3; ++c) re[3 * t + c] = idx[3 * order[t] + c];
    m.indices = re;
    m.convex = convex_planes(v, re, m.planes);
    F3 center = mul(add(lo, hi), 0.5f);
    float r2 = 0;
    for (auto& p : v) r2 = std::max(r2, dot(sub(p, center), sub(p, center)));
    m.lo = {lo.x, lo.y, lo.z};
    m.hi = {hi.x, hi.y, hi.z};
    m.center = {center.x, center.y, center.z};
    m.radius = std::sqrt(r2);
    return m;
}

}  // namespace pmb

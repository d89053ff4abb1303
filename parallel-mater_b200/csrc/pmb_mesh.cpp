// SPDX-License-Identifier: MIT
// Host mesh preparation for rigid triangle meshes, as the reference does at
// upload (src/simulation/runtime_deformables.cu.inc:103-270): a median-split
// BVH (<= 4 triangles per leaf, split axis = longest extent, stable sort of
// triangle centroids) whose leaf order becomes the stored triangle order; the
// closed-convex-plane certificate of runtime_domains.cu.inc:1061-1108 (weld
// exact duplicate positions, every welded edge used twice, one outward plane
// per triangle, every vertex within tolerance behind it); AABB and bounding
// sphere about the AABB centre; the BVH nodes; the certified outward shell
// normals of runtime_domains.cu.inc:1111-1235. Compiled with
// -ffp-contract=off so the plane arithmetic is the reference's FP32 sequence.
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

// A certified outward normal per triangle (zero where uncertified, a quarter
// length for an interior triangle of an open surface). Triangles form
// components through exactly welded positions; a closed convex component
// takes its planes' normals; a closed, consistently wound one its winding
// normals signed by its volume; an open one certifies a triangle with the
// whole component on one side of it. Empty when nothing was certified.
std::vector<std::array<float, 3>> shell_normals(const std::vector<F3>& v, const std::vector<uint32_t>& idx) {
    const uint32_t nv = uint32_t(v.size()), nt = uint32_t(idx.size() / 3);
    std::map<std::array<float, 3>, uint32_t> weld;
    std::vector<uint32_t> remap(nv), parent(nv);
    for (uint32_t i = 0; i < nv; ++i) {
        remap[i] = weld.emplace(std::array<float, 3>{v[i].x, v[i].y, v[i].z}, i).first->second;
        parent[i] = i;
    }
    auto root = [&](uint32_t i) {
        while (parent[i] != i) {
            parent[i] = parent[parent[i]];
            i = parent[i];
        }
        return i;
    };
    for (uint32_t t = 0; t < nt; ++t)
        for (uint32_t c = 1; c < 3; ++c) {
            const uint32_t a = root(remap[idx[3 * t]]), b = root(remap[idx[3 * t + c]]);
            parent[b] = a;
        }
    std::map<uint32_t, std::vector<uint32_t>> comps;
    for (uint32_t t = 0; t < nt; ++t) comps[root(remap[idx[3 * t]])].push_back(t);
    std::vector<std::array<float, 3>> normals(nt, std::array<float, 3>{0.0f, 0.0f, 0.0f});
    bool found = false;
    auto put = [&](uint32_t t, F3 n) { normals[t] = {n.x, n.y, n.z}; };
    for (const auto& kv : comps) {
        const std::vector<uint32_t>& tris = kv.second;
        std::map<uint32_t, uint32_t> local;
        std::vector<F3> pts;
        std::vector<uint32_t> faces;
        for (uint32_t t : tris)
            for (uint32_t c = 0; c < 3; ++c) {
                const uint32_t vert = remap[idx[3 * t + c]];
                auto ins = local.emplace(vert, uint32_t(pts.size()));
                if (ins.second) pts.push_back(v[vert]);
                faces.push_back(ins.first->second);
            }
        std::vector<std::array<float, 4>> planes;
        if (convex_planes(pts, faces, planes)) {
            found = true;
            for (size_t i = 0; i < tris.size(); ++i) put(tris[i], F3{planes[i][0], planes[i][1], planes[i][2]});
            continue;
        }
        std::map<std::pair<uint32_t, uint32_t>, std::pair<unsigned, int>> edges;
        double volume = 0.0;
        for (size_t f = 0; f < faces.size(); f += 3) {
            for (size_t c = 0; c < 3; ++c) {
                const uint32_t a = faces[f + c], b = faces[f + (c + 1) % 3];
                auto& e = edges[{std::min(a, b), std::max(a, b)}];
                ++e.first;
                e.second += a < b ? 1 : -1;
            }
            double q[3][3];
            for (size_t c = 0; c < 3; ++c) {
                const F3 p = pts[faces[f + c]];
                q[c][0] = double(p.x) - pts[0].x;
                q[c][1] = double(p.y) - pts[0].y;
                q[c][2] = double(p.z) - pts[0].z;
            }
            volume += q[0][0] * (q[1][1] * q[2][2] - q[1][2] * q[2][1]) +
                      q[0][1] * (q[1][2] * q[2][0] - q[1][0] * q[2][2]) +
                      q[0][2] * (q[1][0] * q[2][1] - q[1][1] * q[2][0]);
        }
        bool closed = volume != 0.0 && std::isfinite(volume);
        for (const auto& e : edges) closed = closed && e.second.first == 2u && e.second.second == 0;
        if (!closed) {
            float scale = 0.0f;
            for (const auto& p : pts) scale = std::max(scale, len(sub(p, pts[0])));
            const float tol = std::max(1.0e-7f, scale * 1.0e-5f);
            for (size_t i = 0; i < tris.size(); ++i) {
                const F3 a = pts[faces[3 * i]];
                const F3 nrm =
                    normalized_or(cross(sub(pts[faces[3 * i + 1]], a), sub(pts[faces[3 * i + 2]], a)), F3{0, 0, 0});
                float lo = 0.0f, hi = 0.0f;
                for (const auto& p : pts) {
                    const float dist = dot(nrm, sub(p, a));
                    lo = std::min(lo, dist);
                    hi = std::max(hi, dist);
                }
                if (hi <= tol && lo < -tol) {
                    put(tris[i], nrm);
                } else if (lo >= -tol && hi > tol) {
                    put(tris[i], mul(nrm, -1.0f));
                } else {
                    bool interior = true;
                    for (size_t c = 0; c < 3; ++c) {
                        const uint32_t f0 = faces[3 * i + c], f1 = faces[3 * i + (c + 1) % 3];
                        const auto& e = edges.at({std::min(f0, f1), std::max(f0, f1)});
                        interior = interior && e.first == 2u && e.second == 0;
                    }
                    if (!interior) continue;
                    put(tris[i], mul(nrm, 0.25f));
                }
                found = true;
            }
            continue;
        }
        found = true;
        for (size_t i = 0; i < tris.size(); ++i) {
            const F3 a = pts[faces[3 * i]], b = pts[faces[3 * i + 1]], c = pts[faces[3 * i + 2]];
            put(tris[i], mul(normalized_or(cross(sub(b, a), sub(c, a)), F3{0, 0, 0}), volume > 0.0 ? 1.0f : -1.0f));
        }
    }
    if (!found) normals.clear();
    return normals;
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
    std::function<uint32_t(uint32_t, uint32_t)> build = [&](uint32_t b, uint32_t e) -> uint32_t {
        F3 nlo{3.402823466e38f, 3.402823466e38f, 3.402823466e38f};
        F3 nhi = mul(nlo, -1.0f);
        for (uint32_t i = b; i < e; ++i)
            for (uint32_t c = 0; c < 3; ++c) {
                F3 p = v[idx[3 * order[i] + c]];
                nlo = {std::fmin(nlo.x, p.x), std::fmin(nlo.y, p.y), std::fmin(nlo.z, p.z)};
                nhi = {std::fmax(nhi.x, p.x), std::fmax(nhi.y, p.y), std::fmax(nhi.z, p.z)};
            }
        const uint32_t node = uint32_t(m.bvh.size());
        m.bvh.push_back(BvhNodeHost{{nlo.x, nlo.y, nlo.z}, {nhi.x, nhi.y, nhi.z}, 0, 0, 0, 0});
        if (e - b <= 4) {
            m.bvh[node].first = b;
            m.bvh[node].count = e - b;
            return node;
        }
        F3 ext = sub(nhi, nlo);
        int axis = ext.x >= ext.y && ext.x >= ext.z ? 0 : (ext.y >= ext.z ? 1 : 2);
        std::stable_sort(order.begin() + b, order.begin() + e, [&](uint32_t p, uint32_t q) {
            float fp = comp(centroid(p), axis), fq = comp(centroid(q), axis);
            return fp < fq || (fp == fq && p < q);
        });
        uint32_t mid = b + (e - b) / 2;
        const uint32_t left = build(b, mid);
        const uint32_t right = build(mid, e);
        m.bvh[node].left = left;
        m.bvh[node].right = right;
        return node;
    };
    if (nt) build(0, nt);
    std::vector<uint32_t> re(ni);
    for (uint32_t t = 0; t < nt; ++t)
        for (uint32_t c = 0; c < 3; ++c) re[3 * t + c] = idx[3 * order[t] + c];
    m.indices = re;
    m.convex = convex_planes(v, re, m.planes);
    m.shell = shell_normals(v, re);
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

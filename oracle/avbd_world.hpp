// SPDX-License-Identifier: MIT
// ORACLE — test infrastructure only (see avbd_math.hpp). Serial restatement of
// one rigid AVBD tick of the reference, in the order its Slang CPU driver runs
// the kernels (src/device/cpu_dispatch.hpp:127-157: one lane, one group, so
// every grid-stride loop is an in-order loop). Stage by stage:
//   integrate            geometry.slang:524-612
//   spatial proxies      geometry.slang:716-827
//   broadphase + filter  primitives/spatial_build.slang:889-1011,
//                        geometry.slang:829-947
//   face narrowphase     geometry.slang:1129-1270, 1586-1853, 2741-2803
//   finalize             geometry.slang:2805-2873
//   contact cache        geometry.slang:2941-3070
//   prepare + colouring  geometry_constraints.slang:1213-1591
//   solve                geometry_constraints_solve.slang:174-847
//   speed clamp          geometry.slang:3086-3100
// Host mesh preparation follows src/simulation/runtime_deformables.cu.inc:
// 103-270 and runtime_domains.cu.inc:1061-1108.
// Storage is sparse (pairs sorted by code, cache keyed by pair code) instead
// of the reference's N^2 tables; the observable semantics are the same:
// active-pair order, manifold-by-rank, and a cache hit iff the pair saved a
// non-empty manifold in the previous epoch with the same ids and timestep.
#pragma once
#include <algorithm>
#include <array>
#include <cstring>
#include <functional>
#include <map>
#include <numeric>
#include <vector>

#include "avbd_math.hpp"

namespace oracle {

constexpr uint32_t kInvalid = 0xffffffffu;
enum Motion : uint32_t { kStatic = 0, kKinematic = 1, kDynamic = 2 };
enum JointType : uint32_t { kFixed, kPoint, kHinge, kSlider, kPiston, kGeneric, kGenericSpring, kMotor };

// ------------------------------------------------------------ C-ABI records
// Field order of BodyParameters (types.slang:81-95) minus ids/user data.
struct BodyDesc {
    uint32_t motion, mesh;
    float inv_mass, inv_inertia[3], friction, restitution, linear_damping, angular_damping;
    float max_linear_speed, max_angular_speed, margin;
};
// RigidBodyState / PmRigidState: 13 floats.
struct StateDesc { float x[3], q[4], v[3], w[3]; };
// RigidConstraintOptions (geometry.slang:95-113) with dense body indices.
struct JointDesc {
    uint32_t type, body_a, body_b;
    float anchor_a[3], anchor_b[3], frame_a[4], frame_b[4];
    uint32_t lin_limit_axes; float lin_lower[3], lin_upper[3];
    uint32_t ang_limit_axes; float ang_lower[3], ang_upper[3];
    uint32_t lin_spring_axes; float lin_stiffness[3], lin_damping[3];
    uint32_t ang_spring_axes; float ang_stiffness[3], ang_damping[3];
    uint32_t motor_linear, motor_angular;
    float motor_linear_velocity, motor_linear_max_impulse;
    float motor_angular_velocity, motor_angular_max_impulse;
    uint32_t enabled, disable_collisions;
    float breaking_threshold;
    uint32_t solver_iterations;
};
struct StepDesc {
    float dt, gravity[3];
    uint32_t profile;               // 1 = realtime v1 (8 sweeps), else legacy
    uint32_t requested_iterations;  // legacy: 0 -> base_iterations
    uint32_t base_iterations;
    float residual_tolerance;       // > 0: stop sweeping once the residual is below it
    uint32_t max_iterations;        // cap for the residual-driven loop
    uint32_t warm_start;            // 0: plain (the only source the oracle models)
    uint32_t collect_events;        // not used by the oracle (it always keeps its events)
    uint32_t residual_norm;         // stop rule: 0 largest row violation, 1 RMS, 2 99.9th percentile
};
struct StepStats {
    uint32_t candidate_pairs, active_pairs, contacts, colors, islands, iterations, impact, status;
    float residual, residual_max, residual_over;
};

// ------------------------------------------------------------ world types
template <class R> struct State { V3<R> x; Q4<R> q; V3<R> v, w; };
template <class R> struct Plane { V3<R> n; R d{}; };
template <class R> struct BvhNode {
    V3<R> lo, hi;
    uint32_t first{}, count{}, left{}, right{};  // count != 0: a leaf
};
template <class R> struct Mesh {
    std::vector<V3<R>> verts;
    std::vector<uint32_t> idx;      // BVH-reordered triangle order
    std::vector<Plane<R>> planes;   // one per triangle when convex
    std::vector<BvhNode<R>> bvh;    // nodes in build (pre-)order, root first
    std::vector<V3<R>> shell;       // certified outward normal per triangle, or empty
    bool convex{};
    V3<R> lo, hi, center;
    R radius{};
};
template <class R> struct Contact {
    V3<R> normal, point;
    R penetration{};
    R acc_n{};
    V3<R> acc_f;
    R init_speed{};
    uint32_t persistent{};
    R impact_fraction{};
    R rep_n{};
    V3<R> rep_f;
    Dual<R> dual[3];
    V3<R> error, anchor_a, anchor_b;
    uint32_t cached{};
    uint32_t stick{};  // stick flag of the latest dual pass
};
template <class R> struct Manifold {
    Contact<R> c[8];
    uint32_t count{};
    uint32_t next_a{kInvalid}, next_b{kInvalid};
    bool guided{};  // a guided pair's contacts (geometry_constraints.slang:327-333)
};
template <class R> struct JointRt {
    JointDesc d{};
    uint32_t alive{1}, enabled{}, broken{};
    R applied{};
    uint32_t dense_a{kInvalid}, dense_b{kInvalid};
    Row<R> rows[18];
    uint32_t count{};
    uint32_t next_a{kInvalid}, next_b{kInvalid};
    // Residual sink for hard rows visited by an advance pass.
    void (*residual_sink)(void*, R){};
    void* residual_ctx{};
};
template <class R> struct AvbdBody {
    State<R> target;
    Q4<R> dq{0, 0, 0, 1};
    Vec6<R> dx;
    Block<R> inertia;
    uint32_t contact_head{kInvalid}, joint_head{kInvalid}, color{kInvalid}, parent{}, impact{};
    V3<R> prev_velocity;
    uint32_t history{};
};
template <class R> struct SavedContact {
    V3<R> local, normal;
    R normal_impulse{};
    V3<R> friction_impulse;
    Dual<R> dual[3];
    V3<R> anchor_a, anchor_b;
};
template <class R> struct SavedPair {
    uint64_t pair{};  // a * N + b in 64 bits (the reference's uint32 code for N <= 65,535)
    uint64_t epoch{};
    R dt{};
    uint32_t count{};
    SavedContact<R> c[8];
};

template <class R> inline V3<R> v3(const float* p) { return {R(p[0]), R(p[1]), R(p[2])}; }
template <class R> inline Q4<R> q4(const float* p) { return {R(p[0]), R(p[1]), R(p[2]), R(p[3])}; }

// --------------------------------------------------------- mesh preparation
// runtime_domains.cu.inc:1061-1108 (closed convex planes, one per triangle).
template <class R>
inline bool convex_planes(const std::vector<V3<R>>& v, const std::vector<uint32_t>& idx, std::vector<Plane<R>>& out) {
    out.clear();
    std::map<std::array<R, 3>, uint32_t> weld;
    std::vector<uint32_t> remap(v.size());
    V3<R> center{};
    for (uint32_t i = 0; i < v.size(); ++i) {
        auto e = weld.emplace(std::array<R, 3>{v[i].x, v[i].y, v[i].z}, uint32_t(weld.size()));
        remap[i] = e.first->second;
        if (e.second) center = add(center, v[i]);
    }
    if (weld.size() < 4) return false;
    center = mul(center, R(1) / R(weld.size()));
    std::map<uint64_t, uint32_t> edges;
    for (size_t t = 0; t < idx.size(); t += 3)
        for (size_t e = 0; e < 3; ++e) {
            uint64_t a = remap[idx[t + e]], b = remap[idx[t + (e + 1) % 3]];
            ++edges[(std::min(a, b) << 32) | std::max(a, b)];
        }
    for (auto& e : edges)
        if (e.second != 2) return false;
    R scale = 0;
    for (auto& p : v) scale = std::max(scale, len(sub(p, center)));
    const R tol = std::max(R(1.0e-7), scale * R(1.0e-5));
    for (size_t t = 0; t < idx.size(); t += 3) {
        V3<R> a = v[idx[t]];
        V3<R> n = normalized_or(cross(sub(v[idx[t + 1]], a), sub(v[idx[t + 2]], a)), V3<R>{});
        R side = dot(n, sub(a, center));
        if (ab(side) <= tol) { out.clear(); return false; }
        if (side < R(0)) n = mul(n, R(-1));
        R d = dot(n, a);
        for (auto& p : v)
            if (dot(n, p) - d > tol) { out.clear(); return false; }
        out.push_back({n, d});
    }
    return true;
}

// runtime_deformables.cu.inc:103-270: median-split BVH (<=4 triangles per
// leaf) whose leaf order becomes the stored triangle order; bounds, sphere.
template <class R>
inline std::vector<V3<R>> shell_normals(const std::vector<V3<R>>& v, const std::vector<uint32_t>& idx);

template <class R> inline Mesh<R> prepare_mesh(const float* verts, uint32_t nv, const uint32_t* idx, uint32_t ni) {
    Mesh<R> m;
    m.verts.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) m.verts[i] = v3<R>(verts + 3 * i);
    m.lo = m.hi = m.verts[0];
    for (uint32_t i = 1; i < nv; ++i) { m.lo = vmin(m.lo, m.verts[i]); m.hi = vmax(m.hi, m.verts[i]); }
    const uint32_t nt = ni / 3;
    std::vector<uint32_t> order(nt);
    std::iota(order.begin(), order.end(), 0u);
    auto centroid = [&](uint32_t t) {
        return mul(add(add(m.verts[idx[3 * t]], m.verts[idx[3 * t + 1]]), m.verts[idx[3 * t + 2]]), R(1) / R(3));
    };
    std::function<uint32_t(uint32_t, uint32_t)> build = [&](uint32_t b, uint32_t e) -> uint32_t {
        V3<R> lo{R(3.402823466e38), R(3.402823466e38), R(3.402823466e38)};
        V3<R> hi = mul(lo, R(-1));
        for (uint32_t i = b; i < e; ++i)
            for (uint32_t c = 0; c < 3; ++c) {
                lo = vmin(lo, m.verts[idx[3 * order[i] + c]]);
                hi = vmax(hi, m.verts[idx[3 * order[i] + c]]);
            }
        const uint32_t node = uint32_t(m.bvh.size());
        m.bvh.push_back(BvhNode<R>{lo, hi, 0, 0, 0, 0});
        if (e - b <= 4) {
            m.bvh[node].first = b;
            m.bvh[node].count = e - b;
            return node;
        }
        V3<R> ext = sub(hi, lo);
        unsigned axis = ext.x >= ext.y && ext.x >= ext.z ? 0 : (ext.y >= ext.z ? 1 : 2);
        std::stable_sort(order.begin() + b, order.begin() + e, [&](uint32_t p, uint32_t q) {
            R fp = comp(centroid(p), axis), fq = comp(centroid(q), axis);
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
    m.idx.resize(ni);
    for (uint32_t t = 0; t < nt; ++t)
        for (uint32_t c = 0; c < 3; ++c) m.idx[3 * t + c] = idx[3 * order[t] + c];
    m.convex = convex_planes(m.verts, m.idx, m.planes);
    m.shell = shell_normals(m.verts, m.idx);
    m.center = mul(add(m.lo, m.hi), R(0.5));
    R r2 = 0;
    for (auto& p : m.verts) r2 = std::max(r2, len2(sub(p, m.center)));
    m.radius = std::sqrt(r2);
    return m;
}

// ------------------------------------------------------------------ world
template <class R> struct World {
    uint32_t n{};
    std::vector<BodyDesc> body;
    std::vector<State<R>> state;
    std::vector<Mesh<R>> meshes;
    std::vector<JointRt<R>> joints;
    std::vector<AvbdBody<R>> avbd;
    std::vector<V3<R>> force, torque, impulse, angular_impulse;
    // Kinematic targets for the next tick (types.slang KinematicTarget).
    std::vector<State<R>> target;
    std::vector<uint8_t> target_set;
    std::vector<SavedPair<R>> saved;  // sorted by pair code
    uint64_t epoch{};
    // Last tick, for inspection by tests.
    std::vector<uint64_t> candidate_pairs;
    std::vector<uint64_t> active_pairs;  // non-empty manifolds only, code order
    std::vector<Manifold<R>> manifolds;   // parallel to active_pairs
    std::vector<V3<R>> aabb_lo, aabb_hi;
    std::vector<R> residual_trace;
    StepStats stats{};
    // Residual of the current dual pass: squares, rows, largest violation.
    double res_sq{};
    uint64_t res_n{};
    R res_max{}, residual_max_last{}, residual_rms_last{};
    uint64_t res_over{};  // rows above res_tol in the current pass
    R res_tol{};
    float residual_over_last{};
    void residual_add(R v) {
        res_sq += double(v) * double(v);
        ++res_n;
        res_max = v > res_max ? v : res_max;
        if (v > res_tol) ++res_over;
    }
};

template <class R> inline State<R> to_state(const StateDesc& s) {
    return {v3<R>(s.x), q4<R>(s.q), v3<R>(s.v), v3<R>(s.w)};
}
template <class R> inline StateDesc from_state(const State<R>& s) {
    return {{float(s.x.x), float(s.x.y), float(s.x.z)},
            {float(s.q.x), float(s.q.y), float(s.q.z), float(s.q.w)},
            {float(s.v.x), float(s.v.y), float(s.v.z)},
            {float(s.w.x), float(s.w.y), float(s.w.z)}};
}
template <class R> inline bool dynamic(const World<R>& w, uint32_t i) { return w.body[i].motion == kDynamic; }

// math.slang:208-217
template <class R> inline V3<R> inv_inertia_world(const BodyDesc& b, Q4<R> q, V3<R> v) {
    V3<R> l = inv_rotate(q, v);
    return rotate(q, V3<R>{l.x * R(b.inv_inertia[0]), l.y * R(b.inv_inertia[1]), l.z * R(b.inv_inertia[2])});
}

// geometry.slang:524-612 (one substep, impulses applied)
template <class R> inline State<R> integrate(const World<R>& w, uint32_t i, V3<R> g, R dt) {
    const BodyDesc& b = w.body[i];
    State<R> prev = w.state[i], next = prev;
    if (b.motion == kStatic) {
        next.v = {};
        next.w = {};
        return next;
    }
    if (b.motion == kKinematic) {
        // geometry.slang:545-581 with one remaining substep.
        if (w.target_set[i]) {
            const R fraction = R(1) / R(1);
            const State<R>& t = w.target[i];
            next.x = add(prev.x, mul(sub(t.x, prev.x), fraction));
            Q4<R> tq = t.q;
            const R od = prev.q.x * tq.x + prev.q.y * tq.y + prev.q.z * tq.z + prev.q.w * tq.w;
            if (od < R(0)) tq = Q4<R>{-tq.x, -tq.y, -tq.z, -tq.w};
            next.q = qnormalize(Q4<R>{prev.q.x + (tq.x - prev.q.x) * fraction, prev.q.y + (tq.y - prev.q.y) * fraction,
                                      prev.q.z + (tq.z - prev.q.z) * fraction, prev.q.w + (tq.w - prev.q.w) * fraction});
            next.v = mul(sub(next.x, prev.x), R(1) / dt);
            next.w = delta_velocity(prev.q, next.q, dt);
        } else {
            next.v = {};
            next.w = {};
        }
        return next;
    }
    next.v = add(next.v, mul(add(g, mul(w.force[i], R(b.inv_mass))), dt));
    next.w = add(next.w, mul(inv_inertia_world(b, next.q, w.torque[i]), dt));
    next.v = add(next.v, mul(w.impulse[i], R(b.inv_mass)));
    next.w = add(next.w, inv_inertia_world(b, next.q, w.angular_impulse[i]));
    next.v = mul(next.v, R(1) / (R(1) + R(b.linear_damping) * dt));
    next.w = mul(next.w, R(1) / (R(1) + R(b.angular_damping) * dt));
    next.v = clamp_length(next.v, R(b.max_linear_speed));
    next.w = clamp_length(next.w, R(b.max_angular_speed));
    next.x = add(next.x, mul(next.v, dt));
    Q4<R> d = qmul(Q4<R>{next.w.x, next.w.y, next.w.z, R(0)}, next.q);
    next.q = qnormalize(Q4<R>{next.q.x + R(0.5) * d.x * dt, next.q.y + R(0.5) * d.y * dt,
                              next.q.z + R(0.5) * d.z * dt, next.q.w + R(0.5) * d.w * dt});
    return next;
}

// geometry.slang:513-522
// runtime_domains.cu.inc:1111-1235: a certified outward normal per triangle.
// Triangles are grouped into components through shared (exactly welded)
// positions; a closed convex component takes its planes' normals; a closed,
// consistently wound component takes its winding normal signed by its volume;
// an open component certifies a triangle only when the whole component lies
// on one side of it (then the outward side), marks an interior triangle of an
// open surface with a quarter-length normal and leaves boundary triangles
// unrestricted (zero). Empty when no triangle got a normal.
template <class R>
inline std::vector<V3<R>> shell_normals(const std::vector<V3<R>>& v, const std::vector<uint32_t>& idx) {
    const uint32_t nv = uint32_t(v.size()), nt = uint32_t(idx.size() / 3);
    std::map<std::array<R, 3>, uint32_t> weld;
    std::vector<uint32_t> remap(nv), parent(nv);
    for (uint32_t i = 0; i < nv; ++i) {
        remap[i] = weld.emplace(std::array<R, 3>{v[i].x, v[i].y, v[i].z}, i).first->second;
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
    std::vector<V3<R>> normals(nt);
    bool found = false;
    for (const auto& kv : comps) {
        const std::vector<uint32_t>& tris = kv.second;
        std::map<uint32_t, uint32_t> local;
        std::vector<V3<R>> pts;
        std::vector<uint32_t> faces;
        for (uint32_t t : tris)
            for (uint32_t c = 0; c < 3; ++c) {
                const uint32_t vert = remap[idx[3 * t + c]];
                auto ins = local.emplace(vert, uint32_t(pts.size()));
                if (ins.second) pts.push_back(v[vert]);
                faces.push_back(ins.first->second);
            }
        std::vector<Plane<R>> planes;
        if (convex_planes(pts, faces, planes)) {
            found = true;
            for (size_t i = 0; i < tris.size(); ++i) normals[tris[i]] = planes[i].n;
            continue;
        }
        // Closed and consistently wound: every edge used twice, in opposite
        // directions; the signed volume fixes the outward sign.
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
                const V3<R> p = pts[faces[f + c]];
                q[c][0] = double(p.x) - double(pts[0].x);
                q[c][1] = double(p.y) - double(pts[0].y);
                q[c][2] = double(p.z) - double(pts[0].z);
            }
            volume += q[0][0] * (q[1][1] * q[2][2] - q[1][2] * q[2][1]) +
                      q[0][1] * (q[1][2] * q[2][0] - q[1][0] * q[2][2]) +
                      q[0][2] * (q[1][0] * q[2][1] - q[1][1] * q[2][0]);
        }
        bool closed = volume != 0.0 && std::isfinite(volume);
        for (const auto& e : edges) closed = closed && e.second.first == 2u && e.second.second == 0;
        if (!closed) {
            R scale = 0;
            for (const auto& p : pts) scale = std::max(scale, len(sub(p, pts[0])));
            const R tol = std::max(R(1.0e-7), scale * R(1.0e-5));
            for (size_t i = 0; i < tris.size(); ++i) {
                const V3<R> a = pts[faces[3 * i]];
                const V3<R> nrm =
                    normalized_or(cross(sub(pts[faces[3 * i + 1]], a), sub(pts[faces[3 * i + 2]], a)), V3<R>{});
                R lo = 0, hi = 0;
                for (const auto& p : pts) {
                    const R dist = dot(nrm, sub(p, a));
                    lo = std::min(lo, dist);
                    hi = std::max(hi, dist);
                }
                if (hi <= tol && lo < -tol) {
                    normals[tris[i]] = nrm;
                } else if (lo >= -tol && hi > tol) {
                    normals[tris[i]] = mul(nrm, R(-1));
                } else {
                    bool interior = true;
                    for (size_t c = 0; c < 3; ++c) {
                        const uint32_t f0 = faces[3 * i + c], f1 = faces[3 * i + (c + 1) % 3];
                        const auto& e = edges.at({std::min(f0, f1), std::max(f0, f1)});
                        interior = interior && e.first == 2u && e.second == 0;
                    }
                    if (!interior) continue;
                    normals[tris[i]] = mul(nrm, R(0.25));
                }
                found = true;
            }
            continue;
        }
        found = true;
        for (size_t i = 0; i < tris.size(); ++i) {
            const V3<R> a = pts[faces[3 * i]], b = pts[faces[3 * i + 1]], c = pts[faces[3 * i + 2]];
            normals[tris[i]] = mul(normalized_or(cross(sub(b, a), sub(c, a)), V3<R>{}), volume > 0.0 ? R(1) : R(-1));
        }
    }
    return found ? normals : std::vector<V3<R>>{};
}

template <class R> inline R correction_reach(const BodyDesc& b, const Mesh<R>& m) {
    if (b.motion != kDynamic) return R(0);
    V3<R> e = sub(m.hi, m.lo);
    return mn(R(0.5), R(0.25) * mx(R(0), mn(e.x, mn(e.y, e.z))));
}

// math.slang:192-206
template <class R> inline R rotational_motion_bound(const State<R>& prev, const State<R>& cur, const Mesh<R>& m) {
    Q4<R> d = qrelative(prev.q, cur.q, false);
    R s = len(V3<R>{d.x, d.y, d.z});
    V3<R> ma{mx(ab(m.lo.x), ab(m.hi.x)), mx(ab(m.lo.y), ab(m.hi.y)), mx(ab(m.lo.z), ab(m.hi.z))};
    return R(2) * len(ma) * s;
}

// ------------------------------------------------------------ narrowphase
// geometry.slang:1129-1220 (non-guided path)
template <class R> inline void add_contact(Manifold<R>& m, const Contact<R>& c, R spacing) {
    R s2 = spacing * spacing;
    for (uint32_t i = 0; i < m.count; ++i) {
        if (len2(sub(m.c[i].point, c.point)) < s2) {
            if (c.penetration - m.c[i].penetration > R(0)) m.c[i] = c;
            return;
        }
    }
    if (m.count < 8) { m.c[m.count++] = c; return; }
    uint32_t sh = 0;
    for (uint32_t i = 1; i < m.count; ++i)
        if (m.c[i].penetration < m.c[sh].penetration) sh = i;
    if (c.penetration > m.c[sh].penetration) m.c[sh] = c;
}

// geometry.slang:1228-1270
template <class R> inline void reduce_face_patch(Manifold<R>& m, R tol) {
    R t2 = tol * tol;
    bool removed = true;
    while (removed) {
        removed = false;
        for (uint32_t cand = 0; cand < m.count && !removed; ++cand) {
            V3<R> p = m.c[cand].point;
            for (uint32_t f = 0; f < m.count && !removed; ++f) {
                if (f == cand) continue;
                for (uint32_t s = f + 1; s < m.count; ++s) {
                    if (s == cand) continue;
                    V3<R> e = sub(m.c[s].point, m.c[f].point);
                    R e2 = len2(e);
                    if (e2 <= t2) continue;
                    R par = dot(sub(p, m.c[f].point), e) / e2;
                    if (par <= R(1.0e-4) || par >= R(0.9999)) continue;
                    V3<R> cl = add(m.c[f].point, mul(e, par));
                    if (len2(sub(p, cl)) > t2) continue;
                    for (uint32_t k = cand + 1; k < m.count; ++k) m.c[k - 1] = m.c[k];
                    --m.count;
                    removed = true;
                    break;
                }
            }
        }
    }
}

template <class R> inline bool face_capable(const Mesh<R>& m) { return m.convex && m.idx.size() <= 96; }

// geometry.slang:1606-1745
template <class R>
inline bool face_manifold(const State<R>& bs, const Mesh<R>& bm, const State<R>& cs, const Mesh<R>& cm, R margin,
                          R correction, Manifold<R>& out) {
    out = Manifold<R>{};
    const R rest = mn(margin, R(1.0e-3));
    const R reach = margin + correction;
    if (!face_capable(bm) || !face_capable(cm)) return false;
    R best = R(-3.402823466e38);
    uint32_t ref_face = 0;
    bool ref_body = false;
    for (uint32_t side = 0; side < 2; ++side) {
        const Mesh<R>& rm = side == 0 ? cm : bm;
        const State<R>& rs = side == 0 ? cs : bs;
        const Mesh<R>& im = side == 0 ? bm : cm;
        const State<R>& is = side == 0 ? bs : cs;
        for (uint32_t f = 0; f < rm.idx.size() / 3; ++f) {
            const Plane<R>& pl = rm.planes[f];
            V3<R> n = rotate(rs.q, pl.n);
            V3<R> in = inv_rotate(is.q, n);
            R support = R(3.402823466e38);
            for (auto& v : im.verts) support = std::fmin(support, dot(in, v));
            R sep = support + dot(n, sub(is.x, rs.x)) - pl.d;
            if (sep > best) { best = sep; ref_face = f; ref_body = side != 0; }
        }
    }
    if (best > reach) return true;
    const Mesh<R>& rm = ref_body ? bm : cm;
    const State<R>& rs = ref_body ? bs : cs;
    const Mesh<R>& im = ref_body ? cm : bm;
    const State<R>& is = ref_body ? cs : bs;
    const Plane<R> ref = rm.planes[ref_face];
    V3<R> outward = rotate(rs.q, ref.n);
    V3<R> inc_axis = inv_rotate(is.q, outward);
    R align = R(1);
    uint32_t inc_face = 0;
    for (uint32_t f = 0; f < im.idx.size() / 3; ++f) {
        R v = dot(inc_axis, im.planes[f].n);
        if (v < align) { align = v; inc_face = f; }
    }
    V3<R> normal = mul(outward, ref_body ? R(-1) : R(1));
    const Plane<R> inc = im.planes[inc_face];
    for (uint32_t t = 0; t < im.idx.size() / 3; ++t) {
        const Plane<R>& face = im.planes[t];
        if (dot(face.n, inc.n) < R(0.99999) || ab(face.d - inc.d) > R(1.0e-5)) continue;
        V3<R> poly[36], clip[36];
        uint32_t count = 3;
        for (uint32_t c = 0; c < 3; ++c)
            poly[c] = inv_rotate(rs.q, sub(add(is.x, rotate(is.q, im.verts[im.idx[3 * t + c]])), rs.x));
        for (uint32_t pi = 0; pi < rm.idx.size() / 3 && count != 0; ++pi) {
            const Plane<R>& pl = rm.planes[pi];
            R off = pl.d + (dot(pl.n, ref.n) > R(0.99999) ? reach : R(0));
            uint32_t cc = 0;
            V3<R> pv = poly[count - 1];
            R pd = dot(pl.n, pv) - off;
            for (uint32_t k = 0; k < count; ++k) {
                V3<R> cur = poly[k];
                R d = dot(pl.n, cur) - off;
                // Same 36-slot bound as the device narrowphase (rounding-degenerate polygons only).
                if ((d <= R(0)) != (pd <= R(0)) && cc < 36) clip[cc++] = add(pv, mul(sub(cur, pv), pd / (pd - d)));
                if (d <= R(0) && cc < 36) clip[cc++] = cur;
                pv = cur;
                pd = d;
            }
            count = cc;
            for (uint32_t k = 0; k < count; ++k) poly[k] = clip[k];
        }
        for (uint32_t k = 0; k < count; ++k) {
            R dist = dot(ref.n, poly[k]) - ref.d;
            if (dist > reach) continue;
            Contact<R> c{};
            c.normal = normal;
            c.point = add(rs.x, rotate(rs.q, sub(poly[k], mul(ref.n, dist * R(0.5)))));
            c.penetration = rest - dist + R(1.0e-5);
            c.impact_fraction = R(1);
            add_contact(out, c, mx(margin * R(2), R(1.0e-4)));
        }
    }
    if (out.count == 0) return false;
    reduce_face_patch(out, mx(R(1.0e-6), margin * R(1.0e-3)));
    return true;
}

// geometry.slang:1751-1853 (translation-only swept face contact)
template <class R>
inline bool swept_face_manifold(const State<R>& pb, const State<R>& b, const Mesh<R>& bm, const State<R>& pc,
                                const State<R>& c, const Mesh<R>& cm, R margin, Manifold<R>& out) {
    out = Manifold<R>{};
    Q4<R> bd = qrelative(pb.q, b.q, false), cd = qrelative(pc.q, c.q, false);
    if (bd.x != R(0) || bd.y != R(0) || bd.z != R(0) || cd.x != R(0) || cd.y != R(0) || cd.z != R(0)) return false;
    V3<R> bmo = sub(b.x, pb.x), cmo = sub(c.x, pc.x);
    const R rest = mn(margin, R(1.0e-3));
    R entry = 0, exit_t = 1;
    V3<R> entry_n{};
    for (uint32_t side = 0; side < 2; ++side) {
        const Mesh<R>& rm = side == 0 ? cm : bm;
        const Mesh<R>& im = side == 0 ? bm : cm;
        const State<R>& rs = side == 0 ? pc : pb;
        const State<R>& is = side == 0 ? pb : pc;
        V3<R> rel = side == 0 ? sub(bmo, cmo) : sub(cmo, bmo);
        for (uint32_t f = 0; f < rm.idx.size() / 3; ++f) {
            const Plane<R>& pl = rm.planes[f];
            V3<R> n = rotate(rs.q, pl.n);
            V3<R> in = inv_rotate(is.q, n);
            R support = R(3.402823466e38);
            for (auto& v : im.verts) support = std::fmin(support, dot(in, v));
            R gap = support + dot(n, sub(is.x, rs.x)) - pl.d;
            R speed = dot(n, rel);
            if (speed == R(0)) {
                if (gap > rest) return true;
            } else {
                R crossing = (rest - gap) / speed;
                if (speed < R(0) && crossing > entry) { entry = crossing; entry_n = mul(n, side == 0 ? R(1) : R(-1)); }
                if (speed > R(0)) exit_t = mn(exit_t, crossing);
            }
        }
    }
    if (entry > exit_t || entry > R(1) || exit_t < R(0)) return true;
    if (entry == R(0)) {
        bool clipped = face_manifold(b, bm, c, cm, margin, R(0), out);
        if (clipped && out.count != 0) return true;
        if (!face_manifold(pb, bm, pc, cm, margin, R(0), out) || out.count == 0) return false;
        for (uint32_t p = 0; p < out.count; ++p) {
            R closing = -dot(sub(bmo, cmo), out.c[p].normal);
            if (closing <= R(0)) return false;
            out.c[p].penetration += closing;
            out.c[p].impact_fraction = R(0);
        }
        return true;
    }
    State<R> ib = pb, ic = pc;
    ib.x = add(pb.x, mul(bmo, entry));
    ic.x = add(pc.x, mul(cmo, entry));
    if (!face_manifold(ib, bm, ic, cm, rest + R(1.0e-5), R(0), out) || out.count == 0) return false;
    for (uint32_t p = 0; p < out.count; ++p) {
        Contact<R> k = out.c[p];
        if (dot(k.normal, entry_n) < R(0.99999)) return false;
        R remaining = -dot(sub(bmo, cmo), k.normal) * (R(1) - entry);
        k.penetration = mx(R(0), remaining + k.penetration) + rest + R(1.0e-5);
        k.impact_fraction = entry;
        out.c[p] = k;
    }
    return true;
}

// geometry.slang:1272-1280
template <class R> inline R contact_normal_speed(const State<R>& b, const State<R>& c, V3<R> p, V3<R> n) {
    V3<R> bv = add(b.v, cross(b.w, sub(p, b.x)));
    V3<R> cv = add(c.v, cross(c.w, sub(p, c.x)));
    return dot(sub(bv, cv), n);
}

// --------------------------------------------------------------- AVBD path
// geometry_constraints.slang:424-446
template <class R> inline void basis(V3<R> n, V3<R>& t0, V3<R>& t1) {
    t0 = normalized_or(cross(n, ab(n.x) < R(0.57735) ? V3<R>{1, 0, 0} : V3<R>{0, 1, 0}), V3<R>{0, 0, 1});
    t1 = cross(n, t0);
}
template <class R> inline R pair_stiffness(const BodyDesc& a, const BodyDesc& b, R dt) {
    return R(1) / (mx(R(a.inv_mass) + R(b.inv_mass), R(1.0e-6)) * dt * dt);
}
// geometry_constraints.slang:438-446: a guided contact rests at the guided
// offset (1e-4 m), any other at the rest offset (1e-3 m).
template <class R> inline R contact_skin(const BodyDesc& a, const BodyDesc& b, bool guided = false) {
    return mn(R(a.margin) + R(b.margin), guided ? R(1.0e-4) : R(1.0e-3)) + R(2) * R(1.0e-5);
}
template <class R> inline Vec6<R> jac(V3<R> l, V3<R> a) { return {{l.x, l.y, l.z, a.x, a.y, a.z}}; }

// geometry_constraints.slang:362-372
template <class R> inline State<R> pose(const AvbdBody<R>& b) {
    State<R> s = b.target;
    s.x = add(s.x, V3<R>{b.dx.v[0], b.dx.v[1], b.dx.v[2]});
    if (b.dq.x != R(0) || b.dq.y != R(0) || b.dq.z != R(0)) s.q = qnormalize(qmul(b.dq, s.q));
    return s;
}
// geometry_constraints.slang:374-399
template <class R> inline void apply_pose_update(AvbdBody<R>& b, const Vec6<R>& u) {
    for (unsigned k = 0; k < 3; ++k) b.dx.v[k] += u.v[k];
    V3<R> r{u.v[3], u.v[4], u.v[5]};
    if (r.x == R(0) && r.y == R(0) && r.z == R(0)) return;
    Q4<R> rel = b.dq;
    Q4<R> d = qmul(Q4<R>{r.x, r.y, r.z, R(0)}, rel);
    rel = qnormalize(Q4<R>{rel.x + R(0.5) * d.x, rel.y + R(0.5) * d.y, rel.z + R(0.5) * d.z, rel.w + R(0.5) * d.w});
    if (rel.w < R(0)) rel = {-rel.x, -rel.y, -rel.z, -rel.w};
    b.dq = rel;
    b.dx.v[3] = R(2) * rel.x;
    b.dx.v[4] = R(2) * rel.y;
    b.dx.v[5] = R(2) * rel.z;
}
// geometry_constraints.slang:401-422
template <class R> inline V3<R> log_axis(Q4<R> frame, V3<R> lg, unsigned axis) {
    R s = len2(lg);
    R coef = R(1) / R(12) + s * (R(1) / R(720) + s * (R(1) / R(30240) + s * (R(1) / R(1209600) + s / R(47900160))));
    if (s > R(1)) {
        R ang = std::sqrt(s);
        R half = R(0.5) * ang;
        coef = (R(1) - x_cot(half)) / s;
    }
    V3<R> u = unit_axis<R>(axis);
    V3<R> l = add(add(u, mul(cross(lg, u), R(0.5))), mul(cross(lg, cross(lg, u)), coef));
    return rotate(frame, l);
}

// geometry_constraints.slang:508-532: three rows (normal, tangent0, tangent1).
template <class R>
inline void contact_rows(const Contact<R>& c, const AvbdBody<R>& A, const AvbdBody<R>& B, Vec6<R> ja[3], Vec6<R> jb[3],
                         R err[3]) {
    V3<R> t0, t1;
    basis(c.normal, t0, t1);
    V3<R> axes[3] = {c.normal, t0, t1};
    V3<R> arm_a = sub(c.point, A.target.x), arm_b = sub(c.point, B.target.x);
    for (unsigned k = 0; k < 3; ++k) {
        V3<R> ra = k == 0 ? arm_a : rotate(A.target.q, c.anchor_a);
        V3<R> rb = k == 0 ? arm_b : rotate(B.target.q, c.anchor_b);
        ja[k] = jac(mul(axes[k], R(-1)), mul(cross(ra, axes[k]), R(-1)));
        jb[k] = jac(axes[k], cross(rb, axes[k]));
        err[k] = comp(c.error, k) + dot6(ja[k], A.dx) + dot6(jb[k], B.dx);
    }
}
template <class R>
inline R contact_normal_row(const Contact<R>& c, const AvbdBody<R>& A, const AvbdBody<R>& B, Vec6<R>& ja, Vec6<R>& jb) {
    V3<R> arm_a = sub(c.point, A.target.x), arm_b = sub(c.point, B.target.x);
    ja = jac(mul(c.normal, R(-1)), mul(cross(arm_a, c.normal), R(-1)));
    jb = jac(c.normal, cross(arm_b, c.normal));
    return c.error.x + dot6(ja, A.dx) + dot6(jb, B.dx);
}

enum JointVisit : unsigned { kInit = 0, kAccumulate = 1, kAdvance = 2, kImpact = 3 };

// geometry_constraints.slang:626-713
template <class R>
inline void joint_row(JointRt<R>& j, std::vector<AvbdBody<R>>& bodies, Block<R>& blk, uint32_t& index, R& impulse,
                      bool first, const Vec6<R>& ja, const Vec6<R>& jb, R current, R previous, R penalty, R dt,
                      bool angular, R stiffness, R damping, R lower, R upper, bool motor, R motor_speed, V3<R> curv_a,
                      V3<R> curv_b, R stabilization, unsigned visit) {
    uint32_t ri = index++;
    Row<R> row = j.rows[ri];
    const AvbdBody<R>& A = bodies[j.dense_a];
    const AvbdBody<R>& B = bodies[j.dense_b];
    R lin = dot6(ja, A.dx) + dot6(jb, B.dx);
    row.a = ja;
    row.b = jb;
    row.stiffness = stiffness;
    row.damping = damping;
    if (visit == kInit) {
        if (!(row.dual.penalty > K<R>::kmin)) row.dual.penalty = penalty;
        row.dual = warm_start(row.dual, stiffness);
        if (stiffness < K<R>::kmax) row.dual.lambda = R(0);
        row.beta = penalty * (angular ? R(10) : R(100));
        row.reference_force = R(0);
    }
    row.error = current - (stiffness < K<R>::kmax ? R(0) : stabilization * previous) - lin;
    row.velocity = motor ? motor_speed : (current - previous - lin) / dt;
    row.lower = lower;
    row.upper = upper;
    if (visit == kAccumulate) {
        row_accumulate(blk, row, first, A.dx, B.dx, dt);
        if (!angular) {
            V3<R> axis{jb.v[0], jb.v[1], jb.v[2]};
            V3<R> arm = first ? curv_a : curv_b;
            R force = row_force(row, A.dx, B.dx, dt);
            for (unsigned col = 0; col < 3; ++col) {
                V3<R> val = sub(mul(add(mul(axis, comp(arm, col)), mul(arm, comp(axis, col))), R(0.5)),
                                mul(unit_axis<R>(col), dot(axis, arm)));
                blk.h[bidx(3 + col, 3 + col)] += ab(force) * std::sqrt(len2(val));
            }
        }
    } else if (visit == kAdvance) {
        impulse += ab(row_force(row, A.dx, B.dx, dt)) * dt;
        if (stiffness >= K<R>::kmax && j.residual_sink) j.residual_sink(j.residual_ctx, ab(row_error(row, A.dx, B.dx)));
        j.rows[ri] = row_advance(row, A.dx, B.dx);
    } else if (visit == kImpact) {
        if (stiffness < K<R>::kmax) {
            row.reference_force = row_force(row, A.dx, B.dx, dt);
        } else {
            R gap = lower == R(0) ? mn(R(0), current) : (upper == R(0) ? mx(R(0), current) : R(0));
            Vec6<R> va = jac(mul(A.target.v, dt), mul(A.target.w, dt));
            Vec6<R> vb = jac(mul(B.target.v, dt), mul(B.target.w, dt));
            row.reference_force = row.dual.lambda;
            row.error = dot6(ja, va) + dot6(jb, vb) + gap - (motor ? motor_speed * dt : R(0));
        }
        j.rows[ri] = row;
    } else {
        j.rows[ri] = row;
    }
}

// geometry_constraints.slang:715-926
template <class R>
inline R visit_joint(JointRt<R>& j, const World<R>& w, const std::vector<State<R>>& previous,
                     std::vector<AvbdBody<R>>& bodies, R dt, Block<R>& blk, bool first, unsigned visit) {
    uint32_t index = 0;
    R impulse = 0;
    const JointDesc& o = j.d;
    const uint32_t a = j.dense_a, b = j.dense_b;
    State<R> sa = pose(bodies[a]), sb = pose(bodies[b]);
    V3<R> la = v3<R>(o.anchor_a), lb = v3<R>(o.anchor_b);
    Q4<R> fa_l = q4<R>(o.frame_a), fb_l = q4<R>(o.frame_b);
    V3<R> arm_a = rotate(sa.q, la), arm_b = rotate(sb.q, lb);
    V3<R> error = sub(add(sb.x, arm_b), add(sa.x, arm_a));
    V3<R> old_error = sub(add(previous[b].x, rotate(previous[b].q, lb)), add(previous[a].x, rotate(previous[a].q, la)));
    Q4<R> frame_a = qnormalize(qmul(sa.q, fa_l)), frame_b = qnormalize(qmul(sb.q, fb_l));
    Q4<R> old_a = qnormalize(qmul(previous[a].q, fa_l)), old_b = qnormalize(qmul(previous[b].q, fb_l));
    const uint32_t t = o.type;
    // The relative-rotation terms feed angular rows only. A point joint with
    // no angular limit, spring or motor emits none, so for it they are not
    // evaluated (pure functions of the poses: the rows are unchanged).
    const bool angular_rows = t != kPoint || o.ang_limit_axes != 0 || o.ang_spring_axes != 0 || o.motor_angular != 0;
    V3<R> twist{}, old_twist{};
    if (angular_rows) {
        twist = rotation_vector(qrelative(frame_a, frame_b, true));
        old_twist = rotation_vector(qrelative(old_a, old_b, true));
    }
    bool swing = t == kHinge || t == kPiston || (t == kMotor && o.motor_angular != 0);
    V3<R> free_axis = t == kHinge ? V3<R>{0, 0, 1} : V3<R>{1, 0, 0};
    V3<R> swing_axis{}, old_swing{};
    if (angular_rows) {
        swing_axis = inv_rotate(frame_a, rotate(frame_b, free_axis));
        old_swing = inv_rotate(old_a, rotate(old_b, free_axis));
    }
    V3<R> rotation = swing ? cross(free_axis, swing_axis) : twist;
    V3<R> old_rotation = swing ? cross(free_axis, old_swing) : old_twist;
    R lin_pen = pair_stiffness<R>(w.body[a], w.body[b], dt);
    for (unsigned axis = 0; axis < 3; ++axis) {
        V3<R> dir = rotate(frame_a, unit_axis<R>(axis));
        V3<R> old_dir = rotate(old_a, unit_axis<R>(axis));
        bool generic = t == kGeneric || t == kGenericSpring;
        bool motor_type = t == kMotor;
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
            R current = angular ? comp(rotation, axis) : dot(error, dir);
            R old_current = angular ? comp(old_rotation, axis) : dot(old_error, old_dir);
            V3<R> ang_axis = swing ? rotate(frame_a, sub(mul(unit_axis<R>(axis), dot(free_axis, swing_axis)),
                                                         mul(free_axis, comp(swing_axis, axis))))
                                   : log_axis(frame_a, twist, axis);
            Vec6<R> ja = angular ? jac(V3<R>{}, mul(ang_axis, R(-1)))
                                 : jac(mul(dir, R(-1)), add(mul(cross(arm_a, dir), R(-1)), cross(dir, error)));
            Vec6<R> jb = angular ? jac(V3<R>{}, ang_axis) : jac(dir, cross(arm_b, dir));
            R penalty = angular ? R(1) / (mx(dot(dir, add(inv_inertia_world(w.body[a], sa.q, dir),
                                                          inv_inertia_world(w.body[b], sb.q, dir))),
                                             R(1.0e-6)) *
                                          dt * dt)
                                : lin_pen;
            R lock_pen = angular ? mx(penalty, R(2) * lin_pen *
                                                   mx(len2(cross(dir, arm_a)), len2(cross(dir, arm_b))))
                                 : penalty;
            V3<R> curv_a = add(error, arm_a);
            if (lock) {
                if (visit == kInit && angular)
                    j.rows[index].dual.penalty = mx(j.rows[index].dual.penalty, lock_pen / K<R>::gamma);
                joint_row(j, bodies, blk, index, impulse, first, ja, jb, current, old_current, lock_pen, dt, angular,
                          K<R>::kmax, R(0), -K<R>::kmax, K<R>::kmax, false, R(0), curv_a, arm_b, K<R>::alpha, visit);
            }
            bool free_limit = angular ? ((t == kHinge && axis == 2) || (t == kPiston && axis == 0))
                                      : ((t == kSlider || t == kPiston) && axis == 0);
            if ((generic || free_limit) && (lim_axes & (1u << axis)) != 0) {
                R lc = angular ? comp(twist, axis) : current;
                R olc = angular ? comp(old_twist, axis) : old_current;
                V3<R> lax = log_axis(frame_a, twist, axis);
                Vec6<R> la6 = angular ? jac(V3<R>{}, mul(lax, R(-1))) : ja;
                Vec6<R> lb6 = angular ? jac(V3<R>{}, lax) : jb;
                R lower = R(lim_lo[axis]), upper = R(lim_hi[axis]);
                if (lower == upper) {
                    R eq_pen = angular && generic ? lock_pen : penalty;
                    if (visit == kInit && angular && generic)
                        j.rows[index].dual.penalty = mx(j.rows[index].dual.penalty, eq_pen / K<R>::gamma);
                    joint_row(j, bodies, blk, index, impulse, first, la6, lb6, lc - lower, olc - lower, eq_pen, dt,
                              angular, K<R>::kmax, R(0), -K<R>::kmax, K<R>::kmax, false, R(0), curv_a, arm_b,
                              K<R>::alpha, visit);
                } else if (lower < upper) {
                    joint_row(j, bodies, blk, index, impulse, first, la6, lb6, lc - upper, mx(olc - upper, R(0)),
                              penalty, dt, angular, K<R>::kmax, R(0), R(0), K<R>::kmax, false, R(0), curv_a, arm_b,
                              R(0.8), visit);
                    joint_row(j, bodies, blk, index, impulse, first, la6, lb6, lc - lower, mn(olc - lower, R(0)),
                              penalty, dt, angular, K<R>::kmax, R(0), -K<R>::kmax, R(0), false, R(0), curv_a, arm_b,
                              R(0.8), visit);
                }
            }
            if (t == kGenericSpring && (spr_axes & (1u << axis)) != 0)
                joint_row(j, bodies, blk, index, impulse, first, ja, jb, current, old_current, penalty, dt, angular,
                          R(spr_k[axis]), R(spr_c[axis]), -K<R>::kmax, K<R>::kmax, false, R(0), curv_a, arm_b,
                          K<R>::alpha, visit);
            if (motor_type && axis == 0 && (angular ? o.motor_angular != 0 : o.motor_linear != 0)) {
                R speed = R(angular ? o.motor_angular_velocity : o.motor_linear_velocity);
                R bound = R(angular ? o.motor_angular_max_impulse : o.motor_linear_max_impulse) / dt;
                Q4<R> rel = qrelative(frame_a, frame_b, true);
                Q4<R> old_rel = qrelative(old_a, old_b, true);
                V3<R> mrot = rotation_vector(qrelative(Q4<R>{0, 0, 0, 1}, qrelative(old_rel, rel, false), true));
                V3<R> max_ = log_axis(frame_a, mrot, axis);
                Vec6<R> ma = angular ? jac(V3<R>{}, mul(max_, R(-1))) : ja;
                Vec6<R> mb = angular ? jac(V3<R>{}, max_) : jb;
                R travel = angular ? comp(mrot, axis) : current - old_current;
                joint_row(j, bodies, blk, index, impulse, first, ma, mb, travel - speed * dt, R(0), penalty, dt,
                          angular, K<R>::kmax, R(0), -bound, bound, true, speed, curv_a, arm_b, K<R>::alpha, visit);
            }
        }
    }
    if (visit == kInit) j.count = index;
    return impulse;
}

// geometry_constraints.slang:983-1006
template <class R> inline bool contact_impact(const Manifold<R>& m, const BodyDesc& a, const BodyDesc& b, R dt) {
    bool impact = false;
    for (uint32_t p = 0; p < m.count; ++p) {
        const Contact<R>& c = m.c[p];
        R skin = contact_skin<R>(a, b, m.guided);
        bool fresh = (c.cached == 0 || c.dual[0].lambda <= R(1.0e-6) ||
                      (c.impact_fraction > R(0) && c.impact_fraction < R(1))) &&
                     c.init_speed < R(-0.1) && c.penetration >= R(-1.0e-5);
        R prev_pen = c.penetration + c.init_speed * dt;
        impact = impact || fresh || prev_pen > skin + R(1.0e-4);
    }
    return impact;
}

template <class R> inline uint32_t find_root(std::vector<AvbdBody<R>>& bodies, uint32_t i) {
    while (i != bodies[i].parent) i = bodies[i].parent;
    return i;
}

// Residual (added by this build, not in the reference): over contact normal
// rows that carry force or penetrate, |C_n| where the force is positive and
// C_n where only penetration makes the row active (a complementarity
// violation in metres), plus |C| of hard joint rows; reported as the RMS
// over those rows, with the largest single violation kept beside it.
template <class R> inline R contact_row_residual(R err_n, R force_n, bool& active) {
    active = force_n > R(0) || err_n > R(0);
    return force_n > R(0) ? ab(err_n) : err_n;
}

}  // namespace oracle

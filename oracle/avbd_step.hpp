// SPDX-License-Identifier: MIT
// ORACLE — test infrastructure only (see avbd_math.hpp). One rigid tick in
// the reference's order (production_realtime_backend.cu.inc:2642-2654 predict,
// :2656+ spatial build, :7664-7866 emit_rigid_solve).
#pragma once
#include "avbd_mesh.hpp"
#include "avbd_world.hpp"

namespace oracle {

template <class R> struct AabbBox { V3<R> lo, hi; };

// primitives/spatial_build.slang:631-635
template <class R> inline bool overlaps(const V3<R>& alo, const V3<R>& ahi, const V3<R>& blo, const V3<R>& bhi) {
    return ahi.x >= blo.x && ahi.y >= blo.y && ahi.z >= blo.z && bhi.x >= alo.x && bhi.y >= alo.y && bhi.z >= alo.z;
}

// Pair filter of geometry.slang:897-913 with identity order == dense order.
// constrained_collision_disabled (geometry.slang:494-511) scans every joint
// for each pair; the same predicate (an alive, enabled, unbroken joint with
// disable_collisions between a and b, either way round) is answered here from
// the sorted (min, max) body keys of those joints, gathered once per tick.
template <class R> inline std::vector<uint64_t> collision_disabled_keys(const World<R>& w) {
    std::vector<uint64_t> keys;
    for (auto& j : w.joints) {
        if (!j.alive || !j.d.enabled || j.broken || !j.d.disable_collisions) continue;
        const uint64_t lo = std::min(j.d.body_a, j.d.body_b), hi = std::max(j.d.body_a, j.d.body_b);
        keys.push_back(lo << 32 | hi);
    }
    std::sort(keys.begin(), keys.end());
    return keys;
}
inline bool collision_disabled(const std::vector<uint64_t>& keys, uint32_t a, uint32_t b) {
    const uint64_t lo = std::min(a, b), hi = std::max(a, b);
    return std::binary_search(keys.begin(), keys.end(), lo << 32 | hi);
}

// pm_build_fixed_collision_groups (geometry.slang:3102-3136): bodies joined
// through enabled, unbroken, collision-disabling fixed joints form a group
// whose root is its smallest dense index; a pair inside one group is not a
// candidate (:902-904). Empty when the world has no joints (the filter then
// gets no group buffer, production_realtime_backend.cu.inc:7684-7687).
template <class R> inline std::vector<uint32_t> fixed_groups(const World<R>& w) {
    std::vector<uint32_t> root;
    if (w.joints.empty()) return root;
    root.resize(w.n);
    for (uint32_t i = 0; i < w.n; ++i) root[i] = i;
    auto find = [&](uint32_t b) {
        while (root[b] != b) b = root[b];
        return b;
    };
    for (auto& j : w.joints) {
        if (!j.alive || !j.d.enabled || j.broken || !j.d.disable_collisions || j.d.type != kFixed) continue;
        if (j.d.body_a >= w.n || j.d.body_b >= w.n) continue;
        const uint32_t a = find(j.d.body_a), b = find(j.d.body_b);
        if (a != b) root[std::max(a, b)] = std::min(a, b);
    }
    for (uint32_t i = 0; i < w.n; ++i) root[i] = find(i);
    return root;
}

// Sorted candidate pairs over plain boxes: a a dynamic query box, b any
// other box whose bounds overlap a's (inclusive), b dynamic only when a < b
// (identity order == index order), a and b not in one fixed collision group
// (group[i]: the group's root, empty when there are no groups), and no
// collision-disabling joint between them (`disabled`: sorted (min, max) keys).
// A uniform grid keyed on box centre lists the candidates; boxes larger than
// 4x the median extent are tested against every query. Codes a*n+b, in
// (query, identity) order: spatial_build.slang:889-1011 with the filter of
// geometry.slang:829-947.
template <class R>
inline std::vector<uint64_t> broadphase_boxes(uint32_t n, const V3<R>* lo, const V3<R>* hi, const uint8_t* dyn,
                                              const std::vector<uint32_t>& group,
                                              const std::vector<uint64_t>& disabled) {
    std::vector<uint64_t> out;
    std::vector<R> ext(n);
    for (uint32_t i = 0; i < n; ++i) {
        V3<R> e = sub(hi[i], lo[i]);
        ext[i] = std::max(e.x, std::max(e.y, e.z));
    }
    std::vector<R> sorted = ext;
    std::nth_element(sorted.begin(), sorted.begin() + n / 2, sorted.end());
    R h = n ? sorted[n / 2] * R(4) : R(1);
    std::vector<uint32_t> large, small;
    for (uint32_t i = 0; i < n; ++i) (ext[i] > h ? large : small).push_back(i);
    R hs = 0;
    for (uint32_t i : small) hs = std::max(hs, ext[i]);
    if (!(hs > R(0))) hs = R(1);
    auto key = [&](uint32_t i, int dx, int dy, int dz) {
        V3<R> c = mul(add(lo[i], hi[i]), R(0.5));
        int64_t x = int64_t(std::floor(double(c.x / hs))) + dx, y = int64_t(std::floor(double(c.y / hs))) + dy,
                z = int64_t(std::floor(double(c.z / hs))) + dz;
        return std::array<int64_t, 3>{x, y, z};
    };
    std::map<std::array<int64_t, 3>, std::vector<uint32_t>> grid;
    for (uint32_t i : small) grid[key(i, 0, 0, 0)].push_back(i);
    std::vector<uint32_t> cand;
    for (uint32_t a = 0; a < n; ++a) {
        if (!dyn[a]) continue;
        cand.clear();
        auto test = [&](uint32_t b) {
            if (b == a) return;
            if (!overlaps(lo[b], hi[b], lo[a], hi[a])) return;
            if (dyn[b] && !(a < b)) return;
            if (!group.empty() && group[a] == group[b]) return;
            if (collision_disabled(disabled, a, b)) return;
            cand.push_back(b);
        };
        for (uint32_t b : large) test(b);
        if (ext[a] > h) {
            for (uint32_t b : small) test(b);
        } else {
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        auto it = grid.find(key(a, dx, dy, dz));
                        if (it == grid.end()) continue;
                        for (uint32_t b : it->second) test(b);
                    }
        }
        std::sort(cand.begin(), cand.end());
        for (uint32_t b : cand) out.push_back(uint64_t(a) * n + b);
    }
    return out;
}

// The world's candidate pairs: its swept proxies through broadphase_boxes.
template <class R> inline std::vector<uint64_t> broadphase(const World<R>& w) {
    std::vector<uint8_t> dyn(w.n);
    for (uint32_t i = 0; i < w.n; ++i) dyn[i] = dynamic(w, i) ? 1 : 0;
    return broadphase_boxes<R>(w.n, w.aabb_lo.data(), w.aabb_hi.data(), dyn.data(), fixed_groups(w),
                               collision_disabled_keys(w));
}

template <class R> inline void step(World<R>& w, const StepDesc& o) {
    const R dt = R(o.dt);
    const V3<R> g{R(o.gravity[0]), R(o.gravity[1]), R(o.gravity[2])};
    const uint32_t n = w.n;
    const bool realtime = o.profile == 1;
    const uint64_t epoch = w.epoch + 1;
    StepStats st{};
    std::vector<State<R>> prev = w.state;

    // ---- predict (geometry.slang:524-612)
    std::vector<State<R>> pred(n);
    for (uint32_t i = 0; i < n; ++i) pred[i] = integrate(w, i, g, dt);

    // ---- spatial proxies (geometry.slang:716-827)
    w.aabb_lo.assign(n, {});
    w.aabb_hi.assign(n, {});
    for (uint32_t i = 0; i < n; ++i) {
        const Mesh<R>& m = w.meshes[w.body[i].mesh];
        R reach = len(m.center) + m.radius + R(w.body[i].margin) + R(1.0e-5);
        R corr = mn(R(1), correction_reach(w.body[i], m));
        R e = corr + reach;
        V3<R> ex{e, e, e};
        w.aabb_lo[i] = sub(vmin(prev[i].x, pred[i].x), ex);
        w.aabb_hi[i] = add(vmax(prev[i].x, pred[i].x), ex);
    }

    // ---- broadphase (spatial_build.slang:889-1011, geometry.slang:829-947)
    w.candidate_pairs = broadphase(w);
    st.candidate_pairs = uint32_t(w.candidate_pairs.size());

    // ---- face narrowphase, triangle-mesh narrowphase, finalize
    // (geometry.slang:2741-2873, :2156-2299)
    w.active_pairs.clear();
    w.manifolds.clear();
    const std::vector<HingeFrame<R>> frames = hinge_frames(w, pred);
    const std::vector<HingeFrame<R>> prev_frames = hinge_frames(w, prev);
    for (uint64_t code : w.candidate_pairs) {
        uint32_t a = uint32_t(code / n), b = uint32_t(code % n);
        const Mesh<R>& bm = w.meshes[w.body[a].mesh];
        const Mesh<R>& cm = w.meshes[w.body[b].mesh];
        R margin = R(w.body[a].margin) + R(w.body[b].margin);
        Manifold<R> m{};
        bool face = false;
        if (face_capable(bm) && face_capable(cm) && !guided_pair(frames[a], frames[b])) {
            R corr = correction_reach(w.body[a], bm) + correction_reach(w.body[b], cm);
            R moved = len(sub(sub(pred[a].x, prev[a].x), sub(pred[b].x, prev[b].x))) +
                      rotational_motion_bound(prev[a], pred[a], bm) + rotational_motion_bound(prev[b], pred[b], cm);
            bool swept = moved > margin;
            if (swept) face = swept_face_manifold(prev[a], pred[a], bm, prev[b], pred[b], cm, margin, m);
            if (!face) {
                face = face_manifold(pred[a], bm, pred[b], cm, margin, corr, m);
                if (swept && m.count == 0) face = false;
            }
        }
        // A pair the face path declines goes to the triangle-mesh path.
        if (!face) collide_meshes(w, a, b, prev, pred, frames[a], frames[b], prev_frames[a].reference, dt, m);
        m.guided = guided_pair(frames[a], frames[b]);
        if (m.count == 0) continue;
        bool persistent = face_capable(bm) && (!dynamic(w, b) || face_capable(cm));
        for (uint32_t p = 0; p < m.count; ++p) {
            Contact<R>& c = m.c[p];
            c.persistent = persistent;
            c.init_speed = contact_normal_speed(pred[a], pred[b], c.point, c.normal);
            c.rep_n = c.acc_n;
            c.rep_f = c.acc_f;
        }
        w.active_pairs.push_back(code);
        w.manifolds.push_back(m);
    }
    const uint32_t P = uint32_t(w.active_pairs.size());
    st.active_pairs = P;

    // ---- contact cache load (geometry.slang:2941-3009)
    for (uint32_t k = 0; k < P; ++k) {
        const uint64_t code = w.active_pairs[k];
        const uint32_t a = uint32_t(code / n);
        auto it = std::lower_bound(w.saved.begin(), w.saved.end(), code,
                                   [](const SavedPair<R>& s, uint64_t c) { return s.pair < c; });
        if (it == w.saved.end() || it->pair != code || it->epoch + 1 != epoch || ab(it->dt - dt) > R(1.0e-7)) continue;
        const SavedPair<R>& sp = *it;
        Manifold<R>& m = w.manifolds[k];
        uint32_t used = 0;
        for (uint32_t p = 0; p < m.count; ++p) {
            Contact<R>& c = m.c[p];
            V3<R> local = inv_rotate(pred[a].q, sub(c.point, pred[a].x));
            R nearest = R(0.02) * R(0.02);
            uint32_t match = 8;
            for (uint32_t q = 0; q < sp.count; ++q) {
                if ((used & (1u << q)) != 0 || dot(c.normal, sp.c[q].normal) < R(0.99)) continue;
                R d = len2(sub(local, sp.c[q].local));
                if (d < nearest) { nearest = d; match = q; }
            }
            if (match == 8) continue;
            used |= 1u << match;
            const SavedContact<R>& s = sp.c[match];
            for (unsigned x = 0; x < 3; ++x) c.dual[x] = s.dual[x];
            V3<R> t0, t1;
            basis(c.normal, t0, t1);
            c.dual[1].lambda = dot(s.friction_impulse, t0) / dt;
            c.dual[2].lambda = dot(s.friction_impulse, t1) / dt;
            c.anchor_a = s.anchor_a;
            c.anchor_b = s.anchor_b;
            c.cached = 1;
            c.acc_n = s.normal_impulse;
            c.acc_f = sub(s.friction_impulse, mul(c.normal, dot(s.friction_impulse, c.normal)));
        }
    }

    // ---- prepare (geometry_constraints.slang:1213-1591)
    std::vector<AvbdBody<R>>& bodies = w.avbd;
    for (uint32_t i = 0; i < n; ++i) {
        V3<R> old_v = bodies[i].prev_velocity;
        bool hist = bodies[i].history != 0;
        AvbdBody<R> bd{};
        bd.parent = i;
        bd.color = kInvalid;
        bd.contact_head = kInvalid;
        bd.joint_head = kInvalid;
        bd.target = pred[i];
        bd.dq = {0, 0, 0, 1};
        bd.prev_velocity = {};
        bd.history = 0;
        if (!dynamic(w, i)) { bodies[i] = bd; continue; }
        R g2 = len2(g);
        V3<R> acc = mul(sub(prev[i].v, old_v), R(1) / dt);
        R wgt = hist && g2 > R(0) ? clampv(dot(acc, g) / g2, R(0), R(1)) : R(0);
        if (!std::isfinite(double(wgt))) wgt = 0;
        V3<R> corr = mul(g, -(R(1) - wgt) * dt * dt);
        bd.dx.v[0] = corr.x;
        bd.dx.v[1] = corr.y;
        bd.dx.v[2] = corr.z;
        bd.prev_velocity = prev[i].v;
        bd.history = 1;
        R mass = R(1) / mx(R(w.body[i].inv_mass), R(1.0e-12));
        for (unsigned ax = 0; ax < 3; ++ax) {
            bd.inertia.h[bidx(ax, ax)] = mass / (dt * dt);
            V3<R> la = inv_rotate(pred[i].q, unit_axis<R>(ax));
            V3<R> col = rotate(pred[i].q, V3<R>{la.x / mx(R(w.body[i].inv_inertia[0]), R(1.0e-12)),
                                                la.y / mx(R(w.body[i].inv_inertia[1]), R(1.0e-12)),
                                                la.z / mx(R(w.body[i].inv_inertia[2]), R(1.0e-12))});
            for (unsigned r = ax; r < 3; ++r) bd.inertia.h[bidx(3 + r, 3 + ax)] = comp(col, r) / (dt * dt);
        }
        bodies[i] = bd;
    }
    std::vector<bool> pair_impact(P);
    for (uint32_t k = 0; k < P; ++k) {
        uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
        R penalty = pair_stiffness<R>(w.body[a], w.body[b], dt);
        Manifold<R>& m = w.manifolds[k];
        for (uint32_t p = 0; p < m.count; ++p) {
            Contact<R>& c = m.c[p];
            if (c.cached == 0) {
                c.anchor_a = inv_rotate(prev[a].q, sub(c.point, prev[a].x));
                c.anchor_b = inv_rotate(prev[b].q, sub(c.point, prev[b].x));
            }
            V3<R> mo_a = sub(pred[a].x, prev[a].x), mo_b = sub(pred[b].x, prev[b].x);
            V3<R> an_a = mul(delta_velocity(prev[a].q, pred[a].q, dt), dt);
            V3<R> an_b = mul(delta_velocity(prev[b].q, pred[b].q, dt), dt);
            V3<R> arm_a = sub(c.point, pred[a].x), arm_b = sub(c.point, pred[b].x);
            R closing = dot(c.normal, sub(add(mo_b, cross(an_b, arm_b)), add(mo_a, cross(an_a, arm_a))));
            R old_pen = c.penetration - closing;
            V3<R> t0, t1;
            basis(c.normal, t0, t1);
            V3<R> anchor_motion = add(sub(mo_b, mo_a), sub(rotation_displacement(prev[b].q, pred[b].q, c.anchor_b),
                                                           rotation_displacement(prev[a].q, pred[a].q, c.anchor_a)));
            V3<R> old_delta = c.cached == 0 ? V3<R>{}
                                            : add(sub(prev[b].x, prev[a].x),
                                                  sub(rotate(prev[b].q, c.anchor_b), rotate(prev[a].q, c.anchor_a)));
            V3<R> terr = add(anchor_motion, mul(old_delta, R(1) - K<R>::alpha));
            c.init_speed = -closing / dt;
            R skin = contact_skin<R>(w.body[a], w.body[b], m.guided);
            R impact_disp = realtime && c.cached == 0 && c.init_speed < R(-0.1)
                                ? -(R(1) + mn(R(w.body[a].restitution), R(w.body[b].restitution))) * c.init_speed * dt
                                : R(0);
            c.error = {c.penetration - clampv(old_pen, R(0), skin) + impact_disp, dot(terr, t0), dot(terr, t1)};
            for (unsigned x = 0; x < 3; ++x) {
                Dual<R> d = c.dual[x];
                if (c.cached == 0) d = {R(0), penalty};
                c.dual[x] = warm_start(d, K<R>::kmax);
            }
        }
        pair_impact[k] = contact_impact(m, w.body[a], w.body[b], dt);
    }
    Block<R> scratch{};
    for (auto& j : w.joints) {
        j.count = 0;
        if (!j.alive) continue;
        j.enabled = j.d.enabled != 0 && j.broken == 0;
        if (!j.enabled) continue;
        j.applied = 0;
        j.dense_a = j.d.body_a < n ? j.d.body_a : kInvalid;
        j.dense_b = j.d.body_b < n ? j.d.body_b : kInvalid;
        if (j.dense_a != kInvalid && j.dense_b != kInvalid) {
            scratch = Block<R>{};
            visit_joint(j, w, prev, bodies, dt, scratch, true, kInit);
        }
    }
    // Lane-0 graph pass (geometry_constraints.slang:1433-1560).
    uint32_t budget = realtime ? 8u : (o.requested_iterations != 0 ? o.requested_iterations : o.base_iterations);
    auto unite = [&](uint32_t a, uint32_t b) {
        if (!dynamic(w, a) || !dynamic(w, b)) return;
        a = find_root(bodies, a);
        b = find_root(bodies, b);
        if (a != b) bodies[std::max(a, b)].parent = std::min(a, b);
    };
    st.contacts = 0;
    for (uint32_t k = 0; k < P; ++k) {
        st.contacts += w.manifolds[k].count;
        uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
        unite(a, b);
        w.manifolds[k].next_a = bodies[a].contact_head;
        bodies[a].contact_head = k;
        w.manifolds[k].next_b = bodies[b].contact_head;
        bodies[b].contact_head = k;
    }
    for (uint32_t ji = 0; ji < w.joints.size(); ++ji) {
        JointRt<R>& j = w.joints[ji];
        if (j.count == 0) continue;
        if (!realtime && o.requested_iterations == 0) budget = std::max(budget, j.d.solver_iterations);
        unite(j.dense_a, j.dense_b);
        j.next_a = bodies[j.dense_a].joint_head;
        bodies[j.dense_a].joint_head = ji;
        j.next_b = bodies[j.dense_b].joint_head;
        bodies[j.dense_b].joint_head = ji;
    }
    for (uint32_t i = 0; i < n; ++i) bodies[i].parent = find_root(bodies, i);
    bool any_impact = false;
    for (uint32_t k = 0; k < P; ++k) {
        if (!pair_impact[k]) continue;
        uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
        if (dynamic(w, a)) bodies[bodies[a].parent].impact = 1;
        if (dynamic(w, b)) bodies[bodies[b].parent].impact = 1;
        any_impact = true;
    }
    st.islands = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (!dynamic(w, i)) continue;
        bodies[i].impact = bodies[bodies[i].parent].impact;
        if (bodies[i].parent == i && (bodies[i].contact_head != kInvalid || bodies[i].joint_head != kInvalid))
            ++st.islands;
    }
    uint32_t remaining = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (!dynamic(w, i)) continue;
        uint32_t color = 0;
        for (;; ++color) {
            bool conflict = false;
            for (uint32_t k = bodies[i].contact_head; k != kInvalid;) {
                uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
                bool first = i == a;
                conflict = conflict || bodies[first ? b : a].color == color;
                k = first ? w.manifolds[k].next_a : w.manifolds[k].next_b;
            }
            for (uint32_t ji = bodies[i].joint_head; ji != kInvalid;) {
                const JointRt<R>& j = w.joints[ji];
                bool first = i == j.dense_a;
                conflict = conflict || bodies[first ? j.dense_b : j.dense_a].color == color;
                ji = first ? j.next_a : j.next_b;
            }
            if (!conflict) break;
        }
        bodies[i].color = color;
        remaining = std::max(remaining, color + 1);
    }
    st.colors = remaining;
    st.impact = any_impact ? 1u : 0u;

    // ---- solve (geometry_constraints_solve.slang:211-847)
    const bool adaptive = o.residual_tolerance > 0.0f;
    const uint32_t max_it = adaptive ? std::max(1u, o.max_iterations) : budget;
    w.residual_trace.clear();
    uint32_t phase_count = realtime ? 1u : 2u;
    uint32_t used_iterations = 0;
    for (uint32_t phase = 0; phase < phase_count; ++phase) {
        if (phase != 0 && !any_impact) break;
        if (phase != 0) {
            // impact_gaps (:238-262)
            for (uint32_t k = 0; k < P; ++k) {
                uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
                if (bodies[a].impact == 0 && bodies[b].impact == 0) continue;
                Manifold<R>& m = w.manifolds[k];
                for (uint32_t p = 0; p < m.count; ++p) {
                    Vec6<R> ja, jb;
                    Contact<R>& c = m.c[p];
                    Contact<R> tmp = c;
                    tmp.error.x = R(0);
                    contact_normal_row(tmp, bodies[a], bodies[b], ja, jb);
                    c.error.x = mx(R(0), -(c.penetration + dot6(ja, bodies[a].dx) + dot6(jb, bodies[b].dx)));
                }
            }
            // impact_bodies (:263-276)
            for (uint32_t i = 0; i < n; ++i) {
                if (bodies[i].impact != 0 || !dynamic(w, i)) {
                    bodies[i].target = pred[i];
                    bodies[i].dx = Vec6<R>{};
                    bodies[i].dq = {0, 0, 0, 1};
                }
            }
            // impact_constraints (:277-330)
            for (auto& j : w.joints) {
                if (j.count == 0 || !j.enabled) continue;
                if (bodies[j.dense_a].impact == 0 && bodies[j.dense_b].impact == 0) continue;
                scratch = Block<R>{};
                visit_joint(j, w, prev, bodies, dt, scratch, true, kImpact);
            }
            for (uint32_t k = 0; k < P; ++k) {
                uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
                if (bodies[a].impact == 0 && bodies[b].impact == 0) continue;
                Vec6<R> va = jac(mul(pred[a].v, dt), mul(pred[a].w, dt));
                Vec6<R> vb = jac(mul(pred[b].v, dt), mul(pred[b].w, dt));
                Manifold<R>& m = w.manifolds[k];
                for (uint32_t p = 0; p < m.count; ++p) {
                    Contact<R>& c = m.c[p];
                    R gap = c.error.x;
                    Vec6<R> ja[3], jb[3];
                    R err[3];
                    contact_rows(c, bodies[a], bodies[b], ja, jb, err);
                    R rest = c.cached == 0 && c.init_speed < R(-1)
                                 ? mn(R(w.body[a].restitution), R(w.body[b].restitution))
                                 : R(0);
                    c.error = {dot6(ja[0], va) + dot6(jb[0], vb) - gap - rest * c.init_speed * dt,
                               dot6(ja[1], va) + dot6(jb[1], vb), dot6(ja[2], va) + dot6(jb[2], vb)};
                }
            }
        }
        const uint32_t iters = phase == 0 ? max_it : budget;
        for (uint32_t it = 0; it < iters; ++it) {
            for (uint32_t color = 0; color < remaining; ++color) {
                for (uint32_t i = 0; i < n; ++i) {
                    if (bodies[i].color != color) continue;
                    if (phase != 0 && bodies[i].impact == 0) continue;
                    AvbdBody<R>& B = bodies[i];
                    Block<R> blk = B.inertia;
                    for (unsigned r = 0; r < 6; ++r)
                        for (unsigned c = 0; c < 6; ++c) blk.g[r] += blk.h[bidx(r, c)] * B.dx.v[c];
                    for (uint32_t k = B.contact_head; k != kInvalid;) {
                        uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
                        bool first = i == a;
                        R friction = std::sqrt(R(w.body[a].friction) * R(w.body[b].friction));
                        const Manifold<R>& m = w.manifolds[k];
                        for (uint32_t p = 0; p < m.count; ++p) {
                            const Contact<R>& c = m.c[p];
                            Vec6<R> ja[3], jb[3];
                            R err[3];
                            contact_rows(c, bodies[a], bodies[b], ja, jb, err);
                            Force3<R> trial{c.dual[0].lambda + c.dual[0].penalty * err[0],
                                            c.dual[1].lambda + c.dual[1].penalty * err[1],
                                            c.dual[2].lambda + c.dual[2].penalty * err[2]};
                            Force3<R> f = project_contact(trial, friction);
                            Force3<R> s = stiffness_scales(trial, friction);
                            R stiff[3] = {s.n, s.t0, s.t1};
                            V3<R> t0, t1;
                            basis(c.normal, t0, t1);
                            R forces[3] = {f.n - (phase != 0 ? c.acc_n / dt : R(0)),
                                           f.t0 - (phase != 0 ? dot(c.acc_f, t0) / dt : R(0)),
                                           f.t1 - (phase != 0 ? dot(c.acc_f, t1) / dt : R(0))};
                            for (unsigned x = 0; x < 3; ++x)
                                add_row(blk, first ? ja[x] : jb[x], c.dual[x].penalty * stiff[x], forces[x]);
                        }
                        k = first ? m.next_a : m.next_b;
                    }
                    for (uint32_t ji = B.joint_head; ji != kInvalid;) {
                        JointRt<R>& j = w.joints[ji];
                        bool first = i == j.dense_a;
                        if (j.enabled) {
                            if (phase == 0) {
                                visit_joint(j, w, prev, bodies, dt, blk, first, kAccumulate);
                            } else {
                                for (uint32_t r = 0; r < j.count; ++r)
                                    if (j.rows[r].stiffness >= K<R>::kmax)
                                        row_accumulate(blk, j.rows[r], first, bodies[j.dense_a].dx,
                                                       bodies[j.dense_b].dx, dt);
                            }
                        }
                        ji = first ? j.next_a : j.next_b;
                    }
                    Vec6<R> upd{};
                    if (block_solve(blk, upd)) {
                        bool crossing = false;
                        for (uint32_t k = B.contact_head; k != kInvalid;) {
                            uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
                            bool first = i == a;
                            const Manifold<R>& m = w.manifolds[k];
                            for (uint32_t p = 0; p < m.count; ++p) {
                                const Contact<R>& c = m.c[p];
                                Vec6<R> ja, jb;
                                R e = contact_normal_row(c, bodies[a], bodies[b], ja, jb);
                                const Vec6<R>& nr = first ? ja : jb;
                                R trial = c.dual[0].lambda + c.dual[0].penalty * e;
                                if (trial <= R(0) &&
                                    trial + c.dual[0].penalty * dot6(nr, upd) > c.dual[0].penalty * R(1.0e-6)) {
                                    add_row(blk, nr, c.dual[0].penalty, trial);
                                    crossing = true;
                                }
                            }
                            k = first ? m.next_a : m.next_b;
                        }
                        if (crossing) {
                            Vec6<R> safe{};
                            if (block_solve(blk, safe)) upd = safe;
                        }
                        if (phase == 0) {
                            apply_pose_update(B, upd);
                        } else {
                            for (unsigned x = 0; x < 6; ++x) B.dx.v[x] += upd.v[x];
                        }
                    }
                }
            }
            // advance_duals (:492-616). The reference's last-iteration block
            // (impulses, sliding re-anchoring) runs after the loop from the
            // final duals and stick flags, which is the same arithmetic.
            w.res_sq = 0;
            w.res_n = 0;
            w.res_max = 0;
            w.res_over = 0;
            w.res_tol = R(o.residual_tolerance);
            for (uint32_t k = 0; k < P; ++k) {
                uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
                if (phase != 0 && bodies[a].impact == 0 && bodies[b].impact == 0) continue;
                R friction = std::sqrt(R(w.body[a].friction) * R(w.body[b].friction));
                R beta = pair_stiffness<R>(w.body[a], w.body[b], dt) * R(100);
                Manifold<R>& m = w.manifolds[k];
                for (uint32_t p = 0; p < m.count; ++p) {
                    Contact<R>& c = m.c[p];
                    Vec6<R> ja[3], jb[3];
                    R err[3];
                    contact_rows(c, bodies[a], bodies[b], ja, jb, err);
                    Force3<R> f = project_contact(Force3<R>{c.dual[0].lambda + c.dual[0].penalty * err[0],
                                                            c.dual[1].lambda + c.dual[1].penalty * err[1],
                                                            c.dual[2].lambda + c.dual[2].penalty * err[2]},
                                                  friction);
                    R tx = c.dual[1].lambda + c.dual[1].penalty * err[1];
                    R ty = c.dual[2].lambda + c.dual[2].penalty * err[2];
                    R bound = friction * f.n;
                    bool stick = tx * tx + ty * ty <= bound * bound;
                    bool active = false;
                    R rv = contact_row_residual(err[0], f.n, active);
                    if (active) w.residual_add(rv);
                    c.dual[0].lambda = f.n;
                    c.dual[1].lambda = f.t0;
                    c.dual[2].lambda = f.t1;
                    for (unsigned x = 0; x < 3; ++x)
                        if (x == 0 ? f.n > R(0) : stick)
                            c.dual[x].penalty = mn(K<R>::kmax, c.dual[x].penalty + beta * ab(err[x]));
                    c.stick = stick ? 1u : 0u;
                }
            }
            for (auto& j : w.joints) {
                if (j.count == 0 || !j.enabled) continue;
                uint32_t a = j.dense_a, b = j.dense_b;
                if (phase != 0 && bodies[a].impact == 0 && bodies[b].impact == 0) continue;
                R impulse = 0;
                if (phase == 0) {
                    scratch = Block<R>{};
                    j.residual_sink = [](void* ctx, R v) { static_cast<World<R>*>(ctx)->residual_add(v); };
                    j.residual_ctx = &w;
                    impulse = visit_joint(j, w, prev, bodies, dt, scratch, true, kAdvance);
                    j.residual_sink = nullptr;
                } else {
                    for (uint32_t r = 0; r < j.count; ++r) {
                        Row<R> row = j.rows[r];
                        impulse += ab(row.stiffness < K<R>::kmax ? row.reference_force
                                                                 : row_force(row, bodies[a].dx, bodies[b].dx, dt)) *
                                   dt;
                        if (row.stiffness >= K<R>::kmax) j.rows[r] = row_advance(row, bodies[a].dx, bodies[b].dx);
                    }
                }
                j.applied = impulse;
                if (j.d.breaking_threshold > 0.0f && impulse > R(j.d.breaking_threshold)) {
                    j.broken = 1;
                    j.enabled = 0;
                }
            }
            bool last = it + 1 == iters;
            if (phase == 0) {
                const R rms = w.res_n ? R(std::sqrt(w.res_sq / double(w.res_n))) : R(0);
                w.residual_rms_last = rms;
                w.residual_max_last = w.res_max;
                w.residual_over_last = w.res_n ? float(w.res_over) / float(w.res_n) : 0.0f;
                // The schedule's measure: the largest row violation (every
                // constraint within the tolerance), the RMS over the rows, or
                // the 99.9th percentile (at most one row in a thousand above).
                bool met;
                R res;
                if (o.residual_norm == 1) {
                    res = rms;
                    met = rms <= R(o.residual_tolerance);
                } else if (o.residual_norm == 2) {
                    res = R(w.residual_over_last);
                    met = w.res_over * 1000u <= w.res_n;
                } else {
                    res = w.res_max;
                    met = w.res_max <= R(o.residual_tolerance);
                }
                w.residual_trace.push_back(res);
                if (adaptive && met) last = true;
                used_iterations = it + 1;
            }
            if (last) break;
        }
        // Last-iteration contact work (:533-561).
        for (uint32_t k = 0; k < P; ++k) {
            uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
            if (phase != 0 && bodies[a].impact == 0 && bodies[b].impact == 0) continue;
            Manifold<R>& m = w.manifolds[k];
            for (uint32_t p = 0; p < m.count; ++p) {
                Contact<R>& c = m.c[p];
                V3<R> t0, t1;
                basis(c.normal, t0, t1);
                c.acc_n = c.dual[0].lambda * dt;
                c.rep_n = c.acc_n;
                c.acc_f = mul(add(mul(t0, c.dual[1].lambda), mul(t1, c.dual[2].lambda)), dt);
                c.rep_f = c.acc_f;
                if (!c.stick) {
                    State<R> pa = phase != 0 ? bodies[a].target : pose(bodies[a]);
                    State<R> pb = phase != 0 ? bodies[b].target : pose(bodies[b]);
                    c.anchor_a = inv_rotate(pa.q, sub(c.point, pa.x));
                    c.anchor_b = inv_rotate(pb.q, sub(c.point, pb.x));
                }
            }
        }
        if (phase == 0 && adaptive) budget = used_iterations;
        // free_mean / free_subtract / free_clear (:617-698)
        const bool vphase = phase != 0;
        for (uint32_t r = 0; r < n; ++r) {
            if (!dynamic(w, r) || bodies[r].parent != r) continue;
            for (unsigned x = 0; x < 3; ++x) bodies[r].inertia.g[x] = 0;
            if ((vphase && bodies[r].impact == 0) ||
                (bodies[r].contact_head == kInvalid && bodies[r].joint_head == kInvalid))
                continue;
            V3<R> weighted{};
            R total = 0;
            bool anchored = false;
            for (uint32_t i = 0; i < n && !anchored; ++i) {
                if (!dynamic(w, i) || bodies[i].parent != r) continue;
                R mass = R(1) / mx(R(w.body[i].inv_mass), R(1.0e-12));
                weighted = add(weighted, mul(V3<R>{bodies[i].dx.v[0], bodies[i].dx.v[1], bodies[i].dx.v[2]}, mass));
                total += mass;
                for (uint32_t k = bodies[i].contact_head; k != kInvalid;) {
                    uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
                    bool first = i == a;
                    anchored = anchored || !dynamic(w, first ? b : a);
                    k = first ? w.manifolds[k].next_a : w.manifolds[k].next_b;
                }
                for (uint32_t ji = bodies[i].joint_head; ji != kInvalid;) {
                    const JointRt<R>& j = w.joints[ji];
                    bool first = i == j.dense_a;
                    anchored = anchored || !dynamic(w, first ? j.dense_b : j.dense_a);
                    ji = first ? j.next_a : j.next_b;
                }
            }
            if (!anchored && total > R(0)) {
                weighted = mul(weighted, R(1) / total);
                bodies[r].inertia.g[0] = weighted.x;
                bodies[r].inertia.g[1] = weighted.y;
                bodies[r].inertia.g[2] = weighted.z;
            }
        }
        for (uint32_t i = 0; i < n; ++i) {
            if (!dynamic(w, i) || (vphase && bodies[i].impact == 0)) continue;
            const Block<R>& mean = bodies[bodies[i].parent].inertia;
            for (unsigned x = 0; x < 3; ++x) bodies[i].dx.v[x] -= mean.g[x];
        }
        for (uint32_t i = 0; i < n; ++i)
            for (unsigned x = 0; x < 3; ++x) bodies[i].inertia.g[x] = 0;
        // apply_states (:699-733)
        for (uint32_t i = 0; i < n; ++i) {
            if (!dynamic(w, i)) continue;
            if (phase != 0 && bodies[i].impact == 0) continue;
            State<R> s = bodies[i].target;
            const Vec6<R>& d = bodies[i].dx;
            V3<R> lin{d.v[0], d.v[1], d.v[2]}, rot{d.v[3], d.v[4], d.v[5]};
            if (phase != 0) {
                s.v = add(s.v, mul(lin, R(1) / dt));
                s.w = add(s.w, mul(rot, R(1) / dt));
                pred[i] = s;
                continue;
            }
            s.x = add(s.x, lin);
            s.q = pose(bodies[i]).q;
            s.v = add(s.v, mul(lin, R(1) / dt));
            s.w = add(s.w, mul(rotation_vector(bodies[i].dq), R(1) / dt));
            if (realtime) {
                s.v = mul(s.v, R(1) - R(0.05));
                s.w = mul(s.w, R(1) - R(0.05));
            }
            pred[i] = s;
        }
        // project_hinges (:174-209), phase 0 only
        if (phase == 0) {
            for (auto& j : w.joints) {
                if (j.count == 0 || !j.enabled || j.d.type != kHinge) continue;
                uint32_t a = j.dense_a, b = j.dense_b;
                R ima = dynamic(w, a) ? R(w.body[a].inv_mass) : R(0);
                R imb = dynamic(w, b) ? R(w.body[b].inv_mass) : R(0);
                R sum = ima + imb;
                if (sum <= kEps<R>()) continue;
                V3<R> pa = add(pred[a].x, rotate(pred[a].q, v3<R>(j.d.anchor_a)));
                V3<R> pb = add(pred[b].x, rotate(pred[b].q, v3<R>(j.d.anchor_b)));
                V3<R> e = sub(pb, pa);
                pred[a].x = add(pred[a].x, mul(e, ima / sum));
                pred[b].x = sub(pred[b].x, mul(e, imb / sum));
            }
        }
    }
    st.iterations = used_iterations;
    st.residual = w.residual_trace.empty() ? 0.0f : float(w.residual_rms_last);
    st.residual_max = float(w.residual_max_last);
    st.residual_over = w.residual_over_last;

    // ---- speed clamp (geometry.slang:3086-3100)
    for (uint32_t i = 0; i < n; ++i) {
        if (!dynamic(w, i)) continue;
        pred[i].v = clamp_length(pred[i].v, R(w.body[i].max_linear_speed));
        pred[i].w = clamp_length(pred[i].w, R(w.body[i].max_angular_speed));
    }

    // ---- contact cache save (geometry.slang:3011-3070)
    std::vector<SavedPair<R>> saved;
    saved.reserve(P);
    for (uint32_t k = 0; k < P; ++k) {
        const uint64_t code = w.active_pairs[k];
        const uint32_t a = uint32_t(code / n);
        const Manifold<R>& m = w.manifolds[k];
        SavedPair<R> sp{};
        sp.pair = code;
        sp.epoch = epoch;
        sp.dt = dt;
        sp.count = m.count;
        for (uint32_t p = 0; p < m.count; ++p) {
            const Contact<R>& c = m.c[p];
            sp.c[p].local = inv_rotate(pred[a].q, sub(c.point, pred[a].x));
            sp.c[p].normal = c.normal;
            sp.c[p].normal_impulse = c.acc_n;
            sp.c[p].friction_impulse = c.acc_f;
            for (unsigned x = 0; x < 3; ++x) sp.c[p].dual[x] = c.dual[x];
            sp.c[p].anchor_a = c.anchor_a;
            sp.c[p].anchor_b = c.anchor_b;
        }
        saved.push_back(sp);
    }
    w.saved.swap(saved);
    w.state = pred;
    w.epoch = epoch;
    // pm_clear_rigid_inputs (geometry.slang:2877-2886): inputs and targets
    // last one tick.
    for (uint32_t i = 0; i < n; ++i) {
        w.force[i] = w.torque[i] = w.impulse[i] = w.angular_impulse[i] = V3<R>{};
        w.target_set[i] = 0;
    }
    w.stats = st;
}

}  // namespace oracle

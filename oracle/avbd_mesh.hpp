// SPDX-License-Identifier: MIT
// Oracle (test infrastructure): the general triangle-mesh narrowphase of the
// reference, restated for pairs the convex face path does not take.
//
// Reference: src/slang/geometry.slang
//   hinge contact frames            :373-377, :404-492
//   closest points (Ericson)        :949-1105, bounds overlap :1107-1116
//   contact speed / rest offset     :1272-1290
//   shell metadata                  :1308-1357
//   triangle ranges                 :1359-1584
//   swept-pair test                 :1586-1604
//   feature normal                  :1855-1908
//   BVH pair traversal              :2156-2299 (rigid_collide_meshes)
//   bounds transforms               src/slang/math.slang:43-49, :142-190
//   swept triangle ranges           :1921-2155
//   guided contacts                 :1118-1127 (guide direction), :1129-1170
// What is restated: the BVH traversal of rigid_collide_meshes with the
// unswept triangle ranges and, for a pair that moved more than its
// threshold (or a guided pair: a body on an unbreakable slider or piston to
// a static body, against a static body), the swept ranges (conservative
// advancement) after them at each leaf pair, guided contacts merged by guide
// direction; the per-body hinge frames those ranges read.
#pragma once
#include <vector>

#include "avbd_world.hpp"

namespace oracle {

// The fields of HingeContactFrame (geometry.slang:143-157) the unswept ranges
// read, and the body's reference point (the hinge anchor of a non-axial
// hinge member, else its position).
template <class R> struct HingeFrame {
    V3<R> anchor, reference, axis;
    R inv_mass{}, inv_moment{};
    bool present{}, fixed{}, axial{}, axial_rotation{}, fixed_member{}, static_body{};
};

// geometry.slang:384-402: the inverse moment of a body turning about its
// guide axis through the anchor (pistons; zero otherwise).
template <class R> inline R fixed_hinge_inverse_moment(const BodyDesc& b, const State<R>& s, const HingeFrame<R>& f) {
    if ((!f.fixed && !f.axial_rotation) || !(R(b.inv_mass) > kEps<R>())) return R(0);
    const V3<R> l = inv_rotate(s.q, f.axis);
    const R center = l.x * l.x / mx(R(b.inv_inertia[0]), kEps<R>()) + l.y * l.y / mx(R(b.inv_inertia[1]), kEps<R>()) +
                     l.z * l.z / mx(R(b.inv_inertia[2]), kEps<R>());
    const V3<R> arm = sub(s.x, f.anchor);
    const V3<R> perp = sub(arm, mul(f.axis, dot(arm, f.axis)));
    const R pivot = center + len2(perp) / R(b.inv_mass);
    return pivot > kEps<R>() ? R(1) / pivot : R(0);
}

// geometry.slang:404-492. `joints_of_body`: the body's joints in ascending
// index.
template <class R>
inline HingeFrame<R> hinge_frame(const World<R>& w, const std::vector<State<R>>& st, uint32_t i,
                                 const std::vector<uint32_t>& joints_of_body) {
    HingeFrame<R> f;
    f.static_body = w.body[i].motion == kStatic;
    if (!(w.body[i].inv_mass > 0.0f)) {
        f.reference = st[i].x;
        return f;
    }
    uint32_t incident = 0;
    for (uint32_t ji : joints_of_body) {
        const auto& j = w.joints[ji];
        if (!j.alive || !j.d.enabled || j.broken) continue;
        const bool is_a = j.d.body_a == i, is_b = j.d.body_b == i;
        if (!is_a && !is_b) continue;
        ++incident;
        if (j.d.type == kFixed) f.fixed_member = true;
        const bool axial = j.d.type == kPiston || j.d.type == kSlider;
        const uint32_t other = is_a ? j.d.body_b : j.d.body_a;
        const bool static_anchor = other < w.n && w.body[other].motion == kStatic;
        if (f.present || (j.d.type != kHinge && !(axial && static_anchor && !(j.d.breaking_threshold > 0.0f))))
            continue;
        const V3<R> local_axis = axial ? V3<R>{1, 0, 0} : V3<R>{0, 0, 1};
        const float* la = is_a ? j.d.anchor_a : j.d.anchor_b;
        const Q4<R> lq = q4<R>(is_a ? j.d.frame_a : j.d.frame_b);
        f.anchor = add(st[i].x, rotate(st[i].q, v3<R>(la)));
        f.axis = normalized_or(rotate(qmul(st[i].q, lq), local_axis), local_axis);
        f.present = true;
        f.fixed = static_anchor && !axial;
        f.axial = static_anchor && axial;
        f.axial_rotation = f.axial && j.d.type == kPiston;
        if (static_anchor) {
            const float* lo = is_a ? j.d.anchor_b : j.d.anchor_a;
            const Q4<R> oq = q4<R>(is_a ? j.d.frame_b : j.d.frame_a);
            f.anchor = add(st[other].x, rotate(st[other].q, v3<R>(lo)));
            f.axis = normalized_or(rotate(qmul(st[other].q, oq), local_axis), f.axis);
        }
    }
    if (f.axial && incident != 1u) {
        f.axial = false;
        f.axial_rotation = false;
        f.present = false;
    }
    if (f.axial) {
        f.inv_mass = R(w.body[i].inv_mass);
        f.inv_moment = fixed_hinge_inverse_moment(w.body[i], st[i], f);
    }
    f.reference = f.present && !f.axial ? f.anchor : st[i].x;
    return f;
}

// Every body's frame at the given poses.
template <class R> inline std::vector<HingeFrame<R>> hinge_frames(const World<R>& w, const std::vector<State<R>>& st) {
    std::vector<std::vector<uint32_t>> by_body(w.n);
    for (uint32_t j = 0; j < w.joints.size(); ++j) {
        const auto& d = w.joints[j].d;
        if (d.body_a < w.n) by_body[d.body_a].push_back(j);
        if (d.body_b < w.n && d.body_b != d.body_a) by_body[d.body_b].push_back(j);
    }
    std::vector<HingeFrame<R>> out(w.n);
    for (uint32_t i = 0; i < w.n; ++i) out[i] = hinge_frame(w, st, i, by_body[i]);
    return out;
}

// geometry.slang:373-377
template <class R> inline bool guided_pair(const HingeFrame<R>& a, const HingeFrame<R>& b) {
    return (a.axial && b.static_body) || (b.axial && a.static_body);
}

// geometry.slang:1118-1127: a guided contact's direction in the guide's
// (translation, rotation) coordinates, scaled by the guide's inverse mass
// and moment.
template <class R> inline V3<R> guide_direction(V3<R> n, V3<R> p, const HingeFrame<R>& g) {
    return {dot(n, g.axis) * std::sqrt(g.inv_mass),
            g.axial_rotation ? dot(g.axis, cross(sub(p, g.anchor), n)) * std::sqrt(g.inv_moment) : R(0), R(0)};
}

// geometry.slang:1129-1170, the guided merge: a contact whose guide
// direction is too weak is dropped; among impacts only the earliest
// (within 1e-4 of the tick) are kept; a contact with the direction of a kept
// one replaces it when deeper per unit direction; else it is added (a ninth
// replaces the shallowest).
template <class R> inline void add_guided_contact(Manifold<R>& m, const Contact<R>& c, const HingeFrame<R>& g) {
    const V3<R> cd = guide_direction(c.normal, c.point, g);
    const R cl = len(cd);
    if (cl * cl <= kEps<R>()) return;
    if (c.impact_fraction > R(0)) {
        R first = R(1);
        for (uint32_t i = 0; i < m.count; ++i)
            if (m.c[i].impact_fraction > R(0)) first = mn(first, m.c[i].impact_fraction);
        if (c.impact_fraction > first + R(1.0e-4)) return;
        if (c.impact_fraction < first - R(1.0e-4)) {
            uint32_t kept = 0;
            for (uint32_t i = 0; i < m.count; ++i)
                if (m.c[i].impact_fraction == R(0)) m.c[kept++] = m.c[i];
            m.count = kept;
        }
    }
    for (uint32_t i = 0; i < m.count; ++i) {
        const V3<R> d = guide_direction(m.c[i].normal, m.c[i].point, g);
        const R size = len(d);
        if (dot(cd, d) > R(0.9999) * cl * size) {
            if (c.penetration / cl > m.c[i].penetration / size) m.c[i] = c;
            return;
        }
    }
    if (m.count < 8) {
        m.c[m.count++] = c;
        return;
    }
    uint32_t sh = 0;
    for (uint32_t i = 1; i < m.count; ++i)
        if (m.c[i].penetration < m.c[sh].penetration) sh = i;
    if (c.penetration > m.c[sh].penetration) m.c[sh] = c;
}

// geometry.slang:1910-1919
template <class R> inline bool triangle_pair_face_contact(const V3<R> a[3], const V3<R> b[3], V3<R> sep) {
    const V3<R> n = normalized_or(sep, V3<R>{});
    const V3<R> fa = normalized_or(cross(sub(a[1], a[0]), sub(a[2], a[0])), V3<R>{});
    const V3<R> fb = normalized_or(cross(sub(b[1], b[0]), sub(b[2], b[0])), V3<R>{});
    return ab(dot(n, fa)) > R(0.9999) || ab(dot(n, fb)) > R(0.9999);
}

// geometry.slang:949-997
template <class R> inline void closest_segments(V3<R> p0, V3<R> p1, V3<R> q0, V3<R> q1, V3<R>& on_p, V3<R>& on_q) {
    const V3<R> d0 = sub(p1, p0), d1 = sub(q1, q0), r = sub(p0, q0);
    const R a = dot(d0, d0), e = dot(d1, d1);
    R s = 0, t = 0;
    if (a <= R(1.0e-12) && e <= R(1.0e-12)) {
        on_p = p0;
        on_q = q0;
        return;
    }
    if (a <= R(1.0e-12)) {
        t = clampv(dot(d1, r) / e, R(0), R(1));
    } else {
        const R c = dot(d0, r);
        if (e <= R(1.0e-12)) {
            s = clampv(-c / a, R(0), R(1));
        } else {
            const R b = dot(d0, d1), f = dot(d1, r);
            const R den = a * e - b * b;
            if (ab(den) > kEps<R>() * a * e) s = clampv((b * f - c * e) / den, R(0), R(1));
            t = (b * s + f) / e;
            if (t < R(0)) {
                t = 0;
                s = clampv(-c / a, R(0), R(1));
            } else if (t > R(1)) {
                t = 1;
                s = clampv((b - c) / a, R(0), R(1));
            }
        }
    }
    on_p = add(p0, mul(d0, s));
    on_q = add(q0, mul(d1, t));
}

// geometry.slang:1000-1031 (Voronoi regions of a triangle; the interior
// witness is the plane projection of p)
template <class R> inline V3<R> closest_on_triangle(V3<R> p, V3<R> a, V3<R> b, V3<R> c) {
    const V3<R> ab_ = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    const R d1 = dot(ab_, ap), d2 = dot(ac, ap);
    if (d1 <= R(0) && d2 <= R(0)) return a;
    const V3<R> bp = sub(p, b);
    const R d3 = dot(ab_, bp), d4 = dot(ac, bp);
    if (d3 >= R(0) && d4 <= d3) return b;
    const R vc = d1 * d4 - d3 * d2;
    if (vc <= R(0) && d1 >= R(0) && d3 <= R(0)) return add(a, mul(ab_, d1 / (d1 - d3)));
    const V3<R> cp = sub(p, c);
    const R d5 = dot(ab_, cp), d6 = dot(ac, cp);
    if (d6 >= R(0) && d5 <= d6) return c;
    const R vb = d5 * d2 - d1 * d6;
    if (vb <= R(0) && d2 >= R(0) && d6 <= R(0)) return add(a, mul(ac, d2 / (d2 - d6)));
    const R va = d3 * d6 - d5 * d4;
    if (va <= R(0) && d4 - d3 >= R(0) && d5 - d6 >= R(0))
        return add(b, mul(sub(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6))));
    const V3<R> nrm = cross(ab_, ac);
    return sub(p, mul(nrm, dot(ap, nrm) / len2(nrm)));
}

// geometry.slang:1033-1055
template <class R> inline bool point_in_triangle(V3<R> p, V3<R> a, V3<R> b, V3<R> c, V3<R> nrm) {
    const R tol = R(-1.0e-5) * len2(nrm);
    return dot(cross(sub(b, a), sub(p, a)), nrm) >= tol && dot(cross(sub(c, b), sub(p, b)), nrm) >= tol &&
           dot(cross(sub(a, c), sub(p, c)), nrm) >= tol;
}
template <class R> inline bool segment_hits_triangle(V3<R> p, V3<R> q, V3<R> a, V3<R> b, V3<R> c, V3<R>& hit) {
    hit = V3<R>{};
    const V3<R> nrm = cross(sub(b, a), sub(c, a));
    const V3<R> dir = sub(q, p);
    const R den = dot(nrm, dir);
    if (len2(nrm) <= kEps<R>() * kEps<R>() || ab(den) <= kEps<R>()) return false;
    const R amount = dot(nrm, sub(a, p)) / den;
    if (amount < R(0) || amount > R(1)) return false;
    hit = add(p, mul(dir, amount));
    return point_in_triangle(hit, a, b, c, nrm);
}

// geometry.slang:1057-1105: an edge crossing the other triangle is a zero-
// distance witness; else the closest of vertex-face and edge-edge pairs.
template <class R>
inline void closest_triangle_pair(const V3<R> av[3], const V3<R> bv[3], V3<R>& best_a, V3<R>& best_b) {
    V3<R> hit{};
    for (uint32_t e = 0; e < 3; ++e)
        if (segment_hits_triangle(av[e], av[(e + 1) % 3], bv[0], bv[1], bv[2], hit)) {
            best_a = best_b = hit;
            return;
        }
    for (uint32_t e = 0; e < 3; ++e)
        if (segment_hits_triangle(bv[e], bv[(e + 1) % 3], av[0], av[1], av[2], hit)) {
            best_a = best_b = hit;
            return;
        }
    R best = R(3.402823466e38);
    auto consider = [&](V3<R> p, V3<R> q) {
        const R s = len2(sub(p, q));
        if (s < best) {
            best = s;
            best_a = p;
            best_b = q;
        }
    };
    for (uint32_t i = 0; i < 3; ++i) consider(av[i], closest_on_triangle(av[i], bv[0], bv[1], bv[2]));
    for (uint32_t i = 0; i < 3; ++i) consider(closest_on_triangle(bv[i], av[0], av[1], av[2]), bv[i]);
    for (uint32_t i = 0; i < 3; ++i)
        for (uint32_t j = 0; j < 3; ++j) {
            V3<R> on_a, on_b;
            closest_segments(av[i], av[(i + 1) % 3], bv[j], bv[(j + 1) % 3], on_a, on_b);
            consider(on_a, on_b);
        }
}

// math.slang:43-49
template <class R> inline bool bounds_overlap(V3<R> alo, V3<R> ahi, V3<R> blo, V3<R> bhi) {
    return alo.x <= bhi.x && ahi.x >= blo.x && alo.y <= bhi.y && ahi.y >= blo.y && alo.z <= bhi.z && ahi.z >= blo.z;
}

// geometry.slang:1107-1116
template <class R> inline bool triangle_bounds_overlap(const V3<R> a[3], const V3<R> b[3], R margin) {
    const V3<R> ex{margin, margin, margin};
    const V3<R> alo = sub(vmin(a[0], vmin(a[1], a[2])), ex), ahi = add(vmax(a[0], vmax(a[1], a[2])), ex);
    const V3<R> blo = vmin(b[0], vmin(b[1], b[2])), bhi = vmax(b[0], vmax(b[1], b[2]));
    return bounds_overlap(alo, ahi, blo, bhi);
}

// math.slang:142-190: box bounds of a local AABB under a pose, grown by a
// margin, unioned with the previous pose's when swept.
template <class R> struct BoundsXf { V3<R> x, ax, ay, az; };
template <class R> inline BoundsXf<R> bounds_xf(const State<R>& s) {
    return {s.x, rotate(s.q, V3<R>{1, 0, 0}), rotate(s.q, V3<R>{0, 1, 0}), rotate(s.q, V3<R>{0, 0, 1})};
}
template <class R>
inline void xf_bounds(V3<R> llo, V3<R> lhi, const BoundsXf<R>& t, R margin, V3<R>& lo, V3<R>& hi) {
    const V3<R> c = mul(add(llo, lhi), R(0.5)), h = mul(sub(lhi, llo), R(0.5));
    const V3<R> wc = add(t.x, add(mul(t.ax, c.x), add(mul(t.ay, c.y), mul(t.az, c.z))));
    const V3<R> wh{ab(t.ax.x) * h.x + ab(t.ay.x) * h.y + ab(t.az.x) * h.z,
                   ab(t.ax.y) * h.x + ab(t.ay.y) * h.y + ab(t.az.y) * h.z,
                   ab(t.ax.z) * h.x + ab(t.ay.z) * h.y + ab(t.az.z) * h.z};
    const V3<R> ex{margin, margin, margin};
    lo = sub(sub(wc, wh), ex);
    hi = add(add(wc, wh), ex);
}
template <class R>
inline void motion_bounds(V3<R> llo, V3<R> lhi, const BoundsXf<R>& prev, const BoundsXf<R>& cur, bool swept, R margin,
                          V3<R>& lo, V3<R>& hi) {
    xf_bounds(llo, lhi, cur, margin, lo, hi);
    if (!swept) return;
    V3<R> plo, phi;
    xf_bounds(llo, lhi, prev, margin, plo, phi);
    lo = vmin(lo, plo);
    hi = vmax(hi, phi);
}

template <class R> inline V3<R> xf_point(const State<R>& s, V3<R> p) { return add(s.x, rotate(s.q, p)); }

// geometry.slang:1272-1290
template <class R> inline R normal_speed(const State<R>& a, const State<R>& b, V3<R> p, V3<R> n) {
    const V3<R> va = add(a.v, cross(a.w, sub(p, a.x)));
    const V3<R> vb = add(b.v, cross(b.w, sub(p, b.x)));
    return dot(sub(va, vb), n);
}
template <class R>
inline bool reaches_rest_offset(const State<R>& a, const State<R>& b, V3<R> p, V3<R> n, R dist, R rest, R dt) {
    if (dist <= rest + R(1.0e-5)) return true;
    const R speed = normal_speed(a, b, p, n);
    if (speed > R(1.0e-5)) return false;
    return -speed * dt + rest + R(1.0e-5) >= dist;
}

// geometry.slang:1292-1306
template <class R> inline V3<R> advect_triangle_point(V3<R> p, const V3<R> from[3], const V3<R> to[3]) {
    const V3<R> e1 = sub(from[1], from[0]), e2 = sub(from[2], from[0]);
    const V3<R> nrm = cross(e1, e2);
    const R sq = len2(nrm);
    if (sq <= R(1.0e-20)) return to[0];
    const V3<R> rel = sub(p, from[0]);
    const R v = dot(cross(rel, e2), nrm) / sq;
    const R w2 = dot(cross(e1, rel), nrm) / sq;
    return add(to[0], add(mul(sub(to[1], to[0]), v), mul(sub(to[2], to[0]), w2)));
}

// geometry.slang:1308-1322: the certified outward direction carried to the
// posed triangle (unit for a certified face, quarter length for an interior
// open-surface face, zero when uncertified).
template <class R> inline V3<R> shell_outward(const Mesh<R>& m, uint32_t t, V3<R> a, V3<R> b, V3<R> c) {
    if (m.shell.empty()) return {};
    const V3<R> out = m.shell[t];
    const R sq = len2(out);
    if (sq < R(0.01)) return {};
    const V3<R> la = m.verts[m.idx[3 * t]], lb = m.verts[m.idx[3 * t + 1]], lc = m.verts[m.idx[3 * t + 2]];
    const R sign = dot(cross(sub(lb, la), sub(lc, la)), out) >= R(0) ? R(1) : R(-1);
    return mul(normalized_or(cross(sub(b, a), sub(c, a)), V3<R>{}), sign * (sq > R(0.5) ? R(1) : R(0.25)));
}

// geometry.slang:1324-1337
template <class R> inline bool shell_contact_facing(V3<R> n, V3<R> oa, V3<R> ob) {
    const R sa = len2(oa), sb = len2(ob);
    return (sa < R(0.01) || (sa > R(0.5) ? dot(n, oa) < R(-1.0e-3) : ab(dot(n, oa)) > R(2.5e-4))) &&
           (sb < R(0.01) || (sb > R(0.5) ? dot(n, ob) > R(1.0e-3) : ab(dot(n, ob)) > R(2.5e-4)));
}

// geometry.slang:1339-1357 (every plane of a convex mesh; its deduplicated
// plane list gives the same answer)
template <class R> inline bool point_inside_convex(const Mesh<R>& m, const State<R>& s, V3<R> p) {
    if (!m.convex) return false;
    const V3<R> l = inv_rotate(s.q, sub(p, s.x));
    for (const auto& pl : m.planes)
        if (dot(pl.n, l) > pl.d + R(1.0e-5)) return false;
    return true;
}

// geometry.slang:1855-1908
template <class R>
inline V3<R> triangle_feature_normal(const V3<R> a[3], const V3<R> b[3], V3<R> pa, V3<R> pb, V3<R> fallback) {
    const V3<R> delta = sub(pa, pb);
    V3<R> nrm = normalized_or(delta, fallback);
    const V3<R> faces[2] = {normalized_or(cross(sub(a[1], a[0]), sub(a[2], a[0])), nrm),
                            normalized_or(cross(sub(b[1], b[0]), sub(b[2], b[0])), nrm)};
    const V3<R>* tri[2] = {a, b};
    const V3<R> pts[2] = {pa, pb};
    R align_best = R(-1);
    V3<R> interior_n{};
    for (uint32_t side = 0; side < 2; ++side) {
        const V3<R>* v = tri[side];
        const V3<R> raw = cross(sub(v[1], v[0]), sub(v[2], v[0]));
        const R tol = R(1.0e-5) * len2(raw);
        bool interior = tol > R(0);
        for (uint32_t e = 0; e < 3; ++e)
            interior = interior && dot(cross(sub(v[(e + 1) % 3], v[e]), sub(pts[side], v[e])), raw) > tol;
        const R align = ab(dot(faces[side], nrm));
        if (interior && align > align_best) {
            align_best = align;
            const R proj = dot(delta, faces[side]);
            const R dir = ab(proj) > kEps<R>() ? proj : dot(fallback, faces[side]);
            interior_n = dir >= R(0) ? faces[side] : mul(faces[side], R(-1));
        }
    }
    if (align_best >= R(0)) return interior_n;
    R best_err = R(4) * kEps<R>() * kEps<R>();
    if (len2(delta) > kEps<R>() * kEps<R>())
        for (uint32_t side = 0; side < 2; ++side) {
            const R proj = dot(delta, faces[side]);
            const R err = len2(sub(delta, mul(faces[side], proj)));
            if (err < best_err) {
                best_err = err;
                nrm = proj >= R(0) ? faces[side] : mul(faces[side], R(-1));
            }
        }
    return nrm;
}

// geometry.slang:1359-1584: contacts of triangle range [af, af+ac) of the
// body against [bf, bf+bc) of the collider at the current poses.
template <class R>
inline void collide_triangle_ranges(const Mesh<R>& am, const State<R>& aprev, const State<R>& as,
                                    const HingeFrame<R>& ah, uint32_t af, uint32_t ac, const Mesh<R>& bm,
                                    const State<R>& bprev, const State<R>& bs, const HingeFrame<R>& bh, uint32_t bf,
                                    uint32_t bc, R margin, R dt, Manifold<R>& out) {
    if (guided_pair(ah, bh)) return;
    const R rest = mn(margin, R(1.0e-3));
    const bool interior_a = ah.static_body && point_inside_convex(am, aprev, bprev.x);
    const bool interior_b = bh.static_body && point_inside_convex(bm, bprev, aprev.x);
    const uint32_t a_tris = uint32_t(am.idx.size() / 3), b_tris = uint32_t(bm.idx.size() / 3);
    for (uint32_t i = 0; i < ac; ++i) {
        const uint32_t at = af + i;
        if (at >= a_tris) break;
        V3<R> A[3];
        for (uint32_t k = 0; k < 3; ++k) A[k] = xf_point(as, am.verts[am.idx[3 * at + k]]);
        for (uint32_t j = 0; j < bc; ++j) {
            const uint32_t bt = bf + j;
            if (bt >= b_tris) break;
            V3<R> B[3];
            for (uint32_t k = 0; k < 3; ++k) B[k] = xf_point(bs, bm.verts[bm.idx[3 * bt + k]]);
            if (!triangle_bounds_overlap(A, B, margin)) continue;
            const V3<R> out_a = shell_outward(am, at, A[0], A[1], A[2]);
            const V3<R> out_b = shell_outward(bm, bt, B[0], B[1], B[2]);
            const V3<R> c_out_a = ah.static_body && interior_a ? V3<R>{} : out_a;
            const V3<R> c_out_b = bh.static_body && interior_b ? V3<R>{} : out_b;
            if (dot(out_a, out_b) > R(0.9999)) continue;
            V3<R> pa, pb;
            closest_triangle_pair(A, B, pa, pb);
            const V3<R> delta = sub(pa, pb);
            const R sq = len2(delta);
            if (sq > margin * margin) continue;
            const V3<R> cn = normalized_or(cross(sub(B[1], B[0]), sub(B[2], B[0])), V3<R>{0, 1, 0});
            V3<R> fallback = dot(cn, sub(ah.reference, pb)) >= R(0) ? cn : mul(cn, R(-1));
            if (len2(c_out_b) > R(0.5)) fallback = c_out_b;
            const R dist = std::sqrt(mx(sq, R(0)));
            const V3<R> point = mul(add(pa, pb), R(0.5));
            const V3<R> proj = sub(pa, mul(cn, dot(sub(pa, B[0]), cn)));
            const bool on_face = len2(sub(proj, closest_on_triangle(proj, B[0], B[1], B[2]))) <= R(1.0e-10);
            const V3<R> nrm = (dist <= R(1.0e-5) || on_face) ? fallback : normalized_or(delta, fallback);
            if (on_face && len2(out_a) < R(0.01) && len2(out_b) > R(0.5) && bm.convex) {
                const V3<R> face_a = normalized_or(cross(sub(A[1], A[0]), sub(A[2], A[0])), V3<R>{});
                if (ab(dot(face_a, nrm)) < R(1.0e-3)) {
                    const R depth = mx(R(0), -mn(dot(sub(A[0], B[0]), nrm),
                                                 mn(dot(sub(A[1], B[0]), nrm), dot(sub(A[2], B[0]), nrm))));
                    const V3<R> laxis = inv_rotate(bs.q, face_a);
                    const R off = dot(sub(bs.x, A[0]), face_a);
                    R lo = R(3.402823466e38), hi = R(-3.402823466e38);
                    for (const auto& v : bm.verts) {
                        const R pr = dot(v, laxis) + off;
                        lo = mn(lo, pr);
                        hi = mx(hi, pr);
                    }
                    const R alt = mx(R(0), mn(-lo, hi));
                    if (alt + R(1.0e-5) < depth) continue;
                }
            }
            const R separation = on_face && len2(c_out_b) > R(0.5) ? dot(delta, nrm) : dist;
            if (!reaches_rest_offset(as, bs, point, nrm, separation, rest, dt)) continue;
            Contact<R> c{};
            c.normal = nrm;
            c.point = point;
            c.penetration = rest - separation + R(1.0e-5);
            bool recovered = false;
            if (!am.convex && !bm.convex && dist <= R(1.0e-5)) {
                V3<R> oA[3], oB[3];
                for (uint32_t k = 0; k < 3; ++k) {
                    oA[k] = xf_point(aprev, am.verts[am.idx[3 * at + k]]);
                    oB[k] = xf_point(bprev, bm.verts[bm.idx[3 * bt + k]]);
                }
                V3<R> opa, opb;
                closest_triangle_pair(oA, oB, opa, opb);
                V3<R> od = sub(opa, opb);
                if (len2(od) > R(1.0e-10)) {
                    V3<R> iA[3], iB[3];
                    R low = 0, high = 1;
                    const R gap = mn(rest, R(0.5) * std::sqrt(len2(od)));
                    for (uint32_t it = 0; it < 10; ++it) {
                        const R time = R(0.5) * (low + high);
                        for (uint32_t k = 0; k < 3; ++k) {
                            iA[k] = add(oA[k], mul(sub(A[k], oA[k]), time));
                            iB[k] = add(oB[k], mul(sub(B[k], oB[k]), time));
                        }
                        V3<R> p, q;
                        closest_triangle_pair(iA, iB, p, q);
                        if (len2(sub(p, q)) > gap * gap)
                            low = time;
                        else
                            high = time;
                    }
                    for (uint32_t k = 0; k < 3; ++k) {
                        iA[k] = add(oA[k], mul(sub(A[k], oA[k]), low));
                        iB[k] = add(oB[k], mul(sub(B[k], oB[k]), low));
                    }
                    closest_triangle_pair(iA, iB, opa, opb);
                    od = sub(opa, opb);
                    c.normal = triangle_feature_normal(iA, iB, opa, opb, normalized_or(od, fallback));
                    const V3<R> cpa = advect_triangle_point(opa, iA, A);
                    const V3<R> cpb = advect_triangle_point(opb, iB, B);
                    c.point = mul(add(cpa, cpb), R(0.5));
                    c.penetration = rest - dot(sub(cpa, cpb), c.normal) + R(1.0e-5);
                    recovered = true;
                }
            }
            if (dist <= R(1.0e-5)) {
                if (!recovered && (ah.fixed_member || bh.fixed_member || on_face)) {
                    const R depth = mx(R(0), -mn(dot(sub(A[0], pb), nrm),
                                                 mn(dot(sub(A[1], pb), nrm), dot(sub(A[2], pb), nrm))));
                    c.penetration = mn(margin, depth + rest) + R(1.0e-5);
                } else if (!recovered) {
                    c.penetration = margin + R(1.0e-5);
                }
            }
            if (!shell_contact_facing(c.normal, c_out_a, c_out_b)) continue;
            c.impact_fraction = R(1);
            c.init_speed = normal_speed(as, bs, c.point, c.normal);
            add_contact(out, c, mx(R(2) * margin, R(1.0e-4)));
        }
    }
}

// geometry.slang:1921-2154 (the unguided pairs): conservative advancement
// of each triangle pair along its linear vertex paths from the previous to
// the current pose, up to 32 steps; the first pose within the rest offset
// gives a contact whose depth is the distance still to close this tick and
// whose impact fraction is the time reached (zero when it started in contact).
template <class R>
inline void collide_triangle_ranges_swept(const Mesh<R>& am, const State<R>& aprev, const State<R>& as,
                                          V3<R> prev_ref_a, const HingeFrame<R>& ah, uint32_t af, uint32_t ac,
                                          const Mesh<R>& bm, const State<R>& bprev, const State<R>& bs,
                                          const HingeFrame<R>& bh, uint32_t bf, uint32_t bc, R margin, R dt,
                                          Manifold<R>& out) {
    const bool guided = guided_pair(ah, bh);
    const HingeFrame<R>& guide = ah.axial ? ah : bh;
    const R rest = guided ? mn(margin, R(1.0e-4)) : mn(margin, R(1.0e-3));
    const bool interior_a = ah.static_body && point_inside_convex(am, aprev, bprev.x);
    const bool interior_b = bh.static_body && point_inside_convex(bm, bprev, aprev.x);
    const uint32_t a_tris = uint32_t(am.idx.size() / 3), b_tris = uint32_t(bm.idx.size() / 3);
    for (uint32_t i = 0; i < ac; ++i) {
        const uint32_t at = af + i;
        if (at >= a_tris) break;
        V3<R> PA[3], CA[3];
        for (uint32_t k = 0; k < 3; ++k) {
            const V3<R> l = am.verts[am.idx[3 * at + k]];
            PA[k] = xf_point(aprev, l);
            CA[k] = xf_point(as, l);
        }
        V3<R> alo = vmin(PA[0], CA[0]), ahi = vmax(PA[0], CA[0]);
        for (uint32_t k = 1; k < 3; ++k) {
            alo = vmin(alo, vmin(PA[k], CA[k]));
            ahi = vmax(ahi, vmax(PA[k], CA[k]));
        }
        for (uint32_t j = 0; j < bc; ++j) {
            const uint32_t bt = bf + j;
            if (bt >= b_tris) break;
            V3<R> PB[3], CB[3];
            for (uint32_t k = 0; k < 3; ++k) {
                const V3<R> l = bm.verts[bm.idx[3 * bt + k]];
                PB[k] = xf_point(bprev, l);
                CB[k] = xf_point(bs, l);
            }
            V3<R> blo = vmin(PB[0], CB[0]), bhi = vmax(PB[0], CB[0]);
            for (uint32_t k = 1; k < 3; ++k) {
                blo = vmin(blo, vmin(PB[k], CB[k]));
                bhi = vmax(bhi, vmax(PB[k], CB[k]));
            }
            const V3<R> ex{margin, margin, margin};
            if (!bounds_overlap(sub(alo, ex), add(ahi, ex), blo, bhi)) continue;
            V3<R> DA[3], DB[3];
            R abs_speed = 0;
            for (uint32_t k = 0; k < 3; ++k) {
                DA[k] = sub(CA[k], PA[k]);
                DB[k] = sub(CB[k], PB[k]);
                abs_speed = mx(abs_speed, len(DA[k]));
            }
            R col_speed = 0;
            for (uint32_t k = 0; k < 3; ++k) col_speed = mx(col_speed, len(DB[k]));
            abs_speed += col_speed;
            const V3<R> common = DB[0];
            R rel_a = 0, rel_b = 0;
            for (uint32_t k = 0; k < 3; ++k) {
                rel_a = mx(rel_a, len(sub(DA[k], common)));
                rel_b = mx(rel_b, len(sub(DB[k], common)));
            }
            const R bound = mn(abs_speed, rel_a + rel_b);
            if (bound <= kEps<R>()) continue;
            R time = 0;
            bool starts_near = false;
            V3<R> sep_n{};
            bool have_sep = false;
            for (uint32_t it = 0; it < 32; ++it) {
                V3<R> A[3], B[3];
                for (uint32_t k = 0; k < 3; ++k) {
                    A[k] = add(PA[k], mul(DA[k], time));
                    B[k] = add(PB[k], mul(DB[k], time));
                }
                V3<R> pa, pb;
                closest_triangle_pair(A, B, pa, pb);
                const V3<R> delta = sub(pa, pb);
                const R dist = std::sqrt(mx(R(0), len2(delta)));
                R offset = rest;
                if (guided && !triangle_pair_face_contact(A, B, delta)) {
                    // A witness off the guide's face, with both an axial and a
                    // turning component, is held at zero offset.
                    const V3<R> dir = normalized_or(delta, V3<R>{});
                    const R axial = dot(dir, guide.axis);
                    const R angular = dot(guide.axis, cross(sub(pa, guide.anchor), dir));
                    if (ab(axial) > R(1.0e-3) && ab(angular) > R(1.0e-3)) offset = R(0);
                }
                if (it == 0) {
                    starts_near = dist <= offset + R(5.0e-5);
                    // A gap wider than the largest relative motion of the tick
                    // (and 0.1 mm) cannot close: the advancement would end
                    // without contact.
                    if (dist > offset + R(1.0e-5) + bound + R(1.0e-4)) break;
                }
                if (dist <= offset + R(1.0e-5)) {
                    const V3<R> cn = normalized_or(cross(sub(B[1], B[0]), sub(B[2], B[0])), V3<R>{0, 1, 0});
                    const V3<R> center = add(aprev.x, mul(sub(as.x, aprev.x), time));
                    V3<R> fallback = dot(cn, sub(center, pb)) >= R(0) ? cn : mul(cn, R(-1));
                    if (ah.present) {
                        const V3<R> ref = add(prev_ref_a, mul(sub(ah.reference, prev_ref_a), time));
                        fallback = dot(cn, sub(ref, pb)) >= R(0) ? cn : mul(cn, R(-1));
                    }
                    const V3<R> out_a = shell_outward(am, at, A[0], A[1], A[2]);
                    const V3<R> out_b = shell_outward(bm, bt, B[0], B[1], B[2]);
                    const V3<R> c_out_a = ah.static_body && interior_a ? V3<R>{} : out_a;
                    const V3<R> c_out_b = bh.static_body && interior_b ? V3<R>{} : out_b;
                    if (dot(out_a, out_b) > R(0.9999)) break;
                    if (len2(c_out_b) > R(0.5))
                        fallback = c_out_b;
                    else if (len2(c_out_a) > R(0.5))
                        fallback = mul(c_out_a, R(-1));
                    const V3<R> nrm = triangle_feature_normal(A, B, pa, pb, have_sep ? sep_n : fallback);
                    if (!shell_contact_facing(nrm, c_out_a, c_out_b)) break;
                    const V3<R> point = mul(add(pa, pb), R(0.5));
                    const R speed = normal_speed(as, bs, point, nrm);
                    if (speed > R(1.0e-5)) break;
                    const R remaining = -speed * dt * (R(1) - time) - dist;
                    Contact<R> c{};
                    c.normal = nrm;
                    c.point = point;
                    c.penetration = mx(R(0), remaining + offset) + R(1.0e-5);
                    c.impact_fraction = starts_near ? R(0) : time;
                    c.init_speed = speed;
                    if (guided)
                        add_guided_contact(out, c, guide);
                    else
                        add_contact(out, c, mx(margin * R(2), R(1.0e-4)));
                    break;
                }
                sep_n = triangle_feature_normal(A, B, pa, pb, normalized_or(delta, V3<R>{0, 1, 0}));
                have_sep = true;
                R adv = (dist - offset) / (bound + kEps<R>()) * R(0.9);
                if (guided) {
                    // Advance by the gap along the separating feature plane
                    // when that is faster; a separating, opening gap ends it.
                    const V3<R> plane = triangle_feature_normal(A, B, pa, pb, sep_n);
                    R min_a = R(3.402823466e38), max_b = R(-3.402823466e38);
                    R min_va = R(3.402823466e38), max_vb = R(-3.402823466e38);
                    for (uint32_t k = 0; k < 3; ++k) {
                        min_a = mn(min_a, dot(sub(A[k], pb), plane));
                        max_b = mx(max_b, dot(sub(B[k], pb), plane));
                        min_va = mn(min_va, dot(DA[k], plane));
                        max_vb = mx(max_vb, dot(DB[k], plane));
                    }
                    const R gap = min_a - max_b - offset;
                    const R closing = max_vb - min_va;
                    if (gap > R(1.0e-5) && closing <= R(0)) break;
                    if (gap > R(0) && closing > kEps<R>()) adv = mx(adv, R(0.9) * gap / closing);
                }
                time += mx(adv, R(1.0e-5));
                if (time > R(1)) break;
            }
        }
    }
}

// geometry.slang:1586-1604
template <class R>
inline bool requires_swept(const State<R>& pa, const State<R>& a, const Mesh<R>& am, const State<R>& pb,
                           const State<R>& b, const Mesh<R>& bm, R threshold) {
    if (!am.convex || !bm.convex) threshold = mn(threshold, R(1.0e-3));
    const V3<R> rel = sub(sub(a.x, pa.x), sub(b.x, pb.x));
    return len(rel) + rotational_motion_bound(pa, a, am) + rotational_motion_bound(pb, b, bm) > threshold;
}

// geometry.slang:2156-2299 without the swept ranges: BVH pair traversal
// (stack of 64 pairs, children pushed right before left), the unswept
// triangle ranges at each overlapping leaf pair; a traversal that would
// overflow the stack restarts as one pass over all triangle pairs.
template <class R>
inline void collide_meshes(const World<R>& w, uint32_t a, uint32_t b, const std::vector<State<R>>& prev,
                           const std::vector<State<R>>& cur, const HingeFrame<R>& ah, const HingeFrame<R>& bh,
                           V3<R> prev_ref_a, R dt, Manifold<R>& out) {
    out = Manifold<R>{};
    const Mesh<R>& am = w.meshes[w.body[a].mesh];
    const Mesh<R>& bm = w.meshes[w.body[b].mesh];
    const R margin = R(w.body[a].margin) + R(w.body[b].margin);
    const bool swept = guided_pair(ah, bh) || requires_swept(prev[a], cur[a], am, prev[b], cur[b], bm, margin);
    const BoundsXf<R> pxa = swept ? bounds_xf(prev[a]) : BoundsXf<R>{}, pxb = swept ? bounds_xf(prev[b]) : BoundsXf<R>{};
    const BoundsXf<R> xa = bounds_xf(cur[a]), xb = bounds_xf(cur[b]);
    V3<R> alo, ahi, blo, bhi;
    motion_bounds(am.lo, am.hi, pxa, xa, swept, margin, alo, ahi);
    motion_bounds(bm.lo, bm.hi, pxb, xb, swept, R(0), blo, bhi);
    if (!bounds_overlap(alo, ahi, blo, bhi)) return;
    constexpr uint32_t kStack = 64;
    uint32_t sa[kStack] = {}, sb[kStack] = {};
    uint32_t size = 1;
    bool overflow = am.bvh.empty() || bm.bvh.empty();
    while (size > 0 && !overflow) {
        --size;
        const uint32_t na = sa[size], nb = sb[size];
        const BvhNode<R>& A = am.bvh[na];
        const BvhNode<R>& B = bm.bvh[nb];
        motion_bounds(A.lo, A.hi, pxa, xa, swept, margin, alo, ahi);
        motion_bounds(B.lo, B.hi, pxb, xb, swept, R(0), blo, bhi);
        if (!bounds_overlap(alo, ahi, blo, bhi)) continue;
        const bool la = A.count != 0, lb = B.count != 0;
        if (la && lb) {
            collide_triangle_ranges(am, prev[a], cur[a], ah, A.first, A.count, bm, prev[b], cur[b], bh, B.first,
                                    B.count, margin, dt, out);
            if (swept)
                collide_triangle_ranges_swept(am, prev[a], cur[a], prev_ref_a, ah, A.first, A.count, bm, prev[b],
                                              cur[b], bh, B.first, B.count, margin, dt, out);
            continue;
        }
        const uint32_t need = la || lb ? 2u : 4u;
        if (size + need > kStack) {
            overflow = true;
            break;
        }
        if (la) {
            sa[size] = na; sb[size++] = B.right;
            sa[size] = na; sb[size++] = B.left;
        } else if (lb) {
            sa[size] = A.right; sb[size++] = nb;
            sa[size] = A.left; sb[size++] = nb;
        } else {
            sa[size] = A.right; sb[size++] = B.right;
            sa[size] = A.right; sb[size++] = B.left;
            sa[size] = A.left; sb[size++] = B.right;
            sa[size] = A.left; sb[size++] = B.left;
        }
    }
    if (overflow) {
        out = Manifold<R>{};
        const uint32_t na = uint32_t(am.idx.size() / 3), nb = uint32_t(bm.idx.size() / 3);
        collide_triangle_ranges(am, prev[a], cur[a], ah, 0, na, bm, prev[b], cur[b], bh, 0, nb, margin, dt, out);
        if (swept)
            collide_triangle_ranges_swept(am, prev[a], cur[a], prev_ref_a, ah, 0, na, bm, prev[b], cur[b], bh, 0, nb,
                                          margin, dt, out);
    }
}

}  // namespace oracle

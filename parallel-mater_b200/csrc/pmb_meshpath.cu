// SPDX-License-Identifier: MIT
// Triangle-mesh narrowphase: the candidate pairs the convex face path does
// not take (a mesh that is not convex or has more than 96 indices, or a
// convex pair whose face manifold came out empty), as the reference's
// rigid_collide_meshes (geometry.slang:2156-2299) runs them: a traversal of
// the two meshes' BVHs in pairs, children pushed right before left on a
// 64-entry stack (a deeper traversal restarts as one pass over all triangle
// pairs), and at each overlapping pair of leaves the triangle-range contacts
// of :1359-1584 -- closest points of the two triangles (:949-1105), the
// certified shell normals that orient and filter them (:1308-1337), the
// rest-offset reach test (:1272-1290), the intersection recovery of two
// non-convex meshes (:1292-1306, :1855-1908) -- merged into at most eight
// contacts (:1129-1220); for a pair that moved more than its threshold, the
// swept triangle ranges (:1921-2155, conservative advancement) after the
// unswept ones at each leaf pair. A guided pair (a body on an unbreakable
// slider or piston to a static body, against a static body) takes only the
// swept ranges, with the guided offsets and advancement, and its contacts
// merge by guide direction (:1118-1170).
//
// One block per pair on the path: the traversal runs identically in every
// thread and the triangle pairs of each batch of leaf pairs are spread over
// the threads, their contacts merged in the reference's order. Per-body hinge
// contact frames (:404-492) are computed once per tick before the
// narrowphase; the face path uses them to skip guided pairs (:373-377).
#include "pmb_meshpath.cuh"

namespace pmb {

namespace {

constexpr uint32_t kStack = 64;

struct MeshPose { V3 x; Q4 q; V3 v, w; };

struct MeshMan {
    uint32_t count;
    V3 p[8], n[8];
    float pen[8], impact[8];
};

// geometry.slang:1129-1220, the unguided merge: a point within `spacing` of a
// kept one replaces it when deeper; a ninth point replaces the shallowest.
__device__ void mm_put(MeshMan& m, uint32_t i, V3 p, V3 n, float pen, float impact) {
    m.p[i] = p;
    m.n[i] = n;
    m.pen[i] = pen;
    m.impact[i] = impact;
}
__device__ void mm_add(MeshMan& m, V3 p, V3 n, float pen, float impact, float spacing) {
    const float s2 = spacing * spacing;
    for (uint32_t i = 0; i < m.count; ++i)
        if (len2(sub(m.p[i], p)) < s2) {
            if (pen - m.pen[i] > 0.0f) mm_put(m, i, p, n, pen, impact);
            return;
        }
    if (m.count < 8) {
        mm_put(m, m.count++, p, n, pen, impact);
        return;
    }
    uint32_t sh = 0;
    for (uint32_t i = 1; i < m.count; ++i)
        if (m.pen[i] < m.pen[sh]) sh = i;
    if (pen > m.pen[sh]) mm_put(m, sh, p, n, pen, impact);
}

struct Tri { V3 v[3]; };

__device__ __forceinline__ V3 xf(const MeshPose& s, V3 p) { return add(s.x, rotate(s.q, p)); }

struct MeshView {
    const float4* verts;
    const float4* planes;  // nt planes, then nt packed triangles
    const float4* bvh;
    const float4* shell;   // nullptr: no certified normals
    uint32_t nv, nt, nodes;
    bool solid;
    V3 lo, hi;
};

__device__ MeshView mesh_view(const Dev& d, uint32_t m) {
    MeshView v;
    v.verts = d.m_verts + d.m_vo[m];
    v.planes = d.m_planes + d.m_to[m];
    v.nv = d.m_vc[m];
    v.nt = d.m_tc[m];
    v.bvh = d.m_bvh + 3 * size_t(d.m_bo[m]);
    v.nodes = v.nt ? 1u : 0u;  // non-zero: the mesh has a BVH (its root is node 0)
    v.shell = d.m_so[m] == kInvalid ? nullptr : d.m_shell + d.m_so[m];
    v.solid = d.m_solid[m] != 0;
    v.lo = v3(d.m_lo[m]);
    v.hi = v3(d.m_hi[m]);
    return v;
}

__device__ __forceinline__ uint3 tri_index(const MeshView& m, uint32_t t) {
    const float4 k = m.planes[m.nt + t];
    return make_uint3(__float_as_uint(k.x), __float_as_uint(k.y), __float_as_uint(k.z));
}
__device__ __forceinline__ Tri posed_tri(const MeshView& m, uint32_t t, const MeshPose& s) {
    const uint3 k = tri_index(m, t);
    return {{xf(s, v3(m.verts[k.x])), xf(s, v3(m.verts[k.y])), xf(s, v3(m.verts[k.z]))}};
}

// geometry.slang:949-997
__device__ void closest_segments(V3 p0, V3 p1, V3 q0, V3 q1, V3& on_p, V3& on_q) {
    const V3 d0 = sub(p1, p0), d1 = sub(q1, q0), r = sub(p0, q0);
    const float a = dot(d0, d0), e = dot(d1, d1);
    float s = 0.0f, t = 0.0f;
    if (a <= 1.0e-12f && e <= 1.0e-12f) {
        on_p = p0;
        on_q = q0;
        return;
    }
    if (a <= 1.0e-12f) {
        t = fclamp(dot(d1, r) / e, 0.0f, 1.0f);
    } else {
        const float c = dot(d0, r);
        if (e <= 1.0e-12f) {
            s = fclamp(-c / a, 0.0f, 1.0f);
        } else {
            const float b = dot(d0, d1), f = dot(d1, r);
            const float den = a * e - b * b;
            if (fab(den) > kEps * a * e) s = fclamp((b * f - c * e) / den, 0.0f, 1.0f);
            t = (b * s + f) / e;
            if (t < 0.0f) {
                t = 0.0f;
                s = fclamp(-c / a, 0.0f, 1.0f);
            } else if (t > 1.0f) {
                t = 1.0f;
                s = fclamp((b - c) / a, 0.0f, 1.0f);
            }
        }
    }
    on_p = add(p0, mul(d0, s));
    on_q = add(q0, mul(d1, t));
}

// geometry.slang:1000-1031
__device__ V3 closest_on_triangle(V3 p, V3 a, V3 b, V3 c) {
    const V3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) return a;
    const V3 bp = sub(p, b);
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) return b;
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) return add(a, mul(ab, d1 / (d1 - d3)));
    const V3 cp = sub(p, c);
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) return c;
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) return add(a, mul(ac, d2 / (d2 - d6)));
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && d4 - d3 >= 0.0f && d5 - d6 >= 0.0f)
        return add(b, mul(sub(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6))));
    const V3 n = cross(ab, ac);
    return sub(p, mul(n, dot(ap, n) / len2(n)));
}

// geometry.slang:1033-1055
__device__ bool segment_hits_triangle(V3 p, V3 q, const Tri& t, V3& hit) {
    hit = V3{0.0f, 0.0f, 0.0f};
    const V3 n = cross(sub(t.v[1], t.v[0]), sub(t.v[2], t.v[0]));
    const V3 dir = sub(q, p);
    const float den = dot(n, dir);
    if (len2(n) <= kEps * kEps || fab(den) <= kEps) return false;
    const float amount = dot(n, sub(t.v[0], p)) / den;
    if (amount < 0.0f || amount > 1.0f) return false;
    hit = add(p, mul(dir, amount));
    const float tol = -1.0e-5f * len2(n);
    return dot(cross(sub(t.v[1], t.v[0]), sub(hit, t.v[0])), n) >= tol &&
           dot(cross(sub(t.v[2], t.v[1]), sub(hit, t.v[1])), n) >= tol &&
           dot(cross(sub(t.v[0], t.v[2]), sub(hit, t.v[2])), n) >= tol;
}

// geometry.slang:1057-1105
__device__ __noinline__ void closest_triangle_pair(const Tri& A, const Tri& B, V3& best_a, V3& best_b) {
    V3 hit;
    for (uint32_t e = 0; e < 3; ++e)
        if (segment_hits_triangle(A.v[e], A.v[(e + 1) % 3], B, hit)) {
            best_a = best_b = hit;
            return;
        }
    for (uint32_t e = 0; e < 3; ++e)
        if (segment_hits_triangle(B.v[e], B.v[(e + 1) % 3], A, hit)) {
            best_a = best_b = hit;
            return;
        }
    float best = 3.402823466e+38f;
    auto consider = [&](V3 p, V3 q) {
        const float s = len2(sub(p, q));
        if (s < best) {
            best = s;
            best_a = p;
            best_b = q;
        }
    };
    for (uint32_t i = 0; i < 3; ++i) consider(A.v[i], closest_on_triangle(A.v[i], B.v[0], B.v[1], B.v[2]));
    for (uint32_t i = 0; i < 3; ++i) consider(closest_on_triangle(B.v[i], A.v[0], A.v[1], A.v[2]), B.v[i]);
    for (uint32_t i = 0; i < 3; ++i)
        for (uint32_t j = 0; j < 3; ++j) {
            V3 on_a, on_b;
            closest_segments(A.v[i], A.v[(i + 1) % 3], B.v[j], B.v[(j + 1) % 3], on_a, on_b);
            consider(on_a, on_b);
        }
}

// geometry.slang:1272-1290
__device__ __forceinline__ float normal_speed(const MeshPose& a, const MeshPose& b, V3 p, V3 n) {
    const V3 va = add(a.v, cross(a.w, sub(p, a.x)));
    const V3 vb = add(b.v, cross(b.w, sub(p, b.x)));
    return dot(sub(va, vb), n);
}
__device__ bool reaches_rest_offset(const MeshPose& a, const MeshPose& b, V3 p, V3 n, float dist, float rest,
                                    float dt) {
    if (dist <= rest + 1.0e-5f) return true;
    const float speed = normal_speed(a, b, p, n);
    if (speed > 1.0e-5f) return false;
    return -speed * dt + rest + 1.0e-5f >= dist;
}

// geometry.slang:1292-1306
__device__ V3 advect_triangle_point(V3 p, const Tri& from, const Tri& to) {
    const V3 e1 = sub(from.v[1], from.v[0]), e2 = sub(from.v[2], from.v[0]);
    const V3 n = cross(e1, e2);
    const float sq = len2(n);
    if (sq <= 1.0e-20f) return to.v[0];
    const V3 rel = sub(p, from.v[0]);
    const float v = dot(cross(rel, e2), n) / sq;
    const float w = dot(cross(e1, rel), n) / sq;
    return add(to.v[0], add(mul(sub(to.v[1], to.v[0]), v), mul(sub(to.v[2], to.v[0]), w)));
}

// geometry.slang:1308-1322
__device__ V3 shell_outward(const MeshView& m, uint32_t t, const Tri& T) {
    if (!m.shell) return V3{0.0f, 0.0f, 0.0f};
    const V3 out = v3(m.shell[t]);
    const float sq = len2(out);
    if (sq < 0.01f) return V3{0.0f, 0.0f, 0.0f};
    const uint3 k = tri_index(m, t);
    const V3 la = v3(m.verts[k.x]), lb = v3(m.verts[k.y]), lc = v3(m.verts[k.z]);
    const float sign = dot(cross(sub(lb, la), sub(lc, la)), out) >= 0.0f ? 1.0f : -1.0f;
    return mul(normalized_or(cross(sub(T.v[1], T.v[0]), sub(T.v[2], T.v[0])), V3{0.0f, 0.0f, 0.0f}),
               sign * (sq > 0.5f ? 1.0f : 0.25f));
}

// geometry.slang:1324-1337
__device__ __forceinline__ bool shell_contact_facing(V3 n, V3 oa, V3 ob) {
    const float sa = len2(oa), sb = len2(ob);
    return (sa < 0.01f || (sa > 0.5f ? dot(n, oa) < -1.0e-3f : fab(dot(n, oa)) > 2.5e-4f)) &&
           (sb < 0.01f || (sb > 0.5f ? dot(n, ob) > 1.0e-3f : fab(dot(n, ob)) > 2.5e-4f));
}

// geometry.slang:1339-1357 over every plane of a convex mesh.
__device__ bool point_inside_convex(const MeshView& m, const MeshPose& s, V3 p) {
    if (!m.solid) return false;
    const V3 l = inv_rotate(s.q, sub(p, s.x));
    for (uint32_t t = 0; t < m.nt; ++t) {
        const float4 pl = m.planes[t];
        if (dot(v3(pl), l) > pl.w + 1.0e-5f) return false;
    }
    return true;
}

// geometry.slang:1855-1908
__device__ __noinline__ V3 triangle_feature_normal(const Tri& A, const Tri& B, V3 pa, V3 pb, V3 fallback) {
    const V3 delta = sub(pa, pb);
    V3 n = normalized_or(delta, fallback);
    const V3 faces[2] = {normalized_or(cross(sub(A.v[1], A.v[0]), sub(A.v[2], A.v[0])), n),
                         normalized_or(cross(sub(B.v[1], B.v[0]), sub(B.v[2], B.v[0])), n)};
    const Tri* tri[2] = {&A, &B};
    const V3 pts[2] = {pa, pb};
    float align_best = -1.0f;
    V3 interior_n{0.0f, 0.0f, 0.0f};
    for (uint32_t side = 0; side < 2; ++side) {
        const Tri& t = *tri[side];
        const V3 raw = cross(sub(t.v[1], t.v[0]), sub(t.v[2], t.v[0]));
        const float tol = 1.0e-5f * len2(raw);
        bool interior = tol > 0.0f;
        for (uint32_t e = 0; e < 3; ++e)
            interior = interior && dot(cross(sub(t.v[(e + 1) % 3], t.v[e]), sub(pts[side], t.v[e])), raw) > tol;
        const float align = fab(dot(faces[side], n));
        if (interior && align > align_best) {
            align_best = align;
            const float proj = dot(delta, faces[side]);
            const float dir = fab(proj) > kEps ? proj : dot(fallback, faces[side]);
            interior_n = dir >= 0.0f ? faces[side] : mul(faces[side], -1.0f);
        }
    }
    if (align_best >= 0.0f) return interior_n;
    float best_err = 4.0f * kEps * kEps;
    if (len2(delta) > kEps * kEps)
        for (uint32_t side = 0; side < 2; ++side) {
            const float proj = dot(delta, faces[side]);
            const float err = len2(sub(delta, mul(faces[side], proj)));
            if (err < best_err) {
                best_err = err;
                n = proj >= 0.0f ? faces[side] : mul(faces[side], -1.0f);
            }
        }
    return n;
}

struct Frame {
    V3 reference;
    uint32_t flags;
};

__device__ __forceinline__ Frame frame_of(const Dev& d, uint32_t i) {
    if (d.nj) {
        const float4 f = d.frame[i];
        return {v3(f), __float_as_uint(f.w)};
    }
    return {v3(d.tx[i]), d.motion[i] == kStatic ? kFrameStatic : 0u};
}


// The pair-invariant inputs of the triangle ranges (geometry.slang:1359-1379).
// The guide of a guided pair: its axial member's anchor, axis, inverse mass
// and moment, and whether it may turn about the axis (a piston).
struct Guide {
    V3 anchor, axis;
    float inv_mass, inv_moment;
    bool rotation;
};

struct RangeCtx {
    const MeshView* am;
    const MeshView* bm;
    MeshPose aprev, as, bprev, bs;
    Frame fa, fb;
    V3 prev_ref_a;  // the body's reference point at the previous pose
    float margin, rest, dt;
    bool interior_a, interior_b, guided, swept;
    Guide guide;
};

__device__ __forceinline__ Guide guide_of(const Dev& d, uint32_t a, uint32_t b, uint32_t fa) {
    const uint32_t g = (fa & kFrameAxial) ? a : b;
    const float4 ax = d.frame_guide[g], an = d.frame_anchor[g];
    return {v3(an), v3(ax), ax.w, an.w, (__float_as_uint(d.frame[g].w) & kFrameAxialRotation) != 0};
}

// geometry.slang:1118-1127
__device__ __forceinline__ V3 guide_direction(V3 n, V3 p, const Guide& g) {
    return V3{dot(n, g.axis) * sqrtf(g.inv_mass),
              g.rotation ? dot(g.axis, cross(sub(p, g.anchor), n)) * sqrtf(g.inv_moment) : 0.0f, 0.0f};
}

// geometry.slang:1129-1170, the guided merge: weak guide directions are
// dropped; among impacts only the earliest (within 1e-4 of the tick) stay; a
// contact along a kept one's guide direction replaces it when deeper per
// unit direction; else it is added (a ninth replaces the shallowest).
__device__ void mm_add_guided(MeshMan& m, V3 p, V3 n, float pen, float impact, const Guide& g) {
    const V3 cd = guide_direction(n, p, g);
    const float cl = len(cd);
    if (cl * cl <= kEps) return;
    if (impact > 0.0f) {
        float first = 1.0f;
        for (uint32_t i = 0; i < m.count; ++i)
            if (m.impact[i] > 0.0f) first = fmn(first, m.impact[i]);
        if (impact > first + 1.0e-4f) return;
        if (impact < first - 1.0e-4f) {
            uint32_t kept = 0;
            for (uint32_t i = 0; i < m.count; ++i)
                if (m.impact[i] == 0.0f) {
                    mm_put(m, kept, m.p[i], m.n[i], m.pen[i], m.impact[i]);
                    ++kept;
                }
            m.count = kept;
        }
    }
    for (uint32_t i = 0; i < m.count; ++i) {
        const V3 dk = guide_direction(m.n[i], m.p[i], g);
        const float size = len(dk);
        if (dot(cd, dk) > 0.9999f * cl * size) {
            if (pen / cl > m.pen[i] / size) mm_put(m, i, p, n, pen, impact);
            return;
        }
    }
    if (m.count < 8) {
        mm_put(m, m.count++, p, n, pen, impact);
        return;
    }
    uint32_t sh = 0;
    for (uint32_t i = 1; i < m.count; ++i)
        if (m.pen[i] < m.pen[sh]) sh = i;
    if (pen > m.pen[sh]) mm_put(m, sh, p, n, pen, impact);
}

// geometry.slang:1910-1919
__device__ __forceinline__ bool triangle_pair_face_contact(const Tri& A, const Tri& B, V3 sep) {
    const V3 zero{0.0f, 0.0f, 0.0f};
    const V3 n = normalized_or(sep, zero);
    const V3 fa = normalized_or(cross(sub(A.v[1], A.v[0]), sub(A.v[2], A.v[0])), zero);
    const V3 fb = normalized_or(cross(sub(B.v[1], B.v[0]), sub(B.v[2], B.v[0])), zero);
    return fab(dot(n, fa)) > 0.9999f || fab(dot(n, fb)) > 0.9999f;
}


__device__ __forceinline__ RangeCtx range_ctx_flat(const MeshView& am, const MeshPose& aprev, const MeshPose& as,
                                                   const Frame& fa, V3 prev_ref_a, const MeshView& bm,
                                                   const MeshPose& bprev, const MeshPose& bs, const Frame& fb,
                                                   float margin, float dt, bool swept, bool interior_a,
                                                   bool interior_b, bool guided, const Guide& guide) {
    return RangeCtx{&am,    &bm,        aprev,      as,     bprev, bs,   fa, fb, prev_ref_a,
                    margin, guided ? fmn(margin, 1.0e-4f) : fmn(margin, 1.0e-3f),
                    dt,     interior_a, interior_b, guided, swept, guide};
}

// The contact of triangle `at` of the body against triangle `bt` of the
// collider (the loop body of geometry.slang:1380-1583); false: none.
__device__ __noinline__ bool triangle_pair_contact(const RangeCtx& c, uint32_t at, uint32_t bt, V3& c_p, V3& c_n, float& c_pen) {
    if (c.guided) return false;  // a guided pair's ranges return at once (geometry.slang:1373)
    const MeshView& am = *c.am;
    const MeshView& bm = *c.bm;
    const float margin = c.margin, rest = c.rest;
    const Tri A = posed_tri(am, at, c.as);
    const Tri B = posed_tri(bm, bt, c.bs);
    {
        const V3 ex{margin, margin, margin};
        const V3 alo = sub(vmin(A.v[0], vmin(A.v[1], A.v[2])), ex);
        const V3 ahi = add(vmax(A.v[0], vmax(A.v[1], A.v[2])), ex);
        const V3 blo = vmin(B.v[0], vmin(B.v[1], B.v[2])), bhi = vmax(B.v[0], vmax(B.v[1], B.v[2]));
        if (!bounds_overlap(alo, ahi, blo, bhi)) return false;
    }
    const bool a_static = (c.fa.flags & kFrameStatic) != 0, b_static = (c.fb.flags & kFrameStatic) != 0;
    const V3 out_a = shell_outward(am, at, A), out_b = shell_outward(bm, bt, B);
    const V3 zero{0.0f, 0.0f, 0.0f};
    const V3 c_out_a = a_static && c.interior_a ? zero : out_a;
    const V3 c_out_b = b_static && c.interior_b ? zero : out_b;
    if (dot(out_a, out_b) > 0.9999f) return false;
    V3 pa, pb;
    closest_triangle_pair(A, B, pa, pb);
    const V3 delta = sub(pa, pb);
    const float sq = len2(delta);
    if (sq > margin * margin) return false;
    const V3 cn = normalized_or(cross(sub(B.v[1], B.v[0]), sub(B.v[2], B.v[0])), V3{0.0f, 1.0f, 0.0f});
    V3 fallback = dot(cn, sub(c.fa.reference, pb)) >= 0.0f ? cn : mul(cn, -1.0f);
    if (len2(c_out_b) > 0.5f) fallback = c_out_b;
    const float dist = sqrtf(fmx(sq, 0.0f));
    const V3 point = mul(add(pa, pb), 0.5f);
    const V3 proj = sub(pa, mul(cn, dot(sub(pa, B.v[0]), cn)));
    const bool on_face = len2(sub(proj, closest_on_triangle(proj, B.v[0], B.v[1], B.v[2]))) <= 1.0e-10f;
    const V3 nrm = (dist <= 1.0e-5f || on_face) ? fallback : normalized_or(delta, fallback);
    if (on_face && len2(out_a) < 0.01f && len2(out_b) > 0.5f && bm.solid) {
        const V3 face_a = normalized_or(cross(sub(A.v[1], A.v[0]), sub(A.v[2], A.v[0])), zero);
        if (fab(dot(face_a, nrm)) < 1.0e-3f) {
            const float depth = fmx(0.0f, -fmn(dot(sub(A.v[0], B.v[0]), nrm),
                                               fmn(dot(sub(A.v[1], B.v[0]), nrm), dot(sub(A.v[2], B.v[0]), nrm))));
            const V3 laxis = inv_rotate(c.bs.q, face_a);
            const float off = dot(sub(c.bs.x, A.v[0]), face_a);
            float lo = 3.402823466e+38f, hi = -3.402823466e+38f;
            for (uint32_t v = 0; v < bm.nv; ++v) {
                const float pr = dot(v3(bm.verts[v]), laxis) + off;
                lo = fmn(lo, pr);
                hi = fmx(hi, pr);
            }
            const float alt = fmx(0.0f, fmn(-lo, hi));
            if (alt + 1.0e-5f < depth) return false;
        }
    }
    const float separation = on_face && len2(c_out_b) > 0.5f ? dot(delta, nrm) : dist;
    if (!reaches_rest_offset(c.as, c.bs, point, nrm, separation, rest, c.dt)) return false;
    c_n = nrm;
    c_p = point;
    c_pen = rest - separation + 1.0e-5f;
    bool recovered = false;
    if (!am.solid && !bm.solid && dist <= 1.0e-5f) {
        const Tri oA = posed_tri(am, at, c.aprev), oB = posed_tri(bm, bt, c.bprev);
        V3 opa, opb;
        closest_triangle_pair(oA, oB, opa, opb);
        V3 od = sub(opa, opb);
        if (len2(od) > 1.0e-10f) {
            Tri iA, iB;
            float low = 0.0f, high = 1.0f;
            const float gap = fmn(rest, 0.5f * sqrtf(len2(od)));
            for (uint32_t it = 0; it < 10; ++it) {
                const float time = 0.5f * (low + high);
                for (uint32_t k = 0; k < 3; ++k) {
                    iA.v[k] = add(oA.v[k], mul(sub(A.v[k], oA.v[k]), time));
                    iB.v[k] = add(oB.v[k], mul(sub(B.v[k], oB.v[k]), time));
                }
                V3 p, q;
                closest_triangle_pair(iA, iB, p, q);
                if (len2(sub(p, q)) > gap * gap)
                    low = time;
                else
                    high = time;
            }
            for (uint32_t k = 0; k < 3; ++k) {
                iA.v[k] = add(oA.v[k], mul(sub(A.v[k], oA.v[k]), low));
                iB.v[k] = add(oB.v[k], mul(sub(B.v[k], oB.v[k]), low));
            }
            closest_triangle_pair(iA, iB, opa, opb);
            od = sub(opa, opb);
            c_n = triangle_feature_normal(iA, iB, opa, opb, normalized_or(od, fallback));
            const V3 cpa = advect_triangle_point(opa, iA, A);
            const V3 cpb = advect_triangle_point(opb, iB, B);
            c_p = mul(add(cpa, cpb), 0.5f);
            c_pen = rest - dot(sub(cpa, cpb), c_n) + 1.0e-5f;
            recovered = true;
        }
    }
    if (dist <= 1.0e-5f) {
        const bool fixed_member = ((c.fa.flags | c.fb.flags) & kFrameFixedMember) != 0;
        if (!recovered && (fixed_member || on_face)) {
            const float depth = fmx(0.0f, -fmn(dot(sub(A.v[0], pb), nrm),
                                               fmn(dot(sub(A.v[1], pb), nrm), dot(sub(A.v[2], pb), nrm))));
            c_pen = fmn(margin, depth + rest) + 1.0e-5f;
        } else if (!recovered) {
            c_pen = margin + 1.0e-5f;
        }
    }
    return shell_contact_facing(c_n, c_out_a, c_out_b);
}

// The swept contact of triangle `at` against `bt` (the loop body of
// geometry.slang:1963-2151 for an unguided pair): conservative advancement
// along the vertices' linear paths, up to 32 steps; false: none.
__device__ __noinline__ bool triangle_pair_swept_contact(const RangeCtx& c, uint32_t at, uint32_t bt, V3& c_p, V3& c_n,
                                            float& c_pen, float& c_impact) {
    const MeshView& am = *c.am;
    const MeshView& bm = *c.bm;
    const float margin = c.margin, rest = c.rest;
    const Tri PA = posed_tri(am, at, c.aprev), CA = posed_tri(am, at, c.as);
    const Tri PB = posed_tri(bm, bt, c.bprev), CB = posed_tri(bm, bt, c.bs);
    V3 alo = vmin(PA.v[0], CA.v[0]), ahi = vmax(PA.v[0], CA.v[0]);
    V3 blo = vmin(PB.v[0], CB.v[0]), bhi = vmax(PB.v[0], CB.v[0]);
    for (uint32_t k = 1; k < 3; ++k) {
        alo = vmin(alo, vmin(PA.v[k], CA.v[k]));
        ahi = vmax(ahi, vmax(PA.v[k], CA.v[k]));
        blo = vmin(blo, vmin(PB.v[k], CB.v[k]));
        bhi = vmax(bhi, vmax(PB.v[k], CB.v[k]));
    }
    const V3 ex{margin, margin, margin};
    if (!bounds_overlap(sub(alo, ex), add(ahi, ex), blo, bhi)) return false;
    Tri DA, DB;
    float abs_speed = 0.0f;
    for (uint32_t k = 0; k < 3; ++k) {
        DA.v[k] = sub(CA.v[k], PA.v[k]);
        DB.v[k] = sub(CB.v[k], PB.v[k]);
        abs_speed = fmx(abs_speed, len(DA.v[k]));
    }
    float col_speed = 0.0f;
    for (uint32_t k = 0; k < 3; ++k) col_speed = fmx(col_speed, len(DB.v[k]));
    abs_speed += col_speed;
    const V3 common = DB.v[0];
    float rel_a = 0.0f, rel_b = 0.0f;
    for (uint32_t k = 0; k < 3; ++k) {
        rel_a = fmx(rel_a, len(sub(DA.v[k], common)));
        rel_b = fmx(rel_b, len(sub(DB.v[k], common)));
    }
    const float bound = fmn(abs_speed, rel_a + rel_b);
    if (bound <= kEps) return false;
    const bool a_static = (c.fa.flags & kFrameStatic) != 0, b_static = (c.fb.flags & kFrameStatic) != 0;
    const V3 zero{0.0f, 0.0f, 0.0f};
    float time = 0.0f;
    bool starts_near = false, have_sep = false;
    V3 sep_n = zero;
    for (uint32_t it = 0; it < 32; ++it) {
        Tri A, B;
        for (uint32_t k = 0; k < 3; ++k) {
            A.v[k] = add(PA.v[k], mul(DA.v[k], time));
            B.v[k] = add(PB.v[k], mul(DB.v[k], time));
        }
        V3 pa, pb;
        closest_triangle_pair(A, B, pa, pb);
        const V3 delta = sub(pa, pb);
        const float dist = sqrtf(fmx(0.0f, len2(delta)));
        float offset = rest;
        if (c.guided && !triangle_pair_face_contact(A, B, delta)) {
            // A witness off the guide's face, with both an axial and a turning
            // component, is held at zero offset.
            const V3 dir = normalized_or(delta, zero);
            const float axial = dot(dir, c.guide.axis);
            const float angular = dot(c.guide.axis, cross(sub(pa, c.guide.anchor), dir));
            if (fab(axial) > 1.0e-3f && fab(angular) > 1.0e-3f) offset = 0.0f;
        }
        if (it == 0) {
            starts_near = dist <= offset + 5.0e-5f;
            // No point of either triangle moves more than `bound` relative to
            // the other during the tick: a gap wider than that (and 0.1 mm)
            // cannot close, and the advancement would end without contact.
            if (dist > offset + 1.0e-5f + bound + 1.0e-4f) return false;
        }
        if (dist <= offset + 1.0e-5f) {
            const V3 cn = normalized_or(cross(sub(B.v[1], B.v[0]), sub(B.v[2], B.v[0])), V3{0.0f, 1.0f, 0.0f});
            const V3 center = add(c.aprev.x, mul(sub(c.as.x, c.aprev.x), time));
            V3 fallback = dot(cn, sub(center, pb)) >= 0.0f ? cn : mul(cn, -1.0f);
            if (c.fa.flags & kFramePresent) {
                const V3 ref = add(c.prev_ref_a, mul(sub(c.fa.reference, c.prev_ref_a), time));
                fallback = dot(cn, sub(ref, pb)) >= 0.0f ? cn : mul(cn, -1.0f);
            }
            const V3 out_a = shell_outward(am, at, A), out_b = shell_outward(bm, bt, B);
            const V3 c_out_a = a_static && c.interior_a ? zero : out_a;
            const V3 c_out_b = b_static && c.interior_b ? zero : out_b;
            if (dot(out_a, out_b) > 0.9999f) return false;
            if (len2(c_out_b) > 0.5f)
                fallback = c_out_b;
            else if (len2(c_out_a) > 0.5f)
                fallback = mul(c_out_a, -1.0f);
            const V3 nrm = triangle_feature_normal(A, B, pa, pb, have_sep ? sep_n : fallback);
            if (!shell_contact_facing(nrm, c_out_a, c_out_b)) return false;
            const V3 point = mul(add(pa, pb), 0.5f);
            const float speed = normal_speed(c.as, c.bs, point, nrm);
            if (speed > 1.0e-5f) return false;
            const float remaining = -speed * c.dt * (1.0f - time) - dist;
            c_n = nrm;
            c_p = point;
            c_pen = fmx(0.0f, remaining + offset) + 1.0e-5f;
            c_impact = starts_near ? 0.0f : time;
            return true;
        }
        sep_n = triangle_feature_normal(A, B, pa, pb, normalized_or(delta, V3{0.0f, 1.0f, 0.0f}));
        have_sep = true;
        float adv = (dist - offset) / (bound + kEps) * 0.9f;
        if (c.guided) {
            // Advance by the gap along the separating feature plane when that
            // is faster; a separating, opening gap ends the search.
            const V3 plane = triangle_feature_normal(A, B, pa, pb, sep_n);
            float min_a = 3.402823466e+38f, max_b = -3.402823466e+38f;
            float min_va = 3.402823466e+38f, max_vb = -3.402823466e+38f;
            for (uint32_t k = 0; k < 3; ++k) {
                min_a = fmn(min_a, dot(sub(A.v[k], pb), plane));
                max_b = fmx(max_b, dot(sub(B.v[k], pb), plane));
                min_va = fmn(min_va, dot(DA.v[k], plane));
                max_vb = fmx(max_vb, dot(DB.v[k], plane));
            }
            const float gap = min_a - max_b - offset;
            const float closing = max_vb - min_va;
            if (gap > 1.0e-5f && closing <= 0.0f) return false;
            if (gap > 0.0f && closing > kEps) adv = fmx(adv, 0.9f * gap / closing);
        }
        time += fmx(adv, 1.0e-5f);
        if (time > 1.0f) return false;
    }
    return false;
}

__device__ __forceinline__ MeshPose pose_prev(const Dev& d, uint32_t i) {
    return {v3(d.x[i]), q4(d.q[i]), v3(d.v[i]), v3(d.w[i])};
}
__device__ __forceinline__ MeshPose pose_pred(const Dev& d, uint32_t i) {
    return {v3(d.tx[i]), q4(d.tq[i]), v3(d.tv[i]), v3(d.tw[i])};
}

// The mesh path runs flat over the whole tick rather than per pair:
//   1. walk (count): one thread per pair -- swept test, root bounds, the BVH
//      pair traversal of geometry.slang:2156-2299 (children pushed right before
//      left on a 64-entry stack; an overflow makes the pair one range over all
//      triangles); counts its overlapping leaf pairs and triangle-pair items
//      (unswept, then swept for a swept pair, per leaf pair);
//   2. exclusive scans of both counts;
//   3. walk (write): the same traversal records each leaf pair and where its
//      items start;
//   4. items: one thread per triangle pair evaluates its contact;
//   5. merge: one thread per pair merges its items' contacts in item order,
//      which is the reference's order, and stages them.
constexpr uint32_t kPairSwept = 1u, kPairInteriorA = 2u, kPairInteriorB = 4u;

// A BVH node: bounds, (first, count) of a leaf's triangles, children.
__device__ __forceinline__ void node_of(const MeshView& m, uint32_t k, V3& lo, V3& hi, uint32_t& first,
                                        uint32_t& count, uint32_t& left, uint32_t& right) {
    const float4 a = m.bvh[3 * k], b = m.bvh[3 * k + 1], c = m.bvh[3 * k + 2];
    lo = v3(a);
    hi = v3(b);
    first = __float_as_uint(a.w);
    count = __float_as_uint(b.w);
    left = __float_as_uint(c.x);
    right = __float_as_uint(c.y);
}

struct PairSetup {
    MeshView am, bm;
    MeshPose aprev, as, bprev, bs;
    Frame fa, fb;
    V3 prev_ref_a;
    float margin;
};

__device__ PairSetup pair_setup(const Dev& d, uint32_t k) {
    const uint32_t a = d.cand_a[k], b = d.cand_b[k];
    PairSetup p;
    p.am = mesh_view(d, d.mesh[a]);
    p.bm = mesh_view(d, d.mesh[b]);
    p.aprev = pose_prev(d, a);
    p.as = pose_pred(d, a);
    p.bprev = pose_prev(d, b);
    p.bs = pose_pred(d, b);
    p.fa = frame_of(d, a);
    p.fb = frame_of(d, b);
    p.prev_ref_a = d.nj ? v3(d.frame_prev[a]) : v3(d.x[a]);
    p.margin = d.p2[a].z + d.p2[b].z;
    return p;
}

// Steps 1 and 3. kWrite: record the leaf pairs from leaf_base on, their
// items from item_base on.
template <bool kWrite>
__device__ void mesh_walk(const Dev& d, const PairSetup& p, uint32_t pair, bool swept, uint32_t leaf_base,
                          uint32_t item_base, uint32_t& leaves, uint32_t& items) {
    leaves = items = 0;
    const uint32_t kinds = swept ? 2u : 1u;
    const BoundsXf zero_xf{};
    const BoundsXf pxa = swept ? bounds_xf(p.aprev.x, p.aprev.q) : zero_xf;
    const BoundsXf pxb = swept ? bounds_xf(p.bprev.x, p.bprev.q) : zero_xf;
    const BoundsXf xa = bounds_xf(p.as.x, p.as.q), xb = bounds_xf(p.bs.x, p.bs.q);
    auto emit = [&](uint32_t af, uint32_t ac, uint32_t bf, uint32_t bc) {
        if (kWrite && leaf_base + leaves < d.cap_mesh_leaves) {
            d.ml_rec[leaf_base + leaves] = make_uint4(af, ac, bf, bc);
            d.ml_item[leaf_base + leaves] = item_base + items;
            d.ml_pair[leaf_base + leaves] = pair;
        }
        ++leaves;
        items += kinds * ac * bc;
    };
    uint32_t sa[kStack], sb[kStack];
    sa[0] = 0;
    sb[0] = 0;
    uint32_t size = 1;
    bool overflow = p.am.nodes == 0 || p.bm.nodes == 0;
    while (size > 0 && !overflow) {
        --size;
        const uint32_t na = sa[size], nb = sb[size];
        uint32_t af, ac, al, ar, bf, bc, bl, br;
        V3 nlo, nhi, mlo, mhi, alo, ahi, blo, bhi;
        node_of(p.am, na, nlo, nhi, af, ac, al, ar);
        node_of(p.bm, nb, mlo, mhi, bf, bc, bl, br);
        motion_bounds(nlo, nhi, pxa, xa, swept, p.margin, alo, ahi);
        motion_bounds(mlo, mhi, pxb, xb, swept, 0.0f, blo, bhi);
        if (!bounds_overlap(alo, ahi, blo, bhi)) continue;
        const bool la = ac != 0, lb = bc != 0;
        if (la && lb) {
            emit(af, ac, bf, bc);
            continue;
        }
        const uint32_t need = la || lb ? 2u : 4u;
        if (size + need > kStack) {
            overflow = true;
            break;
        }
        if (la) {
            sa[size] = na; sb[size++] = br;
            sa[size] = na; sb[size++] = bl;
        } else if (lb) {
            sa[size] = ar; sb[size++] = nb;
            sa[size] = al; sb[size++] = nb;
        } else {
            sa[size] = ar; sb[size++] = br;
            sa[size] = ar; sb[size++] = bl;
            sa[size] = al; sb[size++] = br;
            sa[size] = al; sb[size++] = bl;
        }
    }
    if (overflow) {
        // The reference clears the manifold and runs every triangle pair.
        leaves = items = 0;
        emit(0, p.am.nt, 0, p.bm.nt);
    }
}

__global__ void k_mesh_walk_count(Dev d) {
    const uint32_t total = min(d.ctr->n_mesh, d.cap_mesh);
    for (uint32_t s = grid_stride_begin(); s < total; s += grid_stride()) {
        const PairSetup p = pair_setup(d, d.np_mesh[s]);
        uint32_t leaves = 0, items = 0, flags = 0;
        const bool guided = frames_guided(p.fa.flags, p.fb.flags);
        const bool swept = mesh_pair_swept(p.aprev.x, p.aprev.q, p.as.x, p.as.q, p.am.lo, p.am.hi, p.am.solid,
                                           p.bprev.x, p.bprev.q, p.bs.x, p.bs.q, p.bm.lo, p.bm.hi, p.bm.solid,
                                           p.margin, guided);
        const BoundsXf zero_xf{};
        V3 alo, ahi, blo, bhi;
        motion_bounds(p.am.lo, p.am.hi, swept ? bounds_xf(p.aprev.x, p.aprev.q) : zero_xf,
                      bounds_xf(p.as.x, p.as.q), swept, p.margin, alo, ahi);
        motion_bounds(p.bm.lo, p.bm.hi, swept ? bounds_xf(p.bprev.x, p.bprev.q) : zero_xf,
                      bounds_xf(p.bs.x, p.bs.q), swept, 0.0f, blo, bhi);
        if (bounds_overlap(alo, ahi, blo, bhi)) {
            mesh_walk<false>(d, p, s, swept, 0, 0, leaves, items);
            flags = swept ? kPairSwept : 0u;
            if ((p.fa.flags & kFrameStatic) && point_inside_convex(p.am, p.aprev, p.bprev.x)) flags |= kPairInteriorA;
            if ((p.fb.flags & kFrameStatic) && point_inside_convex(p.bm, p.bprev, p.aprev.x)) flags |= kPairInteriorB;
        }
        d.mp_leaves[s] = leaves;
        d.mp_items[s] = items;
        d.mp_flags[s] = flags;
    }
    if (grid_stride_begin() == 0 && d.ctr->n_mesh > d.cap_mesh) atomicOr(&d.ctr->status, kStPairOverflow);
}

__global__ void k_mesh_walk_write(Dev d) {
    const uint32_t total = min(d.ctr->n_mesh, d.cap_mesh);
    for (uint32_t s = grid_stride_begin(); s < total; s += grid_stride()) {
        if (!d.mp_leaves[s]) continue;
        const PairSetup p = pair_setup(d, d.np_mesh[s]);
        uint32_t leaves, items;
        mesh_walk<true>(d, p, s, (d.mp_flags[s] & kPairSwept) != 0, d.mp_leaf_off[s], d.mp_item_off[s], leaves,
                        items);
    }
    if (grid_stride_begin() == 0 &&
        (d.ctr->n_mesh_leaves > d.cap_mesh_leaves || d.ctr->n_mesh_items > d.cap_mesh_items))
        atomicOr(&d.ctr->status, kStContactOverflow);
}

// One warp per leaf pair (a leaf pair has at most 2 x 4 x 4 items; the
// single range of an overflowed traversal has more and loops), one lane per
// triangle-pair item.
__global__ void __launch_bounds__(128, 4) k_mesh_items(Dev d, StepParams sp) {
    const uint32_t leaves_total = min(d.ctr->n_mesh_leaves, d.cap_mesh_leaves);
    const uint32_t items_total = min(d.ctr->n_mesh_items, d.cap_mesh_items);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < leaves_total; j += warps) {
        const uint32_t s = d.ml_pair[j];
        const uint4 rec = d.ml_rec[j];
        const uint32_t flags = d.mp_flags[s];
        const bool swept = (flags & kPairSwept) != 0;
        const uint32_t size = rec.y * rec.w, count = (swept ? 2u : 1u) * size, base = d.ml_item[j];
        if (!size) continue;
        const PairSetup p = pair_setup(d, d.np_mesh[s]);
        const uint32_t k = d.np_mesh[s];
        const bool guided = d.nj && frames_guided(p.fa.flags, p.fb.flags);
        const Guide guide = guided ? guide_of(d, d.cand_a[k], d.cand_b[k], p.fa.flags) : Guide{};
        const RangeCtx c = range_ctx_flat(p.am, p.aprev, p.as, p.fa, p.prev_ref_a, p.bm, p.bprev, p.bs, p.fb, p.margin,
                                          sp.dt, swept, (flags & kPairInteriorA) != 0, (flags & kPairInteriorB) != 0,
                                          guided, guide);
        for (uint32_t local = lane; local < count; local += 32) {
            const uint32_t f = base + local;
            if (f >= items_total) break;
            const uint32_t t = local % size;
            const uint32_t at = rec.x + t / rec.w, bt = rec.z + t % rec.w;
            V3 cp{0.0f, 0.0f, 0.0f}, cn{0.0f, 0.0f, 0.0f};
            float pen = 0.0f, impact = 1.0f;
            bool valid = false;
            if (at < p.am.nt && bt < p.bm.nt)
                valid = local >= size ? triangle_pair_swept_contact(c, at, bt, cp, cn, pen, impact)
                                      : triangle_pair_contact(c, at, bt, cp, cn, pen);
            d.mi_valid[f] = valid ? 1u : 0u;
            d.mi_p[f] = f4(cp, impact);
            d.mi_n[f] = f4(cn, pen);
        }
    }
}

// One thread per pair: its items' contacts merged in item order (the
// reference's), then staged like the face path's.
__global__ void k_mesh_merge(Dev d, StepParams sp) {
    const uint32_t pairs = min(d.ctr->n_mesh, d.cap_mesh);
    const uint32_t total = min(d.ctr->n_mesh_items, d.cap_mesh_items);
    for (uint32_t s = grid_stride_begin(); s < pairs; s += grid_stride()) {
        const uint32_t k = d.np_mesh[s];
        const uint32_t i0 = d.mp_item_off[s], i1 = d.mp_item_off[s + 1];
        MeshMan m;
        m.count = 0;
        if (i1 > total) {
            // Items past the capacity were not evaluated (overflow reported).
            d.np_count[k] = 0;
            d.np_scan[k] = 0ull;
            continue;
        }
        const uint32_t a = d.cand_a[k], b = d.cand_b[k];
        const float spacing = fmx(2.0f * (d.p2[a].z + d.p2[b].z), 1.0e-4f);
        const uint32_t fa = d.nj ? __float_as_uint(d.frame[a].w) : 0u, fb = d.nj ? __float_as_uint(d.frame[b].w) : 0u;
        const bool guided = d.nj && frames_guided(fa, fb);
        const Guide guide = guided ? guide_of(d, a, b, fa) : Guide{};
        for (uint32_t f = i0; f < i1; ++f) {
            if (!d.mi_valid[f]) continue;
            const float4 pv = d.mi_p[f], nv = d.mi_n[f];
            if (guided)
                mm_add_guided(m, v3(pv), v3(nv), nv.w, pv.w, guide);
            else
                mm_add(m, v3(pv), v3(nv), nv.w, pv.w, spacing);
        }
        const uint32_t count = m.count;
        d.np_count[k] = count;
        d.np_scan[k] = count ? ((uint64_t(1) << 32) | count) : 0ull;
        if (!count) continue;
        const uint32_t slot = atomicAdd(&d.ctr->n_stage, count);
        if (slot + count > d.cap_stage) {
            atomicOr(&d.ctr->status, kStContactOverflow);
            d.np_scan[k] = 0ull;
            d.np_count[k] = 0;
            continue;
        }
        d.np_stage[k] = slot;
        for (uint32_t p = 0; p < count; ++p) {
            d.st_n[slot + p] = f4(m.n[p], m.pen[p]);
            d.st_p[slot + p] = f4(m.p[p], m.impact[p]);
        }
    }
}

// The frame of body i at one set of poses (pos/rot: the predicted or the
// previous positions and orientations of every body): reference point, flags.
// guide/guide_anchor (optional): the axis and inverse mass, the anchor and
// the inverse moment (geometry.slang:384-402) of an axial frame.
__device__ float4 hinge_frame_at(const Dev& d, uint32_t i, const float4* pos, const float4* rot,
                                 float4* guide = nullptr, float4* guide_anchor = nullptr) {
    uint32_t flags = d.motion[i] == kStatic ? kFrameStatic : 0u;
    const V3 x = v3(pos[i]);
    const Q4 q = q4(rot[i]);
    if (guide) *guide = *guide_anchor = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (!(d.p0[i].x > 0.0f)) return f4(x, __uint_as_float(flags));
    uint32_t incident = 0;
    bool present = false, axial = false, fixed_member = false, fixed = false, rotation = false;
    V3 anchor{0.0f, 0.0f, 0.0f}, axis{0.0f, 0.0f, 0.0f};
    for (uint32_t k = d.jb_off[i]; k < d.jb_off[i + 1]; ++k) {
        const uint32_t j = d.jb_list[k];
        const Joint& o = d.joints[j];
        if (!o.enabled || d.jstate[j].broken) continue;
        const bool is_a = o.body_a == i;
        ++incident;
        if (o.type == kFixed) fixed_member = true;
        const bool ax = o.type == kPiston || o.type == kSlider;
        const uint32_t other = is_a ? o.body_b : o.body_a;
        const bool static_anchor = other < d.n && d.motion[other] == kStatic;
        if (present || (o.type != kHinge && !(ax && static_anchor && !(o.breaking_threshold > 0.0f)))) continue;
        const V3 local_axis = ax ? V3{1.0f, 0.0f, 0.0f} : V3{0.0f, 0.0f, 1.0f};
        const float* la = is_a ? o.anchor_a : o.anchor_b;
        const float* lq = is_a ? o.frame_a : o.frame_b;
        anchor = add(x, rotate(q, V3{la[0], la[1], la[2]}));
        axis = normalized_or(rotate(qmul(q, Q4{lq[0], lq[1], lq[2], lq[3]}), local_axis), local_axis);
        present = true;
        fixed = static_anchor && !ax;
        axial = static_anchor && ax;
        rotation = axial && o.type == kPiston;
        if (static_anchor) {
            const float* lo = is_a ? o.anchor_b : o.anchor_a;
            const float* oq = is_a ? o.frame_b : o.frame_a;
            const Q4 qo = q4(rot[other]);
            anchor = add(v3(pos[other]), rotate(qo, V3{lo[0], lo[1], lo[2]}));
            axis = normalized_or(rotate(qmul(qo, Q4{oq[0], oq[1], oq[2], oq[3]}), local_axis), axis);
        }
    }
    if (axial && incident != 1u) axial = rotation = present = false;
    if (axial && guide) {
        const float4 p0 = d.p0[i];
        float moment = 0.0f;
        if ((fixed || rotation) && p0.x > kEps) {
            const V3 l = inv_rotate(q, axis);
            const float center = l.x * l.x / fmx(p0.y, kEps) + l.y * l.y / fmx(p0.z, kEps) + l.z * l.z / fmx(p0.w, kEps);
            const V3 arm = sub(x, anchor);
            const V3 perp = sub(arm, mul(axis, dot(arm, axis)));
            const float pivot = center + len2(perp) / p0.x;
            moment = pivot > kEps ? 1.0f / pivot : 0.0f;
        }
        *guide = f4(axis, p0.x);
        *guide_anchor = f4(anchor, moment);
    }
    flags |= (present ? kFramePresent : 0u) | (axial ? kFrameAxial : 0u) | (fixed_member ? kFrameFixedMember : 0u) |
             (rotation ? kFrameAxialRotation : 0u);
    return f4(present && !axial ? anchor : x, __uint_as_float(flags));
}

// Hinge contact frames (geometry.slang:404-492) at the predicted and at the
// previous poses: the first hinge joint, or unbreakable slider/piston to a
// static body, gives the frame; a fixed joint marks a fixed member; an axial
// frame needs the body's only joint. One thread per body.
__global__ void k_hinge_frames(Dev d) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        float4 guide, guide_anchor;
        d.frame[i] = hinge_frame_at(d, i, d.tx, d.tq, &guide, &guide_anchor);
        d.frame_guide[i] = guide;
        d.frame_anchor[i] = guide_anchor;
        d.frame_prev[i] = hinge_frame_at(d, i, d.x, d.q);
    }
}


}  // namespace

void launch_hinge_frames(const Dev& d, cudaStream_t s) {
    if (!d.nj) return;
    k_hinge_frames<<<blocks_for(d.n), kBlock, 0, s>>>(d);
    note_launch(blocks_for(d.n));
}

void launch_mesh_narrowphase(const Dev& d, const StepParams& sp, cudaStream_t s) {
    const uint32_t pairs_grid = cap_blocks(d.cap_mesh, 128);
    k_mesh_walk_count<<<pairs_grid, 128, 0, s>>>(d);
    note_launch(pairs_grid);
    prof_mark(s, "mesh walk");
    scan_u32(d.mp_leaves, d.mp_leaf_off, &d.ctr->n_mesh, d.cap_mesh, &d.ctr->n_mesh_leaves, d.scan_tmp32, s);
    scan_u32(d.mp_items, d.mp_item_off, &d.ctr->n_mesh, d.cap_mesh, &d.ctr->n_mesh_items, d.scan_tmp32, s);
    prof_mark(s, "mesh scans");
    k_mesh_walk_write<<<pairs_grid, 128, 0, s>>>(d);
    note_launch(pairs_grid);
    prof_mark(s, "mesh leaf pairs");
    const uint32_t items_grid = cap_blocks(32 * size_t(d.cap_mesh_leaves), 128);
    k_mesh_items<<<items_grid, 128, 0, s>>>(d, sp);
    note_launch(items_grid);
    prof_mark(s, "mesh triangle pairs");
    k_mesh_merge<<<pairs_grid, 128, 0, s>>>(d, sp);
    note_launch(pairs_grid);
}

}  // namespace pmb

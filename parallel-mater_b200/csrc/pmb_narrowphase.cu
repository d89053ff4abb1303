// SPDX-License-Identifier: MIT
// Convex face narrowphase, manifold compaction and the persistent contact
// cache.
//
// One thread per candidate pair runs the reference's convex face contact:
// SAT over every reference-face plane of both meshes (support = min over the
// incident mesh's vertices), most anti-aligned incident face, Sutherland-
// Hodgman clipping of each incident triangle coplanar with it against the
// reference planes, points within reach kept at the mid-plane, merged within
// 2*margin and capped at 8 by replacing the shallowest, then the collinear
// reduction (geometry.slang:1129-1270, 1606-1745), with the translation-only
// swept variant first for pairs that moved more than their margin
// (:1586-1604, :1751-1853) and the selection of pm_prepare_rigid_face_manifolds
// (:2741-2803). A pair the face path declines (not both face-capable, or an
// empty face manifold) goes to the triangle-mesh path (pmb_meshpath.cu); a
// guided pair skips the face path.
//
// Manifolds are staged by atomic allocation, then placed in pair order by a
// 64-bit scan (high word: non-empty pair rank, low word: contact offset), so
// pairs and contacts come out in the reference's active-pair order.
#include "pmb_meshpath.cuh"

namespace pmb {

struct Pose { V3 x; Q4 q; };
struct MeshRef {
    const float4* verts;
    const float4* planes;
    uint32_t nv, nt;
};
struct Man {
    V3 normal;
    float impact;
    uint32_t count;
    V3 p[8];
    float pen[8];
};

__device__ __forceinline__ MeshRef mesh_ref(const Dev& d, uint32_t m) {
    return {d.m_verts + d.m_vo[m], d.m_planes + d.m_to[m], d.m_vc[m], d.m_tc[m]};
}
__device__ __forceinline__ V3 pv(const MeshRef& m, uint32_t k) { return v3(m.verts[k]); }

__device__ void add_contact(Man& m, V3 p, float pen, float spacing) {
    float s2 = spacing * spacing;
    for (uint32_t i = 0; i < m.count; ++i) {
        if (len2(sub(m.p[i], p)) < s2) {
            if (pen - m.pen[i] > 0.0f) {
                m.p[i] = p;
                m.pen[i] = pen;
            }
            return;
        }
    }
    if (m.count < 8) {
        m.p[m.count] = p;
        m.pen[m.count] = pen;
        ++m.count;
        return;
    }
    uint32_t sh = 0;
    for (uint32_t i = 1; i < m.count; ++i)
        if (m.pen[i] < m.pen[sh]) sh = i;
    if (pen > m.pen[sh]) {
        m.p[sh] = p;
        m.pen[sh] = pen;
    }
}

__device__ void reduce_face_patch(Man& m, float tol) {
    float t2 = tol * tol;
    bool removed = true;
    while (removed) {
        removed = false;
        for (uint32_t cand = 0; cand < m.count && !removed; ++cand) {
            V3 p = m.p[cand];
            for (uint32_t f = 0; f < m.count && !removed; ++f) {
                if (f == cand) continue;
                for (uint32_t s = f + 1; s < m.count; ++s) {
                    if (s == cand) continue;
                    V3 e = sub(m.p[s], m.p[f]);
                    float e2 = len2(e);
                    if (e2 <= t2) continue;
                    float par = dot(sub(p, m.p[f]), e) / e2;
                    if (par <= 1.0e-4f || par >= 0.9999f) continue;
                    V3 cl = add(m.p[f], mul(e, par));
                    if (len2(sub(p, cl)) > t2) continue;
                    for (uint32_t k = cand + 1; k < m.count; ++k) {
                        m.p[k - 1] = m.p[k];
                        m.pen[k - 1] = m.pen[k];
                    }
                    --m.count;
                    removed = true;
                    break;
                }
            }
        }
    }
}

__device__ __forceinline__ bool same_plane(float4 a, float4 b) {
    return __float_as_uint(a.x) == __float_as_uint(b.x) && __float_as_uint(a.y) == __float_as_uint(b.y) &&
           __float_as_uint(a.z) == __float_as_uint(b.z) && __float_as_uint(a.w) == __float_as_uint(b.w);
}

// The separating-axis test of face_manifold (geometry.slang:1606-1640): the
// largest separation over every reference-face plane of both meshes (support
// = min over the other mesh's vertices), the face and side that give it. A
// plane equal to the one before it (a quad's second triangle) gives the same
// separation, which never wins the strict max, and is skipped. With
// `stop_above`, returns as soon as a separation exceeds it (the pair then
// has an empty manifold, whatever the later planes give).
struct FaceSat {
    float best;
    uint32_t ref_face;
    bool ref_body;
};
__device__ FaceSat face_sat(const Pose& bs, const MeshRef& bm, const Pose& cs, const MeshRef& cm,
                            float stop_above = kFltMax) {
    FaceSat r{-kFltMax, 0u, false};
    for (uint32_t side = 0; side < 2; ++side) {
        const MeshRef& rm = side == 0 ? cm : bm;
        const Pose& rs = side == 0 ? cs : bs;
        const MeshRef& im = side == 0 ? bm : cm;
        const Pose& is = side == 0 ? bs : cs;
        const V3 rel = sub(is.x, rs.x);
        for (uint32_t f = 0; f < rm.nt; ++f) {
            float4 pl = rm.planes[f];
            if (f != 0 && same_plane(pl, rm.planes[f - 1])) continue;
            V3 n = rotate(rs.q, v3(pl));
            V3 in = inv_rotate(is.q, n);
            float support = kFltMax;
            for (uint32_t k = 0; k < im.nv; ++k) support = fminf(support, dot(in, pv(im, k)));
            float sep = support + dot(n, rel) - pl.w;
            if (sep > r.best) {
                r.best = sep;
                r.ref_face = f;
                r.ref_body = side != 0;
                if (sep > stop_above) return r;
            }
        }
    }
    return r;
}

// geometry.slang:1606-1745. `sat`: the pair's separating-axis result when the
// caller already has it.
__device__ bool face_manifold(const Pose& bs, const MeshRef& bm, const Pose& cs, const MeshRef& cm, float margin,
                              float correction, Man& out, const FaceSat* sat = nullptr) {
    out.count = 0;
    out.impact = 1.0f;
    out.normal = {0, 0, 0};
    const float rest = fmn(margin, 1.0e-3f);
    const float reach = margin + correction;
    const FaceSat fs = sat ? *sat : face_sat(bs, bm, cs, cm);
    const float best = fs.best;
    const uint32_t ref_face = fs.ref_face;
    const bool ref_body = fs.ref_body;
    if (best > reach) return true;
    const MeshRef& rm = ref_body ? bm : cm;
    const Pose& rs = ref_body ? bs : cs;
    const MeshRef& im = ref_body ? cm : bm;
    const Pose& is = ref_body ? cs : bs;
    const float4 ref = rm.planes[ref_face];
    const V3 refn = v3(ref);
    V3 outward = rotate(rs.q, refn);
    V3 inc_axis = inv_rotate(is.q, outward);
    float align = 1.0f;
    uint32_t inc_face = 0;
    for (uint32_t f = 0; f < im.nt; ++f) {
        float v = dot(inc_axis, v3(im.planes[f]));
        if (v < align) {
            align = v;
            inc_face = f;
        }
    }
    out.normal = mul(outward, ref_body ? -1.0f : 1.0f);
    const float4 inc = im.planes[inc_face];
    const float spacing = fmx(margin * 2.0f, 1.0e-4f);
    V3 poly[36], clip[36];
    for (uint32_t t = 0; t < im.nt; ++t) {
        const float4 face = im.planes[t];
        if (dot(v3(face), v3(inc)) < 0.99999f || fab(face.w - inc.w) > 1.0e-5f) continue;
        // Incident triangle corners in the reference body's frame. A mesh's
        // plane block holds nt planes followed by nt packed index triples.
        uint32_t count = 3;
        const float4 packed = im.planes[im.nt + t];
        const uint32_t idx[3] = {__float_as_uint(packed.x), __float_as_uint(packed.y), __float_as_uint(packed.z)};
        for (uint32_t c = 0; c < 3; ++c)
            poly[c] = inv_rotate(rs.q, sub(add(is.x, rotate(is.q, pv(im, idx[c]))), rs.x));
        for (uint32_t pi = 0; pi < rm.nt && count != 0; ++pi) {
            const float4 pl = rm.planes[pi];
            const V3 pn = v3(pl);
            float off = pl.w + (dot(pn, refn) > 0.99999f ? reach : 0.0f);
            uint32_t cc = 0;
            V3 pvv = poly[count - 1];
            float pd = dot(pn, pvv) - off;
            for (uint32_t k = 0; k < count; ++k) {
                V3 cur = poly[k];
                float dd = dot(pn, cur) - off;
                // 36 slots hold any convex clip of a triangle by <= 32 planes;
                // the bound only guards rounding-degenerate polygons.
                if ((dd <= 0.0f) != (pd <= 0.0f) && cc < 36) clip[cc++] = add(pvv, mul(sub(cur, pvv), pd / (pd - dd)));
                if (dd <= 0.0f && cc < 36) clip[cc++] = cur;
                pvv = cur;
                pd = dd;
            }
            count = cc;
            for (uint32_t k = 0; k < count; ++k) poly[k] = clip[k];
        }
        for (uint32_t k = 0; k < count; ++k) {
            float dist = dot(refn, poly[k]) - ref.w;
            if (dist > reach) continue;
            V3 p = add(rs.x, rotate(rs.q, sub(poly[k], mul(refn, dist * 0.5f))));
            add_contact(out, p, rest - dist + 1.0e-5f, spacing);
        }
    }
    if (out.count == 0) return false;
    reduce_face_patch(out, fmx(1.0e-6f, margin * 1.0e-3f));
    return true;
}

// geometry.slang:1751-1853
__device__ bool swept_face_manifold(const Pose& pb, const Pose& b, const MeshRef& bm, const Pose& pc, const Pose& c,
                                    const MeshRef& cm, float margin, Man& out) {
    out.count = 0;
    Q4 bd = qrelative(pb.q, b.q, false), cd = qrelative(pc.q, c.q, false);
    if (bd.x != 0.0f || bd.y != 0.0f || bd.z != 0.0f || cd.x != 0.0f || cd.y != 0.0f || cd.z != 0.0f) return false;
    V3 bmo = sub(b.x, pb.x), cmo = sub(c.x, pc.x);
    const float rest = fmn(margin, 1.0e-3f);
    float entry = 0.0f, exit_t = 1.0f;
    V3 entry_n{0, 0, 0};
    for (uint32_t side = 0; side < 2; ++side) {
        const MeshRef& rm = side == 0 ? cm : bm;
        const MeshRef& im = side == 0 ? bm : cm;
        const Pose& rs = side == 0 ? pc : pb;
        const Pose& is = side == 0 ? pb : pc;
        V3 rel = side == 0 ? sub(bmo, cmo) : sub(cmo, bmo);
        for (uint32_t f = 0; f < rm.nt; ++f) {
            float4 pl = rm.planes[f];
            V3 n = rotate(rs.q, v3(pl));
            V3 in = inv_rotate(is.q, n);
            float support = kFltMax;
            for (uint32_t k = 0; k < im.nv; ++k) support = fminf(support, dot(in, pv(im, k)));
            float gap = support + dot(n, sub(is.x, rs.x)) - pl.w;
            float speed = dot(n, rel);
            if (speed == 0.0f) {
                if (gap > rest) return true;
            } else {
                float crossing = (rest - gap) / speed;
                if (speed < 0.0f && crossing > entry) {
                    entry = crossing;
                    entry_n = mul(n, side == 0 ? 1.0f : -1.0f);
                }
                if (speed > 0.0f) exit_t = fmn(exit_t, crossing);
            }
        }
    }
    if (entry > exit_t || entry > 1.0f || exit_t < 0.0f) return true;
    if (entry == 0.0f) {
        bool clipped = face_manifold(b, bm, c, cm, margin, 0.0f, out);
        if (clipped && out.count != 0) return true;
        if (!face_manifold(pb, bm, pc, cm, margin, 0.0f, out) || out.count == 0) return false;
        for (uint32_t p = 0; p < out.count; ++p) {
            float closing = -dot(sub(bmo, cmo), out.normal);
            if (closing <= 0.0f) return false;
            out.pen[p] += closing;
        }
        out.impact = 0.0f;
        return true;
    }
    Pose ib = pb, ic = pc;
    ib.x = add(pb.x, mul(bmo, entry));
    ic.x = add(pc.x, mul(cmo, entry));
    if (!face_manifold(ib, bm, ic, cm, rest + 1.0e-5f, 0.0f, out) || out.count == 0) return false;
    if (dot(out.normal, entry_n) < 0.99999f) return false;
    for (uint32_t p = 0; p < out.count; ++p) {
        float remaining = -dot(sub(bmo, cmo), out.normal) * (1.0f - entry);
        out.pen[p] = fmx(0.0f, remaining + out.pen[p]) + rest + 1.0e-5f;
    }
    out.impact = entry;
    return true;
}

__device__ __forceinline__ float rotational_bound(Q4 prev, Q4 cur, float rotb) {
    Q4 d = qrelative(prev, cur, false);
    return 2.0f * rotb * len(V3{d.x, d.y, d.z});
}

struct CandidateMotion {
    Pose prev_a, prev_b, pred_a, pred_b;
    float margin, corr;
    bool swept;
};
__device__ __forceinline__ CandidateMotion candidate_motion(const Dev& d, uint32_t a, uint32_t b) {
    CandidateMotion c;
    const float4 pa2 = d.p2[a], pb2 = d.p2[b];
    c.margin = pa2.z + pb2.z;
    c.corr = pa2.w + pb2.w;
    c.prev_a = {v3(d.x[a]), q4(d.q[a])};
    c.prev_b = {v3(d.x[b]), q4(d.q[b])};
    c.pred_a = {v3(d.tx[a]), q4(d.tq[a])};
    c.pred_b = {v3(d.tx[b]), q4(d.tq[b])};
    float moved = len(sub(sub(c.pred_a.x, c.prev_a.x), sub(c.pred_b.x, c.prev_b.x))) +
                  rotational_bound(c.prev_a.q, c.pred_a.q, d.rotb[a]) +
                  rotational_bound(c.prev_b.q, c.pred_b.q, d.rotb[b]);
    c.swept = moved > c.margin;
    return c;
}

// A candidate the face path leaves to the triangle-mesh path, queued for the
// mesh kernel with an empty manifold until then.
__device__ __forceinline__ void to_mesh_path(const Dev& d, uint32_t k) {
    d.np_count[k] = 0;
    d.np_scan[k] = 0ull;
    const uint32_t slot = atomicAdd(&d.ctr->n_mesh, 1u);
    d.np_mesh[slot] = k;
}

// Pass 1, one thread per candidate: pairs that are not both face-capable, and
// guided pairs, go to the triangle-mesh path; unswept pairs separated by a
// face plane get an empty manifold here; the rest go to the survivor list for
// pass 2 with their separating-axis result. Light enough for full occupancy.
__global__ void __launch_bounds__(256) k_narrow_sat(Dev d) {
    const uint32_t total = d.ctr->n_cand;
    for (uint32_t k = grid_stride_begin(); k < total; k += grid_stride()) {
        const uint32_t a = d.cand_a[k], b = d.cand_b[k];
        const uint32_t ma = d.mesh[a], mb = d.mesh[b];
        const bool guided = d.nj && frames_guided(__float_as_uint(d.frame[a].w), __float_as_uint(d.frame[b].w));
        if (!(d.m_convex[ma] && d.m_convex[mb]) || guided) {
            to_mesh_path(d, k);
            continue;
        }
        bool empty = false;
        FaceSat fs{0.0f, kInvalid, false};  // kInvalid face: no result kept (swept pair)
        {
            const CandidateMotion c = candidate_motion(d, a, b);
            if (!c.swept) {
                const float reach = c.margin + c.corr;
                fs = face_sat(c.pred_a, mesh_ref(d, ma), c.pred_b, mesh_ref(d, mb), reach);
                empty = fs.best > reach;
            }
        }
        if (empty) {
            d.np_count[k] = 0;
            d.np_scan[k] = 0ull;
        } else {
            const uint32_t slot = atomicAdd(&d.ctr->n_surv, 1u);
            d.np_list[slot] = k;
            d.np_sat[slot] = make_uint2(__float_as_uint(fs.best), fs.ref_face | (fs.ref_body ? 0x80000000u : 0u));
        }
    }
}

// Pass 2, one thread per surviving candidate: the full face manifold
// (swept variant first when the pair moved more than its margin).
__global__ void __launch_bounds__(128, 6) k_narrow(Dev d) {
    const uint32_t total = d.ctr->n_surv;
    for (uint32_t s = grid_stride_begin(); s < total; s += grid_stride()) {
        const uint32_t k = d.np_list[s];
        const uint2 sat = d.np_sat[s];
        const uint32_t a = d.cand_a[k], b = d.cand_b[k];
        const uint32_t ma = d.mesh[a], mb = d.mesh[b];
        Man m;
        m.count = 0;
        const MeshRef bm = mesh_ref(d, ma), cm = mesh_ref(d, mb);
        const CandidateMotion c = candidate_motion(d, a, b);
        bool ok = false;
        if (c.swept) ok = swept_face_manifold(c.prev_a, c.pred_a, bm, c.prev_b, c.pred_b, cm, c.margin, m);
        if (!ok) {
            // An unswept pair's separating-axis result comes from pass 1.
            const FaceSat fs{__uint_as_float(sat.x), sat.y & 0x7fffffffu, (sat.y >> 31) != 0};
            ok = face_manifold(c.pred_a, bm, c.pred_b, cm, c.margin, c.corr, m, c.swept ? nullptr : &fs);
            if (c.swept && m.count == 0) ok = false;
        }
        if (!ok) {
            // Most declined pairs lie beyond the pair margin: their root
            // bounds (the mesh path's first test) settle them here.
            if (mesh_pair_bounds_overlap(d, a, b, false)) {
                to_mesh_path(d, k);
            } else {
                d.np_count[k] = 0;
                d.np_scan[k] = 0ull;
            }
            continue;
        }
        const uint32_t count = m.count;
        d.np_count[k] = count;
        d.np_scan[k] = count ? ((uint64_t(1) << 32) | count) : 0ull;
        if (count) {
            uint32_t slot = atomicAdd(&d.ctr->n_stage, count);
            if (slot + count > d.cap_stage) {
                atomicOr(&d.ctr->status, kStContactOverflow);
                d.np_scan[k] = 0ull;
                d.np_count[k] = 0;
                continue;
            }
            d.np_stage[k] = slot;
            for (uint32_t p = 0; p < count; ++p) {
                d.st_n[slot + p] = f4(m.normal, m.pen[p]);
                d.st_p[slot + p] = f4(m.p[p], m.impact);
            }
        }
    }
}

// Scatter non-empty manifolds to their pair-ordered place and finalize them
// (geometry.slang:2852-2872: initial normal speed from predicted velocities).
__global__ void k_compact(Dev d) {
    const uint32_t total = d.ctr->n_cand;
    const uint64_t grand = d.np_scan[total];
    const uint32_t n_act = uint32_t(grand >> 32), n_con = uint32_t(grand & 0xffffffffu);
    if (grid_stride_begin() == 0) {
        uint32_t st = 0;
        if (n_act > d.cap_pair) st |= kStPairOverflow;
        if (n_con > d.cap_contact) st |= kStContactOverflow;
        if (st) atomicOr(&d.ctr->status, st);
        d.ctr->n_act = min(n_act, d.cap_pair);
        d.ctr->n_contacts = min(n_con, d.cap_contact);
    }
    for (uint32_t k = grid_stride_begin(); k < total; k += grid_stride()) {
        const uint32_t count = d.np_count[k];
        if (!count) continue;
        const uint64_t s = d.np_scan[k];
        const uint32_t i = uint32_t(s >> 32), off = uint32_t(s & 0xffffffffu);
        if (i >= d.cap_pair || off + count > d.cap_contact) continue;
        const uint32_t a = d.cand_a[k], b = d.cand_b[k];
        d.act_a[i] = a;
        d.act_b[i] = b;
        d.act_code[i] = uint64_t(a) * d.n + b;
        d.act_off[i] = off;
        d.act_cnt[i] = count;
        const uint32_t src = d.np_stage[k];
        const V3 xa = v3(d.tx[a]), xb = v3(d.tx[b]);
        const V3 va = v3(d.tv[a]), wa = v3(d.tw[a]), vb = v3(d.tv[b]), wb = v3(d.tw[b]);
        for (uint32_t p = 0; p < count; ++p) {
            const uint32_t c = off + p;
            float4 n = d.st_n[src + p], pt = d.st_p[src + p];
            V3 nn = v3(n), pp = v3(pt);
            V3 bv = add(va, cross(wa, sub(pp, xa)));
            V3 cv = add(vb, cross(wb, sub(pp, xb)));
            float speed = dot(sub(bv, cv), nn);
            d.c_pair[c] = i;
            d.c_bodies[c] = make_uint2(a, b);
            d.c_n[c] = n;
            d.c_p[c] = pt;
            d.c_e[c] = make_float4(0, 0, 0, speed);
            d.c_aa[c] = make_float4(0, 0, 0, 0);  // w: cached flag
            d.c_ab[c] = make_float4(0, 0, 0, 0);
            d.c_lam[c] = make_float4(0, 0, 0, 0);  // w: accumulated normal impulse
            d.c_pen[c] = make_float4(0, 0, 0, 0);  // w: stick flag of the latest dual pass
            d.c_accf[c] = make_float4(0, 0, 0, 0);
        }
    }
}

// geometry.slang:2941-3009, keyed by pair code against the previous tick's
// sorted saved pairs.
__global__ void k_cache_load(Dev d, StepParams sp) {
    const uint32_t n_act = d.ctr->n_act;
    const uint32_t n_saved = *d.sv_n_pairs;
    const float dt = sp.dt;
    const bool dt_ok = !(fab(*d.sv_dt - dt) > 1.0e-7f);
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        if (!dt_ok || n_saved == 0) continue;
        const uint64_t code = d.act_code[i];
        uint32_t lo = 0, hi = n_saved;
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (d.sv_code[mid] < code) lo = mid + 1;
            else hi = mid;
        }
        if (lo >= n_saved || d.sv_code[lo] != code) continue;
        const uint32_t so = d.sv_off[lo], sc = d.sv_cnt[lo];
        const uint32_t a = d.act_a[i];
        const V3 xa = v3(d.tx[a]);
        const Q4 qa = q4(d.tq[a]);
        const uint32_t off = d.act_off[i], cnt = d.act_cnt[i];
        uint32_t used = 0;
        for (uint32_t p = 0; p < cnt; ++p) {
            const uint32_t c = off + p;
            const V3 n = v3(d.c_n[c]);
            const V3 local = inv_rotate(qa, sub(v3(d.c_p[c]), xa));
            float nearest = 0.02f * 0.02f;
            uint32_t match = 8;
            for (uint32_t q = 0; q < sc; ++q) {
                if ((used & (1u << q)) != 0 || dot(n, v3(d.sv_normal[so + q])) < 0.99f) continue;
                float dd = len2(sub(local, v3(d.sv_local[so + q])));
                if (dd < nearest) {
                    nearest = dd;
                    match = q;
                }
            }
            if (match == 8) continue;
            used |= 1u << match;
            const uint32_t s = so + match;
            const float4 lam = d.sv_lam[s], pen = d.sv_pen[s], fimp = d.sv_fimp[s];
            V3 t0, t1;
            basis(n, t0, t1);
            const V3 fi = v3(fimp);
            float l1 = dot(fi, t0) / dt, l2 = dot(fi, t1) / dt;
            d.c_lam[c] = make_float4(lam.x, l1, l2, fimp.w);
            d.c_pen[c] = make_float4(pen.x, pen.y, pen.z, 0.0f);
            float4 aa = d.sv_aa[s], ab = d.sv_ab[s];
            aa.w = 1.0f;
            d.c_aa[c] = aa;
            d.c_ab[c] = ab;
            d.c_accf[c] = f4(sub(fi, mul(n, dot(fi, n))));
        }
    }
}

void launch_narrowphase(const Dev& d, const StepParams& sp, cudaStream_t s) {
    k_narrow_sat<<<cap_blocks(d.cap_cand, 256), 256, 0, s>>>(d);
    note_launch(cap_blocks(d.cap_cand, 256));
    prof_mark(s, "narrowphase SAT");
    k_narrow<<<cap_blocks(d.cap_cand, 128), 128, 0, s>>>(d);
    note_launch(cap_blocks(d.cap_cand, 128));
    prof_mark(s, "narrowphase manifolds");
    launch_mesh_narrowphase(d, sp, s);
    prof_mark(s, "narrowphase meshes");
    scan_u64(d.np_scan, d.np_scan, &d.ctr->n_cand, d.cap_cand, d.scan_tmp, s);
    k_compact<<<cap_blocks(d.cap_cand), kBlock, 0, s>>>(d);
    note_launch(cap_blocks(d.cap_cand));
    prof_mark(s, "compact");
    k_cache_load<<<cap_blocks(d.cap_pair, 128), 128, 0, s>>>(d, sp);
    note_launch(cap_blocks(d.cap_pair, 128));
    prof_mark(s, "cache load");
}

}  // namespace pmb

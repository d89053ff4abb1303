// SPDX-License-Identifier: MIT
// Bounds tests of the triangle-mesh path shared by the narrowphase passes:
// the transformed (and, for a swept pair, motion-unioned) AABBs of
// math.slang:142-190, the swept-pair test of geometry.slang:1586-1604, and
// the root-bounds test rigid_collide_meshes starts with (:2156-2188). A pair
// whose root bounds do not overlap has no triangle-mesh contacts, so the
// narrowphase only hands the others to the mesh kernel.
#pragma once
#include "pmb_world.cuh"

namespace pmb {

__device__ __forceinline__ bool bounds_overlap(V3 alo, V3 ahi, V3 blo, V3 bhi) {
    return alo.x <= bhi.x && ahi.x >= blo.x && alo.y <= bhi.y && ahi.y >= blo.y && alo.z <= bhi.z && ahi.z >= blo.z;
}

// math.slang:142-190
struct BoundsXf { V3 x, ax, ay, az; };
__device__ __forceinline__ BoundsXf bounds_xf(V3 x, Q4 q) {
    return {x, rotate(q, V3{1.0f, 0.0f, 0.0f}), rotate(q, V3{0.0f, 1.0f, 0.0f}),
            rotate(q, V3{0.0f, 0.0f, 1.0f})};
}
__device__ __forceinline__ void xf_bounds(V3 llo, V3 lhi, const BoundsXf& t, float margin, V3& lo, V3& hi) {
    const V3 c = mul(add(llo, lhi), 0.5f), h = mul(sub(lhi, llo), 0.5f);
    const V3 wc = add(t.x, add(mul(t.ax, c.x), add(mul(t.ay, c.y), mul(t.az, c.z))));
    const V3 wh{fab(t.ax.x) * h.x + fab(t.ay.x) * h.y + fab(t.az.x) * h.z,
                fab(t.ax.y) * h.x + fab(t.ay.y) * h.y + fab(t.az.y) * h.z,
                fab(t.ax.z) * h.x + fab(t.ay.z) * h.y + fab(t.az.z) * h.z};
    const V3 ex{margin, margin, margin};
    lo = sub(sub(wc, wh), ex);
    hi = add(add(wc, wh), ex);
}
__device__ __forceinline__ void motion_bounds(V3 llo, V3 lhi, const BoundsXf& prev, const BoundsXf& cur, bool swept,
                                              float margin, V3& lo, V3& hi) {
    xf_bounds(llo, lhi, cur, margin, lo, hi);
    if (!swept) return;
    V3 plo, phi;
    xf_bounds(llo, lhi, prev, margin, plo, phi);
    lo = vmin(lo, plo);
    hi = vmax(hi, phi);
}

// math.slang:192-206 for a mesh with local bounds [lo, hi].
__device__ __forceinline__ float mesh_rot_bound(Q4 prev, Q4 cur, V3 lo, V3 hi) {
    const Q4 dq = qrelative(prev, cur, false);
    const float s = len(V3{dq.x, dq.y, dq.z});
    const V3 ma{fmx(fab(lo.x), fab(hi.x)), fmx(fab(lo.y), fab(hi.y)), fmx(fab(lo.z), fab(hi.z))};
    return 2.0f * len(ma) * s;
}

// geometry.slang:1586-1604 (or a guided pair, :2168-2172).
__device__ __forceinline__ bool mesh_pair_swept(V3 xa0, Q4 qa0, V3 xa, Q4 qa, V3 alo, V3 ahi, bool asolid, V3 xb0,
                                                Q4 qb0, V3 xb, Q4 qb, V3 blo, V3 bhi, bool bsolid, float margin,
                                                bool guided) {
    float threshold = margin;
    if (!asolid || !bsolid) threshold = fmn(threshold, 1.0e-3f);
    const V3 rel = sub(sub(xa, xa0), sub(xb, xb0));
    return guided || len(rel) + mesh_rot_bound(qa0, qa, alo, ahi) + mesh_rot_bound(qb0, qb, blo, bhi) > threshold;
}

// The first test of rigid_collide_meshes: do the meshes' (motion) bounds
// overlap, the body's grown by the pair margin?
__device__ __forceinline__ bool mesh_pair_bounds_overlap(const Dev& d, uint32_t a, uint32_t b, bool guided) {
    const uint32_t ma = d.mesh[a], mb = d.mesh[b];
    const V3 alo = v3(d.m_lo[ma]), ahi = v3(d.m_hi[ma]), blo = v3(d.m_lo[mb]), bhi = v3(d.m_hi[mb]);
    const float margin = d.p2[a].z + d.p2[b].z;
    const V3 xa0 = v3(d.x[a]), xa = v3(d.tx[a]), xb0 = v3(d.x[b]), xb = v3(d.tx[b]);
    const Q4 qa0 = q4(d.q[a]), qa = q4(d.tq[a]), qb0 = q4(d.q[b]), qb = q4(d.tq[b]);
    const bool swept = mesh_pair_swept(xa0, qa0, xa, qa, alo, ahi, d.m_solid[ma] != 0, xb0, qb0, xb, qb, blo, bhi,
                                       d.m_solid[mb] != 0, margin, guided);
    const BoundsXf zero_xf{};
    const BoundsXf pxa = swept ? bounds_xf(xa0, qa0) : zero_xf, pxb = swept ? bounds_xf(xb0, qb0) : zero_xf;
    V3 lo_a, hi_a, lo_b, hi_b;
    motion_bounds(alo, ahi, pxa, bounds_xf(xa, qa), swept, margin, lo_a, hi_a);
    motion_bounds(blo, bhi, pxb, bounds_xf(xb, qb), swept, 0.0f, lo_b, hi_b);
    return bounds_overlap(lo_a, hi_a, lo_b, hi_b);
}

}  // namespace pmb

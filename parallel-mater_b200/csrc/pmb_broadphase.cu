// SPDX-License-Identifier: MIT
// Predict, swept proxies and broadphase.
//
// k_integrate fuses the reference's predictor (geometry.slang:524-612) with
// its spatial proxy emitter (geometry.slang:716-827): one thread per body
// writes the predicted state and the swept AABB min/max(prev, pred) +- (reach
// + bounded correction).
//
// The reference builds a Karras LBVH over those AABBs and queries it per
// dynamic body (primitives/spatial_build.slang:889-1011); the pair SET is
// defined by the inclusive AABB overlap predicate (:631-635) and the filter of
// geometry.slang:897-913, and its ORDER by (query body, candidate identity).
// Here the same predicate is evaluated over a uniform grid whose cell is the
// largest AABB extent among "small" bodies, so two overlapping small AABBs
// always sit in adjacent cells; bodies beyond a size threshold (ground,
// walls) are tested against every query. Cells are bucketed by the low bits
// of their Morton code and bodies are placed by a one-pass counting sort; each
// query's candidates are sorted by body index, which is the identity order of
// a world built without removals. Pair codes are a*N+b as in the reference.
#include "pmb_world.cuh"

namespace pmb {

__device__ __forceinline__ uint32_t expand10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
// Bucket of a grid cell; in a batched world the scene is part of the key.
__device__ __forceinline__ uint32_t cell_bucket(int cx, int cy, int cz, uint32_t size, uint32_t scene) {
    uint32_t m = expand10(uint32_t(cx)) | (expand10(uint32_t(cy)) << 1) | (expand10(uint32_t(cz)) << 2);
    uint32_t hi = (uint32_t(cx) >> 10) * 73856093u ^ (uint32_t(cy) >> 10) * 19349663u ^ (uint32_t(cz) >> 10) * 83492791u;
    return (m ^ hi ^ (scene * 0x9E3779B1u)) & (size - 1u);
}
__device__ __forceinline__ uint32_t scene_of(const Dev& d, uint32_t i) { return batched(d) ? d.scene_of[i] : 0u; }
__device__ __forceinline__ int4 cell_of(float4 lo, float4 hi, float hs) {
    V3 c = mul(add(v3(lo), v3(hi)), 0.5f);
    return make_int4(int(floorf(c.x / hs)), int(floorf(c.y / hs)), int(floorf(c.z / hs)), 0);
}

// Per-body constants computed once on the device, with the reference's
// operation order: reach = |centre| + radius + margin + 1e-5 and
// correction = min(0.5, 0.25 * max(0, min extent)) for dynamic bodies.
__global__ void k_body_constants(Dev d, const float4* mesh_lo, const float4* mesh_hi, const float4* mesh_sphere) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        uint32_t m = d.mesh[i];
        V3 lo = v3(mesh_lo[m]), hi = v3(mesh_hi[m]);
        float4 sph = mesh_sphere[m];
        float4 p2 = d.p2[i];
        float corr = 0.0f;
        if (d.motion[i] == kDynamic) {
            V3 e = sub(hi, lo);
            corr = fmn(0.5f, 0.25f * fmx(0.0f, fmn(e.x, fmn(e.y, e.z))));
        }
        p2.w = corr;
        d.p2[i] = p2;
        float reach = len(v3(sph)) + sph.w + p2.z + 1.0e-5f;
        d.expand[i] = fmn(1.0f, corr) + reach;
        V3 ma{fmx(fab(lo.x), fab(hi.x)), fmx(fab(lo.y), fab(hi.y)), fmx(fab(lo.z), fab(hi.z))};
        d.rotb[i] = len(ma);
    }
}
void launch_body_constants(const Dev& d, const float4* lo, const float4* hi, const float4* sph, cudaStream_t s) {
    k_body_constants<<<blocks_for(d.n), kBlock, 0, s>>>(d, lo, hi, sph);
    note_launch(blocks_for(d.n));
}

__global__ void k_integrate(Dev d, StepParams sp, float4* ox, float4* oq, float4* ov, float4* ow) {
    const float dt = sp.dt;
    const V3 g{sp.gx, sp.gy, sp.gz};
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        const uint32_t motion = d.motion[i];
        float4 x = d.x[i], q = d.q[i], v = d.v[i], w = d.w[i];
        V3 nx = v3(x), nv = v3(v), nw = v3(w);
        Q4 nq = q4(q);
        if (motion == kKinematic) {
            // Kinematic bodies follow a target set for this tick (one
            // substep: the whole way), else stand still (geometry.slang:545-581).
            const float4 tgt = d.tgt_x[i];
            if (tgt.w != 0.0f) {
                const float fraction = 1.0f;
                nx = add(v3(x), mul(sub(v3(tgt), v3(x)), fraction));
                Q4 t = q4(d.tgt_q[i]);
                const Q4 p = q4(q);
                const float od = p.x * t.x + p.y * t.y + p.z * t.z + p.w * t.w;
                if (od < 0.0f) t = Q4{-t.x, -t.y, -t.z, -t.w};
                nq = qnormalize(Q4{p.x + (t.x - p.x) * fraction, p.y + (t.y - p.y) * fraction,
                                   p.z + (t.z - p.z) * fraction, p.w + (t.w - p.w) * fraction});
                nv = mul(sub(nx, v3(x)), 1.0f / dt);
                nw = delta_velocity(p, nq, dt);
                d.tgt_x[i] = make_float4(0, 0, 0, 0);
            } else {
                nv = {0, 0, 0};
                nw = {0, 0, 0};
            }
        } else if (motion != kDynamic) {
            nv = {0, 0, 0};
            nw = {0, 0, 0};
        } else {
            const float4 p0 = d.p0[i], p1 = d.p1[i], p2 = d.p2[i];
            const V3 force = v3(d.force[i]), torque = v3(d.torque[i]);
            nv = add(nv, mul(add(g, mul(force, p0.x)), dt));
            nw = add(nw, mul(inv_inertia_world(p0, nq, torque), dt));
            nv = add(nv, mul(v3(d.lin_imp[i]), p0.x));
            nw = add(nw, inv_inertia_world(p0, nq, v3(d.ang_imp[i])));
            nv = mul(nv, 1.0f / (1.0f + p1.z * dt));
            nw = mul(nw, 1.0f / (1.0f + p1.w * dt));
            nv = clamp_length(nv, p2.x);
            nw = clamp_length(nw, p2.y);
            nx = add(nx, mul(nv, dt));
            Q4 dq = qmul(Q4{nw.x, nw.y, nw.z, 0.0f}, nq);
            nq = qnormalize(Q4{nq.x + 0.5f * dq.x * dt, nq.y + 0.5f * dq.y * dt, nq.z + 0.5f * dq.z * dt,
                               nq.w + 0.5f * dq.w * dt});
            const float4 z = make_float4(0, 0, 0, 0);
            d.force[i] = d.torque[i] = d.lin_imp[i] = d.ang_imp[i] = z;
        }
        // The predicted state is both the AVBD target and the initial solved
        // state (bodies the solve does not move keep it).
        d.tx[i] = ox[i] = f4(nx);
        d.tq[i] = oq[i] = f4(nq);
        d.tv[i] = ov[i] = f4(nv);
        d.tw[i] = ow[i] = f4(nw);
        // Swept proxy.
        const float e = d.expand[i];
        const V3 ex{e, e, e};
        V3 lo = sub(vmin(v3(x), nx), ex), hi = add(vmax(v3(x), nx), ex);
        d.lo[i] = f4(lo);
        d.hi[i] = f4(hi);
        bool finite = isfinite(lo.x) && isfinite(lo.y) && isfinite(lo.z) && isfinite(hi.x) && isfinite(hi.y) &&
                      isfinite(hi.z);
        V3 ext = sub(hi, lo);
        float m = fmx(ext.x, fmx(ext.y, ext.z));
        if (!finite) {
            atomicOr(&d.ctr->status, kStInvalidBounds);
            d.is_large[i] = 2;  // excluded
            continue;
        }
        if (m > d.large_extent) {
            d.is_large[i] = 1;
            uint32_t slot = atomicAdd(&d.ctr->n_large, 1u);
            d.large_list[slot] = i;
        } else {
            d.is_large[i] = 0;
            // Cell size: the largest small proxy (per scene in a batched
            // world, so a scene of small links keeps small cells).
            float* hs = batched(d) ? d.scene_hs + d.scene_of[i] : &d.ctr->hs;
            atomicMax(reinterpret_cast<int*>(hs), __float_as_int(m));
        }
    }
}

// Sparse record writes between ticks (host staging -> per-body arrays).
// kind 0: force, torque, linear impulse, angular impulse (replaces the
// body's pending inputs, src/simulation/runtime_rigid.cu.inc:265-294);
// kind 1: kinematic target position + normalised orientation (:197-230);
// kind 2: full state with normalised orientation, clearing the body's
// velocity history, pending inputs and target (:147-195). All of them are
// consumed and cleared by the next predictor, as pm_clear_rigid_inputs
// (src/slang/geometry.slang:2877-2886) does at the end of the reference tick.
__global__ void k_scatter_records(Dev d, uint32_t kind, uint32_t count) {
    for (uint32_t k = grid_stride_begin(); k < count; k += grid_stride()) {
        const uint32_t b = d.io_index[k];
        if (b >= d.n) continue;
        const float4* r = d.io_rec + 4 * size_t(k);
        if (kind == 0) {
            d.force[b] = r[0];
            d.torque[b] = r[1];
            d.lin_imp[b] = r[2];
            d.ang_imp[b] = r[3];
        } else if (kind == 1) {
            d.tgt_x[b] = make_float4(r[0].x, r[0].y, r[0].z, 1.0f);
            d.tgt_q[b] = f4(qnormalize(q4(r[1])));
        } else {
            d.x[b] = make_float4(r[0].x, r[0].y, r[0].z, 0.0f);
            d.q[b] = f4(qnormalize(q4(r[1])));
            d.v[b] = make_float4(r[2].x, r[2].y, r[2].z, 0.0f);
            d.w[b] = make_float4(r[3].x, r[3].y, r[3].z, 0.0f);
            d.prev_vel[b] = make_float4(0, 0, 0, 0);
            const float4 z = make_float4(0, 0, 0, 0);
            d.force[b] = d.torque[b] = d.lin_imp[b] = d.ang_imp[b] = z;
            d.tgt_x[b] = z;
        }
    }
}
void launch_scatter_records(const Dev& d, uint32_t kind, uint32_t count, cudaStream_t s) {
    if (count == 0) return;
    k_scatter_records<<<blocks_for(count), kBlock, 0, s>>>(d, kind, count);
    note_launch(blocks_for(count));
}

// States [first, first + count) as packed 13-float records (position,
// orientation xyzw, linear and angular velocity) at dst.
__global__ void k_pack_states(Dev d, uint32_t first, uint32_t count, float* dst) {
    for (uint32_t k = grid_stride_begin(); k < count; k += grid_stride()) {
        const uint32_t b = first + k;
        const float4 x = d.x[b], q = d.q[b], v = d.v[b], w = d.w[b];
        float* o = dst + 13 * size_t(k);
        o[0] = x.x; o[1] = x.y; o[2] = x.z;
        o[3] = q.x; o[4] = q.y; o[5] = q.z; o[6] = q.w;
        o[7] = v.x; o[8] = v.y; o[9] = v.z;
        o[10] = w.x; o[11] = w.y; o[12] = w.z;
    }
}
// The inverse for every body: x, q, v, w exactly as given (no
// renormalisation, unlike the record writes).
__global__ void k_unpack_states(Dev d, uint32_t count, const float* src) {
    for (uint32_t b = grid_stride_begin(); b < count; b += grid_stride()) {
        const float* o = src + 13 * size_t(b);
        d.x[b] = make_float4(o[0], o[1], o[2], 0.0f);
        d.q[b] = make_float4(o[3], o[4], o[5], o[6]);
        d.v[b] = make_float4(o[7], o[8], o[9], 0.0f);
        d.w[b] = make_float4(o[10], o[11], o[12], 0.0f);
    }
}
void launch_unpack_states(const Dev& d, uint32_t count, const float* src, cudaStream_t s) {
    if (count == 0) return;
    k_unpack_states<<<blocks_for(count), kBlock, 0, s>>>(d, count, src);
    note_launch(blocks_for(count));
}
void launch_pack_states(const Dev& d, uint32_t first, uint32_t count, float* dst, cudaStream_t s) {
    if (count == 0) return;
    k_pack_states<<<blocks_for(count), kBlock, 0, s>>>(d, first, count, dst);
    note_launch(blocks_for(count));
}

void launch_integrate(const Dev& d, const StepParams& sp, cudaStream_t s, const SolveBuffers& o) {
    if (d.n_scenes > 1) cudaMemsetAsync(d.scene_hs, 0, sizeof(float) * d.n_scenes, s);
    k_integrate<<<blocks_for(d.n), kBlock, 0, s>>>(d, sp, o.ox, o.oq, o.ov, o.ow);
    note_launch(blocks_for(d.n));
    prof_mark(s, "integrate+proxy");
}

__global__ void k_grid_count(Dev d) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        if (d.is_large[i] != 0) continue;
        const float h = batched(d) ? d.scene_hs[d.scene_of[i]] : d.ctr->hs;
        int4 c = cell_of(d.lo[i], d.hi[i], h > 0.0f ? h : 1.0f);
        d.grid_cell[i] = c;
        atomicAdd(&d.bucket_count[cell_bucket(c.x, c.y, c.z, d.grid_size, scene_of(d, i))], 1u);
    }
}

__global__ void k_grid_scatter(Dev d) {
    for (uint32_t i = grid_stride_begin(); i < d.n; i += grid_stride()) {
        if (d.is_large[i] != 0) continue;
        int4 c = d.grid_cell[i];
        uint32_t b = cell_bucket(c.x, c.y, c.z, d.grid_size, scene_of(d, i));
        uint32_t slot = d.bucket_off[b] + atomicAdd(&d.bucket_cursor[b], 1u);
        d.grid_body[slot] = i;
    }
}

__device__ __forceinline__ bool aabb_overlap(float4 alo, float4 ahi, float4 blo, float4 bhi) {
    return ahi.x >= blo.x && ahi.y >= blo.y && ahi.z >= blo.z && bhi.x >= alo.x && bhi.y >= alo.y && bhi.z >= alo.z;
}

__device__ __forceinline__ bool collision_disabled(const Dev& d, uint32_t a, uint32_t b) {
    if (d.n_dis == 0) return false;
    const uint64_t* keys = reinterpret_cast<const uint64_t*>(d.dis_keys);
    uint64_t key = (uint64_t(a < b ? a : b) << 32) | uint64_t(a < b ? b : a);
    uint32_t lo = 0, hi = d.n_dis;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    // constrained_collision_disabled (geometry.slang:494-511): only joints
    // that are not broken disable the pair.
    for (; lo < d.n_dis && keys[lo] == key; ++lo)
        if (d.jstate[d.dis_joint[lo]].broken == 0) return true;
    return false;
}

// Candidate predicate: overlap (leaf b against query a), a != b, identity
// order between two dynamic bodies, different fixed collision groups, no
// collision-disabling joint (geometry.slang:897-913).
__device__ __forceinline__ bool candidate(const Dev& d, uint32_t a, uint32_t b, float4 alo, float4 ahi) {
    if (b == a || d.is_large[b] == 2) return false;
    if (!aabb_overlap(d.lo[b], d.hi[b], alo, ahi)) return false;
    if (d.motion[b] == kDynamic && !(a < b)) return false;
    if (d.n_fixed && d.fixed_root[a] == d.fixed_root[b]) return false;
    if (collision_disabled(d, a, b)) return false;
    return true;
}

__device__ __forceinline__ uint32_t group_root(const volatile uint32_t* root, uint32_t b, uint32_t n) {
    for (uint32_t hop = 0; hop < n; ++hop) {
        const uint32_t p = root[b];
        if (p == b) break;
        b = p;
    }
    return b;
}

// Fixed collision groups (pm_build_fixed_collision_groups,
// geometry.slang:3102-3136): the groups are the connected components of the
// unbroken fixed joints that disable collisions, and each body's root is the
// smallest body of its component. One block: the unions run concurrently,
// every link hangs the larger of two roots under the smaller with a
// compare-and-swap, so a tree's root is always its smallest member and the
// result does not depend on the order the joints are taken in. Each loop is
// bounded by the body count (a failed swap means another union progressed).
__global__ void __launch_bounds__(1024) k_fixed_groups(Dev d) {
    volatile uint32_t* root = d.fixed_root;
    for (uint32_t i = threadIdx.x; i < d.n; i += blockDim.x) root[i] = i;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < d.n_fixed; k += blockDim.x) {
        const uint32_t j = d.fixed_list[k];
        if (d.jstate[j].broken) continue;
        uint32_t a = d.joints[j].body_a, b = d.joints[j].body_b;
        for (uint32_t attempt = 0; attempt <= d.n; ++attempt) {
            a = group_root(root, a, d.n);
            b = group_root(root, b, d.n);
            if (a == b) break;
            const uint32_t hi = a > b ? a : b, lo = a > b ? b : a;
            if (atomicCAS(d.fixed_root + hi, hi, lo) == hi) break;
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < d.n; i += blockDim.x) {
        const uint32_t r = group_root(root, i, d.n);
        root[i] = r;
    }
}

// The candidates of query body a that lane gl of a kQueryLanes-lane group
// finds: large bodies k = gl (mod lanes), then either every small body of
// the scene (a large dynamic a) or the grid cells q = gl (mod lanes) of the
// 27 around a's cell. The group's union is the reference's candidate set;
// the write pass sorts it by identity.
template <bool kWrite>
__device__ uint32_t visit_candidates(const Dev& d, uint32_t a, uint32_t gl, uint32_t* out, uint32_t cap) {
    const float4 alo = d.lo[a], ahi = d.hi[a];
    uint32_t count = 0;
    auto emit = [&](uint32_t b) {
        if (kWrite && count < cap) out[count] = b;
        ++count;
    };
    const bool multi = batched(d);
    const uint32_t scene = scene_of(d, a);
    // Large bodies (all of them, or this scene's).
    const uint32_t l0 = multi ? d.scene_large_off[scene] : 0u;
    const uint32_t l1 = multi ? d.scene_large_off[scene + 1] : d.ctr->n_large;
    const uint32_t* large = multi ? d.scene_large_list : d.large_list;
    for (uint32_t k = l0 + gl; k < l1; k += kQueryLanes) {
        uint32_t b = large[k];
        if (candidate(d, a, b, alo, ahi)) emit(b);
    }
    if (d.is_large[a] == 1) {
        const uint32_t b0 = multi ? d.scene_body_off[scene] : 0u, b1 = multi ? d.scene_body_off[scene + 1] : d.n;
        for (uint32_t b = b0 + gl; b < b1; b += kQueryLanes)
            if (d.is_large[b] == 0 && candidate(d, a, b, alo, ahi)) emit(b);
        return count;
    }
    const int4 c = d.grid_cell[a];
    for (uint32_t q = gl; q < 27u; q += kQueryLanes) {
        const int cx = c.x + int(q % 3u) - 1, cy = c.y + int((q / 3u) % 3u) - 1, cz = c.z + int(q / 9u) - 1;
        uint32_t bk = cell_bucket(cx, cy, cz, d.grid_size, scene);
        uint32_t s = d.bucket_off[bk], e = d.bucket_off[bk + 1];
        for (uint32_t k = s; k < e; ++k) {
            uint32_t b = d.grid_body[k];
            int4 cb = d.grid_cell[b];
            if (cb.x != cx || cb.y != cy || cb.z != cz) continue;
            if (multi && d.scene_of[b] != scene) continue;
            if (candidate(d, a, b, alo, ahi)) emit(b);
        }
    }
    return count;
}

// Per-scene large-body lists (batched worlds): count, offsets, scatter.
__global__ void k_scene_large_count(Dev d) {
    const uint32_t nl = d.ctr->n_large;
    for (uint32_t k = grid_stride_begin(); k < nl; k += grid_stride())
        atomicAdd(&d.scene_large_count[d.scene_of[d.large_list[k]]], 1u);
}
__global__ void k_scene_large_scatter(Dev d) {
    const uint32_t nl = d.ctr->n_large;
    for (uint32_t k = grid_stride_begin(); k < nl; k += grid_stride()) {
        const uint32_t b = d.large_list[k], s = d.scene_of[b];
        d.scene_large_list[d.scene_large_off[s] + atomicAdd(&d.scene_large_cursor[s], 1u)] = b;
    }
}

// kQueryLanes lanes per query body; each lane's count is kept for the
// write pass.
__global__ void k_query_count(Dev d) {
    const uint32_t gl = threadIdx.x % kQueryLanes;
    const uint32_t gmask = ((1u << kQueryLanes) - 1u) << (threadIdx.x & 31u & ~(kQueryLanes - 1u));
    const uint32_t groups = grid_stride() / kQueryLanes;
    for (uint32_t a = grid_stride_begin() / kQueryLanes; a < d.n; a += groups) {
        uint32_t c = 0;
        if (d.motion[a] == kDynamic && d.is_large[a] != 2) c = visit_candidates<false>(d, a, gl, nullptr, 0);
        d.cand_lane[size_t(a) * kQueryLanes + gl] = c;
        for (uint32_t o = kQueryLanes / 2; o > 0; o >>= 1) c += __shfl_xor_sync(gmask, c, o);
        if (gl == 0) d.cand_count[a] = c;
    }
}

__global__ void k_query_write(Dev d) {
    const uint32_t total = d.ctr->n_cand;
    if (grid_stride_begin() == 0 && total > d.cap_cand) atomicOr(&d.ctr->status, kStCandidateOverflow);
    const uint32_t gl = threadIdx.x % kQueryLanes;
    const uint32_t gmask = ((1u << kQueryLanes) - 1u) << (threadIdx.x & 31u & ~(kQueryLanes - 1u));
    const uint32_t groups = grid_stride() / kQueryLanes;
    for (uint32_t a = grid_stride_begin() / kQueryLanes; a < d.n; a += groups) {
        const uint32_t c = d.cand_count[a];
        const uint32_t off = d.cand_off[a];
        if (c == 0 || off >= d.cap_cand) continue;  // uniform over the group
        const uint32_t cap = min(c, d.cap_cand - off);
        uint32_t lane_off = 0;
        for (uint32_t k = 0; k < gl; ++k) lane_off += d.cand_lane[size_t(a) * kQueryLanes + k];
        uint32_t* seg = d.cand_b + off;
        if (lane_off < cap) visit_candidates<true>(d, a, gl, seg + lane_off, cap - lane_off);
        __syncwarp(gmask);
        if (gl == 0) {
            // Insertion sort by identity (dense index).
            for (uint32_t i = 1; i < cap; ++i) {
                uint32_t v = seg[i];
                uint32_t j = i;
                while (j > 0 && seg[j - 1] > v) {
                    seg[j] = seg[j - 1];
                    --j;
                }
                seg[j] = v;
            }
        }
        for (uint32_t i = gl; i < cap; i += kQueryLanes) d.cand_a[off + i] = a;
        __syncwarp(gmask);
    }
}

__global__ void k_clamp_count(uint32_t* count, uint32_t cap) {
    if (*count > cap) *count = cap;
}

void launch_broadphase(const Dev& d, cudaStream_t s) {
    if (d.n_scenes > 1) {
        cudaMemsetAsync(d.scene_large_count, 0, sizeof(uint32_t) * (d.n_scenes + 1), s);
        cudaMemsetAsync(d.scene_large_cursor, 0, sizeof(uint32_t) * d.n_scenes, s);
        k_scene_large_count<<<blocks_for(d.n), kBlock, 0, s>>>(d);
        note_launch(blocks_for(d.n));
        scan_u32(d.scene_large_count, d.scene_large_off, nullptr, d.n_scenes, nullptr, d.scan_tmp32, s);
        k_scene_large_scatter<<<blocks_for(d.n), kBlock, 0, s>>>(d);
        note_launch(blocks_for(d.n));
    }
    cudaMemsetAsync(d.bucket_count, 0, sizeof(uint32_t) * (d.grid_size + 1), s);
    cudaMemsetAsync(d.bucket_cursor, 0, sizeof(uint32_t) * d.grid_size, s);
    k_grid_count<<<blocks_for(d.n), kBlock, 0, s>>>(d);
    note_launch(blocks_for(d.n));
    scan_u32(d.bucket_count, d.bucket_off, nullptr, d.grid_size, nullptr, d.scan_tmp32, s);
    k_grid_scatter<<<blocks_for(d.n), kBlock, 0, s>>>(d);
    note_launch(blocks_for(d.n));
    prof_mark(s, "grid build");
    set_phase(kPhCandidates);
    if (d.n_fixed) {
        k_fixed_groups<<<1, 1024, 0, s>>>(d);
        note_launch(1);
    }
    k_query_count<<<blocks_for(kQueryLanes * d.n, 128), 128, 0, s>>>(d);
    note_launch(blocks_for(kQueryLanes * d.n, 128));
    prof_mark(s, "query count");
    scan_u32(d.cand_count, d.cand_off, nullptr, d.n, &d.ctr->n_cand, d.scan_tmp32, s);
    k_query_write<<<blocks_for(kQueryLanes * d.n, 128), 128, 0, s>>>(d);
    note_launch(blocks_for(kQueryLanes * d.n, 128));
    k_clamp_count<<<1, 1, 0, s>>>(&d.ctr->n_cand, d.cap_cand);
    note_launch(1);
    prof_mark(s, "query write");
}

}  // namespace pmb

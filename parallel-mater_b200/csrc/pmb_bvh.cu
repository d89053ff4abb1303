// SPDX-License-Identifier: MIT
// Mesh BVH build on the GPU: the same tree as the host builder the reference
// runs at mesh upload (src/simulation/runtime_deformables.cu.inc:136-210,
// restated in pmb_mesh.cpp) -- median split, split axis = longest extent of
// the node's triangle bounds, triangles ordered by the centroid coordinate
// on that axis (ties by triangle index), leaves of at most four triangles,
// nodes in pre-order -- for meshes too large to prepare on the host.
//
// The shape of the tree depends only on the triangle count, so the host lays
// out every node (range, children, pre-order index) and the device does the
// data-dependent part level by level: a block per node reduces its bounds and
// picks its axis; then every triangle of the nodes still to split gets the
// key (node start, centroid on the node's axis, triangle index) -- a finished
// leaf's triangles keep their place -- and a stable LSD radix sort (8-bit
// digits, one thread per 256-key tile for the histogram and the stable
// scatter) puts the level in order. The keys are total, so the order equals
// the host builder's comparison sort.
#include <cstring>
#include <vector>

#include "../../include/pmb200_core.h"
#include "pmb_world.cuh"

namespace pmb {
namespace {

constexpr uint32_t kTile = 256;

struct BvhSeg {
    uint32_t b, e, node, leaf;
};

__device__ __forceinline__ V3 tri_centroid(const float* v, const uint32_t* idx, uint32_t t) {
    const uint32_t i0 = idx[3 * t], i1 = idx[3 * t + 1], i2 = idx[3 * t + 2];
    const V3 a{v[3 * i0], v[3 * i0 + 1], v[3 * i0 + 2]};
    const V3 b{v[3 * i1], v[3 * i1 + 1], v[3 * i1 + 2]};
    const V3 c{v[3 * i2], v[3 * i2 + 1], v[3 * i2 + 2]};
    return mul(add(add(a, b), c), 1.0f / 3.0f);
}

// An order-preserving unsigned image of a float (-0 taken as +0, so the two
// compare equal as the host's `<` does).
__device__ __forceinline__ uint32_t float_key(float f) {
    uint32_t u = f == 0.0f ? 0u : __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// One block per node of the level: its bounds over its triangles, written to
// the node record, and (an inner node) its split axis.
__global__ void k_bvh_bounds(const BvhSeg* segs, const uint32_t* order, const float* v, const uint32_t* idx,
                             float* nodes, uint32_t* axes) {
    const BvhSeg s = segs[blockIdx.x];
    V3 lo{3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    V3 hi{-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    for (uint32_t i = s.b + threadIdx.x; i < s.e; i += blockDim.x) {
        const uint32_t t = order[i];
        for (uint32_t c = 0; c < 3; ++c) {
            const uint32_t k = idx[3 * t + c];
            const V3 p{v[3 * k], v[3 * k + 1], v[3 * k + 2]};
            lo = V3{fminf(lo.x, p.x), fminf(lo.y, p.y), fminf(lo.z, p.z)};
            hi = V3{fmaxf(hi.x, p.x), fmaxf(hi.y, p.y), fmaxf(hi.z, p.z)};
        }
    }
    __shared__ float red[6][256];
    red[0][threadIdx.x] = lo.x;
    red[1][threadIdx.x] = lo.y;
    red[2][threadIdx.x] = lo.z;
    red[3][threadIdx.x] = hi.x;
    red[4][threadIdx.x] = hi.y;
    red[5][threadIdx.x] = hi.z;
    __syncthreads();
    for (uint32_t w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 6; ++k) {
                const float o = red[k][threadIdx.x + w];
                red[k][threadIdx.x] = k < 3 ? fminf(red[k][threadIdx.x], o) : fmaxf(red[k][threadIdx.x], o);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        float* n = nodes + 10 * size_t(s.node);
        for (int k = 0; k < 6; ++k) n[k] = red[k][0];
        const float ex = red[3][0] - red[0][0], ey = red[4][0] - red[1][0], ez = red[5][0] - red[2][0];
        axes[blockIdx.x] = ex >= ey && ex >= ez ? 0u : (ey >= ez ? 1u : 2u);
    }
}

// Keys of the level: every position keeps (position, 0, 0) -- a finished
// leaf stays where it is -- unless a node still to split overwrites it below.
__global__ void k_bvh_keys_default(uint32_t* kp, uint32_t* ks, uint32_t* kt, uint32_t n) {
    for (uint32_t i = grid_stride_begin(); i < n; i += grid_stride()) {
        kp[i] = i;
        ks[i] = 0u;
        kt[i] = 0u;
    }
}
__global__ void k_bvh_keys_split(const BvhSeg* segs, const uint32_t* axes, const uint32_t* order, const float* v,
                                 const uint32_t* idx, uint32_t* kp, uint32_t* ks, uint32_t* kt) {
    const BvhSeg s = segs[blockIdx.x];
    if (s.leaf) return;
    const uint32_t axis = axes[blockIdx.x];
    for (uint32_t i = s.b + threadIdx.x; i < s.e; i += blockDim.x) {
        const uint32_t t = order[i];
        kp[i] = s.b;
        ks[i] = float_key(comp(tri_centroid(v, idx, t), axis));
        kt[i] = t;
    }
}

// Radix pass over the 8-bit digit at `shift` of key word `kd`: per-tile digit
// counts (digit-major, so their exclusive scan gives every tile's first slot
// per digit), then a stable scatter of all four arrays.
__global__ void k_bvh_hist(const uint32_t* kd, uint32_t shift, uint32_t n, uint32_t tiles, uint32_t* hist) {
    for (uint32_t tile = grid_stride_begin(); tile < tiles; tile += grid_stride()) {
        uint32_t count[256];
        for (uint32_t k = 0; k < 256; ++k) count[k] = 0;
        const uint32_t end = min(n, (tile + 1) * kTile);
        for (uint32_t i = tile * kTile; i < end; ++i) ++count[(kd[i] >> shift) & 255u];
        for (uint32_t k = 0; k < 256; ++k) hist[k * tiles + tile] = count[k];
    }
}
__global__ void k_bvh_scatter(const uint32_t* kd, uint32_t shift, uint32_t n, uint32_t tiles, const uint32_t* offs,
                              const uint32_t* kp, const uint32_t* ks, const uint32_t* kt, const uint32_t* val,
                              uint32_t* kp2, uint32_t* ks2, uint32_t* kt2, uint32_t* val2) {
    for (uint32_t tile = grid_stride_begin(); tile < tiles; tile += grid_stride()) {
        uint32_t next[256];
        for (uint32_t k = 0; k < 256; ++k) next[k] = offs[k * tiles + tile];
        const uint32_t end = min(n, (tile + 1) * kTile);
        for (uint32_t i = tile * kTile; i < end; ++i) {
            const uint32_t o = next[(kd[i] >> shift) & 255u]++;
            kp2[o] = kp[i];
            ks2[o] = ks[i];
            kt2[o] = kt[i];
            val2[o] = val[i];
        }
    }
}

// Any index at or past the vertex count sets *bad (checked before use).
__global__ void k_bvh_check(const uint32_t* idx, uint32_t count, uint32_t vertices, uint32_t* bad) {
    for (uint32_t i = grid_stride_begin(); i < count; i += grid_stride())
        if (idx[i] >= vertices) atomicOr(bad, 1u);
}

struct DeviceBuffers {
    std::vector<void*> owned;
    template <class T> T* get(size_t count, int& rc) {
        void* p = nullptr;
        if (rc == PMB_SUCCESS && cudaMalloc(&p, count * sizeof(T) + 16) != cudaSuccess) rc = PMB_ERROR_OUT_OF_DEVICE_MEMORY;
        if (p) owned.push_back(p);
        return static_cast<T*>(p);
    }
    ~DeviceBuffers() {
        for (void* p : owned) cudaFree(p);
    }
};

uint32_t lay_out(uint32_t b, uint32_t e, uint32_t level, std::vector<std::vector<BvhSeg>>& levels,
                 std::vector<uint32_t>& words) {
    const uint32_t node = uint32_t(words.size() / 10);
    words.resize(words.size() + 10, 0u);
    if (levels.size() <= level) levels.resize(level + 1);
    const bool leaf = e - b <= 4;
    levels[level].push_back(BvhSeg{b, e, node, leaf ? 1u : 0u});
    if (leaf) {
        words[10 * node + 6] = b;
        words[10 * node + 7] = e - b;
        return node;
    }
    const uint32_t mid = b + (e - b) / 2;
    const uint32_t left = lay_out(b, mid, level + 1, levels, words);
    const uint32_t right = lay_out(mid, e, level + 1, levels, words);
    words[10 * node + 8] = left;
    words[10 * node + 9] = right;
    return node;
}

}  // namespace
}  // namespace pmb

using namespace pmb;

extern "C" int pmb_mesh_bvh_build(const float* vertices, uint32_t vertex_count, const uint32_t* indices,
                                  uint32_t index_count, uint32_t* order, float* nodes, uint32_t node_capacity,
                                  uint32_t* node_count, void* stream) {
    if (!vertices || !indices || !order || !nodes || !node_count || vertex_count == 0 || index_count == 0 ||
        index_count % 3)
        return PMB_ERROR_INVALID_ARGUMENT;
    const uint32_t n = index_count / 3;
    std::vector<std::vector<BvhSeg>> levels;
    std::vector<uint32_t> words;
    lay_out(0, n, 0, levels, words);
    const uint32_t count = uint32_t(words.size() / 10);
    *node_count = count;
    if (count > node_capacity) return PMB_ERROR_CAPACITY_EXCEEDED;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = PMB_SUCCESS;
    DeviceBuffers buf;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    uint32_t* kp[2] = {buf.get<uint32_t>(n, rc), buf.get<uint32_t>(n, rc)};
    uint32_t* ks[2] = {buf.get<uint32_t>(n, rc), buf.get<uint32_t>(n, rc)};
    uint32_t* kt[2] = {buf.get<uint32_t>(n, rc), buf.get<uint32_t>(n, rc)};
    uint32_t* val[2] = {order, buf.get<uint32_t>(n, rc)};
    uint32_t* hist = buf.get<uint32_t>(size_t(256) * tiles + 1, rc);
    uint32_t* offs = buf.get<uint32_t>(size_t(256) * tiles + 1, rc);
    uint32_t* scan_tmp = buf.get<uint32_t>(size_t(256) * tiles / 2048 + 4, rc);
    size_t max_level = 0;
    for (const auto& l : levels) max_level = std::max(max_level, l.size());
    BvhSeg* segs = buf.get<BvhSeg>(max_level, rc);
    uint32_t* axes = buf.get<uint32_t>(max_level, rc);
    uint32_t* bad = buf.get<uint32_t>(1, rc);
    if (rc != PMB_SUCCESS) return rc;
    uint32_t bad_host = 0;
    cudaMemsetAsync(bad, 0, 4, s);
    k_bvh_check<<<cap_blocks(index_count, kBlock), kBlock, 0, s>>>(indices, index_count, vertex_count, bad);
    note_launch(cap_blocks(index_count, kBlock));
    if (cudaMemcpyAsync(&bad_host, bad, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess || bad_host)
        return PMB_ERROR_INVALID_ARGUMENT;
    // Node structure (range, children) from the host; bounds from the device.
    if (cudaMemcpyAsync(nodes, words.data(), 4 * words.size(), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return PMB_ERROR_INVALID_ARGUMENT;
    std::vector<uint32_t> iota(n);
    for (uint32_t i = 0; i < n; ++i) iota[i] = i;
    cudaMemcpyAsync(order, iota.data(), 4 * size_t(n), cudaMemcpyHostToDevice, s);
    const uint32_t pgrid = cap_blocks(n, kBlock), tgrid = cap_blocks(tiles, 64);
    for (const auto& level : levels) {
        const uint32_t m = uint32_t(level.size());
        cudaMemcpyAsync(segs, level.data(), sizeof(BvhSeg) * m, cudaMemcpyHostToDevice, s);
        k_bvh_bounds<<<m, 256, 0, s>>>(segs, val[0], vertices, indices, nodes, axes);
        note_launch(m);
        bool split = false;
        for (const auto& g : level) split = split || !g.leaf;
        if (!split) continue;
        k_bvh_keys_default<<<pgrid, kBlock, 0, s>>>(kp[0], ks[0], kt[0], n);
        note_launch(pgrid);
        k_bvh_keys_split<<<m, 256, 0, s>>>(segs, axes, val[0], vertices, indices, kp[0], ks[0], kt[0]);
        note_launch(m);
        // LSD: triangle index, then centroid key, then node start (only the
        // bytes a position can use).
        uint32_t pos_bytes = 1;
        while (pos_bytes < 4 && (uint64_t(n) >> (8 * pos_bytes)) != 0) ++pos_bytes;
        for (int word = 0; word < 3; ++word) {
            const uint32_t bytes = word == 2 ? pos_bytes : 4u;
            for (uint32_t byte = 0; byte < bytes; ++byte) {
                uint32_t* kd = word == 0 ? kt[0] : (word == 1 ? ks[0] : kp[0]);
                k_bvh_hist<<<tgrid, 64, 0, s>>>(kd, 8 * byte, n, tiles, hist);
                note_launch(tgrid);
                scan_u32(hist, offs, nullptr, 256 * tiles, nullptr, scan_tmp, s);
                k_bvh_scatter<<<tgrid, 64, 0, s>>>(kd, 8 * byte, n, tiles, offs, kp[0], ks[0], kt[0], val[0], kp[1],
                                                   ks[1], kt[1], val[1]);
                note_launch(tgrid);
                std::swap(kp[0], kp[1]);
                std::swap(ks[0], ks[1]);
                std::swap(kt[0], kt[1]);
                std::swap(val[0], val[1]);
            }
        }
    }
    // The order may have ended in the scratch copy.
    if (val[0] != order) cudaMemcpyAsync(order, val[0], 4 * size_t(n), cudaMemcpyDeviceToDevice, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? PMB_SUCCESS : PMB_ERROR_INVALID_ARGUMENT;
}

// SPDX-License-Identifier: MIT
// Device-wide exclusive prefix sums whose length is read from device memory,
// so compaction stages (candidate pairs, contacts) need no host round trip.
// Three passes: per-tile totals, one-block scan of the tile totals, per-tile
// scan with the tile's offset. Tiles are 2048 elements (256 threads x 8).
#include "pmb_world.cuh"

namespace pmb {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

template <class T> __device__ T block_exclusive_scan(T v, T* total) {
    __shared__ T warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_sums[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        T s = lane < kScanThreads / 32 ? warp_sums[lane] : T(0);
        T si = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += y;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = si - s;
        if (lane == kScanThreads / 32 - 1 && total) *total = si;
    }
    __syncthreads();
    T r = inc - v + warp_sums[wid];
    __syncthreads();
    return r;
}

template <class T>
__global__ void k_tile_sums(const T* in, const uint32_t* count_ptr, uint32_t capacity, T* tile_sums) {
    uint32_t count = count_ptr ? min(*count_ptr, capacity) : capacity;
    uint32_t base = blockIdx.x * kScanTile;
    T s = 0;
    if (base < count) {
        for (int k = 0; k < kScanItems; ++k) {
            uint32_t i = base + threadIdx.x * kScanItems + k;
            if (i < count) s += in[i];
        }
    }
    __shared__ T total;
    block_exclusive_scan<T>(s, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

template <class T> __global__ void k_scan_tiles(T* tile_sums, uint32_t tiles, T* grand_total) {
    // One block: each thread owns a contiguous run of tile sums.
    const uint32_t per = (tiles + kScanThreads - 1) / kScanThreads;
    uint32_t b = threadIdx.x * per;
    T s = 0;
    for (uint32_t k = 0; k < per; ++k)
        if (b + k < tiles) s += tile_sums[b + k];
    __shared__ T total;
    T off = block_exclusive_scan<T>(s, &total);
    for (uint32_t k = 0; k < per; ++k) {
        if (b + k < tiles) {
            T v = tile_sums[b + k];
            tile_sums[b + k] = off;
            off += v;
        }
    }
    if (threadIdx.x == 0 && grand_total) *grand_total = total;
}

template <class T>
__global__ void k_scan_apply(const T* in, T* out, const uint32_t* count_ptr, uint32_t capacity, const T* tile_sums) {
    uint32_t count = count_ptr ? min(*count_ptr, capacity) : capacity;
    uint32_t base = blockIdx.x * kScanTile;
    if (base >= count) return;
    T vals[kScanItems];
    T s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint32_t i = base + threadIdx.x * kScanItems + k;
        vals[k] = i < count ? in[i] : T(0);
        s += vals[k];
    }
    T off = block_exclusive_scan<T>(s, nullptr) + tile_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        uint32_t i = base + threadIdx.x * kScanItems + k;
        if (i < count) out[i] = off;
        off += vals[k];
    }
}

template <class T>
__global__ void k_scan_total(T* out, const uint32_t* count_ptr, uint32_t capacity, const T* grand_total) {
    uint32_t count = count_ptr ? min(*count_ptr, capacity) : capacity;
    out[count] = *grand_total;
}

template <class T>
static void scan_impl(const T* in, T* out, const uint32_t* count_ptr, uint32_t capacity, T* tmp, cudaStream_t s) {
    uint32_t tiles = (capacity + kScanTile - 1) / kScanTile;
    if (tiles == 0) tiles = 1;
    k_tile_sums<T><<<tiles, kScanThreads, 0, s>>>(in, count_ptr, capacity, tmp);
    note_launch(tiles);
    k_scan_tiles<T><<<1, kScanThreads, 0, s>>>(tmp, tiles, tmp + tiles);
    note_launch(1);
    k_scan_apply<T><<<tiles, kScanThreads, 0, s>>>(in, out, count_ptr, capacity, tmp);
    note_launch(tiles);
    k_scan_total<T><<<1, 1, 0, s>>>(out, count_ptr, capacity, tmp + tiles);
    note_launch(1);
}

// out must hold capacity + 1 entries; out[count] receives the total and, when
// total is non-null, so does *total.
__global__ void k_copy_total(const uint32_t* out, const uint32_t* count_ptr, uint32_t capacity, uint32_t* total) {
    uint32_t count = count_ptr ? min(*count_ptr, capacity) : capacity;
    *total = out[count];
}

void scan_u32(const uint32_t* in, uint32_t* out, const uint32_t* count_ptr, uint32_t capacity, uint32_t* total,
              uint32_t* tmp, cudaStream_t s) {
    scan_impl<uint32_t>(in, out, count_ptr, capacity, tmp, s);
    if (total) {
        k_copy_total<<<1, 1, 0, s>>>(out, count_ptr, capacity, total);
        note_launch(1);
    }
}

void scan_u64(const uint64_t* in, uint64_t* out, const uint32_t* count_ptr, uint32_t capacity, uint64_t* tmp,
              cudaStream_t s) {
    scan_impl<uint64_t>(in, out, count_ptr, capacity, tmp, s);
}

}  // namespace pmb

// SPDX-License-Identifier: MIT
// Learned warm start on the tensor cores (see pmb_mlp.cuh for the model).
//
// k_mlp_tiles runs the MLP over 128-contact tiles with tcgen05.mma: one CTA
// of 4 warps per SM walks tiles persistently; thread 0 issues the MMAs and
// commits them to an mbarrier, every thread owns one contact row of the tile
// (TMEM lane = row) for the element-wise work between layers. Tiles of X and
// their row metadata arrive by bulk copy (cp.async.bulk) into a double
// buffer. In training mode the same CTA runs the backward pass for its tile
// and accumulates the three weight gradients in TMEM across all its tiles;
// each CTA writes one partial gradient vector, reduced in CTA order by
// k_mlp_reduce_adam (deterministic).
//
// Shared-memory operands use the no-swizzle canonical layout: 8-row x
// 16-byte core matrices. Activation tiles store column block j/8 at
// 2048 * (j/8) and row group r/8 at 128 * (r/8), which serves both as a
// K-major operand (rows = contacts) and as an MN-major operand (the
// transposed view the weight gradients need), so no transposed copies are
// made.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "pmb_mlp.cuh"
#include "pmb_world.cuh"

namespace pmb {
namespace {

// ---------------------------------------------------------------- PTX
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// Bounded wait on an mbarrier phase: gives up after ~1 s and reports it.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    const uint64_t start = globaltimer();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if (globaltimer() - start > 1000000000ull) return false;
    }
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor: kind::f16 with BF16 A and B, FP32 accumulator.
__host__ __device__ constexpr uint32_t idesc(uint32_t m, uint32_t n, uint32_t a_mn_major, uint32_t b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn_major << 15) | (b_mn_major << 16) | ((n >> 3) << 17) |
           ((m >> 4) << 24);
}
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(
            d_tmem),
        "l"(a), "l"(b), "r"(id), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(a));
    const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(b));
    return lo | (hi << 16);
}
// Stores 8 FP32 values as one 16-byte BF16 row chunk.
__device__ __forceinline__ void store8(uint8_t* base, uint32_t off, const float* v) {
    uint4 q;
    q.x = pack_bf16(v[0], v[1]);
    q.y = pack_bf16(v[2], v[3]);
    q.z = pack_bf16(v[4], v[5]);
    q.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4*>(base + off) = q;
}

// ---------------------------------------------------------------- layout
constexpr uint32_t kSmW = 0;                      // weight images (kImgBytes = 14848)
constexpr uint32_t kSmX = 15360;                  // 2 x 4096
constexpr uint32_t kSmMeta = kSmX + 2 * 4096;     // 2 x 2048
constexpr uint32_t kSmH1 = kSmMeta + 2 * 2048;    // 20480: 10 column blocks
constexpr uint32_t kSmH2 = kSmH1 + 20480;         // 32768: 16 column blocks (MN-major A of dW3)
constexpr uint32_t kSmDO = kSmH2 + 32768;         // 4096
constexpr uint32_t kSmDZ2 = kSmDO + 4096;         // 32768
constexpr uint32_t kSmDZ1 = kSmDZ2 + 32768;       // 32768
constexpr uint32_t kSmBars = kSmDZ1 + 32768;      // 4 mbarriers + TMEM slot
constexpr uint32_t kSmRed = kSmBars + 64;         // 128 floats
constexpr uint32_t kSmBytes = kSmRed + 512 + 1024;  // + alignment slack

// TMEM columns.
constexpr uint32_t kTmD1 = 0, kTmD2 = 64, kTmD3 = 128, kTmDH2 = 160, kTmDH1 = 224;
constexpr uint32_t kTmDW3 = 288, kTmDW2 = 320, kTmDW1 = 416, kTmCols = 512;

struct MlpArgs {
    const uint8_t* x;        // tiles of X, 4096 B each
    const MlpMeta* meta;     // 128 per tile
    const uint8_t* images;   // BF16 weight images (kImgBytes)
    uint32_t rows;           // valid rows (contacts)
    uint32_t tiles;
    const uint32_t* rows_ptr;  // when set, the row count is read here (device counter)
    float* out;              // raw outputs [rows][2] (inference: required)
    float* partial;          // training: [gridDim.x][kMlpParams + 1]
    uint32_t* status;        // status word; status_bit is set when a wait times out
    uint32_t status_bit;
};

template <bool kTrain>
__global__ void __launch_bounds__(128, 1) k_mlp_tiles(MlpArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kSmBars);  // 0,1: X buffers, 2: MMA, 3: weights
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kSmBars + 32);
    float* red = reinterpret_cast<float*>(sm + kSmRed);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, row = tid;
    const uint32_t lane_base = (warp * 32u) << 16;
    if (a.rows_ptr) {
        a.rows = *a.rows_ptr;
        a.tiles = (a.rows + kMlpTile - 1) / kMlpTile;
    }

    if (tid == 0) {
        for (int k = 0; k < 4; ++k) mbar_init(&bar[k], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTrain ? kTmCols : 256u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // Constant columns of this thread's rows: the bias one at column 64 of
    // both hidden tiles, zero padding elsewhere.
    {
        const float one[8] = {1, 0, 0, 0, 0, 0, 0, 0}, zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        store8(sm + kSmH1, tile_offset(row, 64), one);
        store8(sm + kSmH1, tile_offset(row, 72), zero);
        store8(sm + kSmH2, tile_offset(row, 64), one);
        for (uint32_t j = 72; j < 128; j += 8) store8(sm + kSmH2, tile_offset(row, j), zero);
        if (kTrain) {
            store8(sm + kSmDO, tile_offset(row, 0), zero);
            store8(sm + kSmDO, tile_offset(row, 8), zero);
            for (uint32_t j = 64; j < 128; j += 8) {
                store8(sm + kSmDZ2, tile_offset(row, j), zero);
                store8(sm + kSmDZ1, tile_offset(row, j), zero);
            }
        }
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    bool ok = true;
    const uint32_t first = blockIdx.x;
    if (tid == 0) {
        mbar_expect_tx(&bar[3], kImgBytes);
        bulk_load(sm + kSmW, a.images, kImgBytes, &bar[3]);
        if (first < a.tiles) {
            mbar_expect_tx(&bar[0], 4096 + 2048);
            bulk_load(sm + kSmX, a.x + size_t(first) * 4096, 4096, &bar[0]);
            bulk_load(sm + kSmMeta, a.meta + size_t(first) * 128, 2048, &bar[0]);
        }
    }
    ok = __syncthreads_and(mbar_wait(&bar[3], 0)) != 0;

    const uint32_t sW1 = smem_u32(sm + kSmW + kImgW1), sW2 = smem_u32(sm + kSmW + kImgW2),
                   sW3 = smem_u32(sm + kSmW + kImgW3);
    const uint32_t sH1 = smem_u32(sm + kSmH1), sH2 = smem_u32(sm + kSmH2), sDO = smem_u32(sm + kSmDO),
                   sDZ2 = smem_u32(sm + kSmDZ2), sDZ1 = smem_u32(sm + kSmDZ1);
    uint32_t mma_phase = 0;
    float loss = 0.0f, base = 0.0f;  // weighted squared error; the same for a zero prediction
    uint32_t it = 0;
    bool pending = false;  // a prefetch is in flight into the other buffer
    for (uint32_t tile = first; tile < a.tiles && ok; tile += gridDim.x, ++it) {
        const uint32_t buf = it & 1u;
        __syncthreads();
        if (tid == 0 && tile + gridDim.x < a.tiles) {
            const uint32_t next = tile + gridDim.x;
            mbar_expect_tx(&bar[buf ^ 1u], 4096 + 2048);
            bulk_load(sm + kSmX + (buf ^ 1u) * 4096, a.x + size_t(next) * 4096, 4096, &bar[buf ^ 1u]);
            bulk_load(sm + kSmMeta + (buf ^ 1u) * 2048, a.meta + size_t(next) * 128, 2048, &bar[buf ^ 1u]);
        }
        pending = tile + gridDim.x < a.tiles;
        if (!__syncthreads_and(mbar_wait(&bar[buf], (it >> 1) & 1u))) {
            ok = false;
            break;
        }
        const uint32_t sX = smem_u32(sm + kSmX + buf * 4096);
        const MlpMeta meta = reinterpret_cast<const MlpMeta*>(sm + kSmMeta + buf * 2048)[row];

        // ---- layer 1: D1 = X W1^T (bias through X column 8)
        if (tid == 0) {
            tc_after_sync();
            mma(tmem + kTmD1, sdesc(sX, 2048, 128), sdesc(sW1, 1024, 128), idesc(128, 64, 0, 0), 0);
            mma_commit(&bar[2]);
        }
        if (!__syncthreads_and(mbar_wait(&bar[2], mma_phase))) { ok = false; break; }
        mma_phase ^= 1u;
        tc_after_sync();
        uint32_t mask1[2] = {0, 0}, mask2[2] = {0, 0};
        for (uint32_t c = 0; c < 64; c += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + kTmD1 + c, v);
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                if (v[k] > 0.0f) mask1[(c + k) >> 5] |= 1u << ((c + k) & 31u);
                v[k] = fmaxf(v[k], 0.0f);
            }
            store8(sm + kSmH1, tile_offset(row, c), v);
            store8(sm + kSmH1, tile_offset(row, c + 8), v + 8);
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();

        // ---- layer 2: D2 = H1 W2^T (bias through H1 column 64), K = 80
        if (tid == 0) {
            tc_after_sync();
            for (uint32_t c = 0; c < 5; ++c)
                mma(tmem + kTmD2, sdesc(sH1 + c * 4096, 2048, 128), sdesc(sW2 + c * 2048, 1024, 128),
                    idesc(128, 64, 0, 0), c > 0);
            mma_commit(&bar[2]);
        }
        if (!__syncthreads_and(mbar_wait(&bar[2], mma_phase))) { ok = false; break; }
        mma_phase ^= 1u;
        tc_after_sync();
        for (uint32_t c = 0; c < 64; c += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + kTmD2 + c, v);
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                if (v[k] > 0.0f) mask2[(c + k) >> 5] |= 1u << ((c + k) & 31u);
                v[k] = fmaxf(v[k], 0.0f);
            }
            store8(sm + kSmH2, tile_offset(row, c), v);
            store8(sm + kSmH2, tile_offset(row, c + 8), v + 8);
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();

        // ---- layer 3: D3 = H2 W3^T, N = 16 (outputs in columns 0 and 1)
        if (tid == 0) {
            tc_after_sync();
            for (uint32_t c = 0; c < 5; ++c)
                mma(tmem + kTmD3, sdesc(sH2 + c * 4096, 2048, 128), sdesc(sW3 + c * 512, 256, 128),
                    idesc(128, 16, 0, 0), c > 0);
            mma_commit(&bar[2]);
        }
        if (!__syncthreads_and(mbar_wait(&bar[2], mma_phase))) { ok = false; break; }
        mma_phase ^= 1u;
        tc_after_sync();
        float o[16];
        tmem_ld16(tmem + lane_base + kTmD3, o);
        const uint32_t c_row = tile * kMlpTile + row;
        const bool valid = c_row < a.rows;
        if (valid && a.out) {
            a.out[2 * size_t(c_row)] = o[0];
            a.out[2 * size_t(c_row) + 1] = o[1];
        }
        if (!kTrain) continue;

        // ---- backward: squared error on (lambda, penalty), row weights in meta
        const float w = valid ? meta.weight : 0.0f;
        const float e0 = valid ? o[0] - meta.y0 : 0.0f, e1 = valid ? o[1] - meta.y1 : 0.0f;
        loss += w * (e0 * e0 + e1 * e1);
        if (valid) base += w * (meta.y0 * meta.y0 + meta.y1 * meta.y1);
        {
            const float d[8] = {2.0f * w * e0, 2.0f * w * e1, 0, 0, 0, 0, 0, 0};
            store8(sm + kSmDO, tile_offset(row, 0), d);
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc_after_sync();
            // dH2 = dO W3[:, :64]   (B = W3 viewed MN-major: N = hidden, K = output)
            mma(tmem + kTmDH2, sdesc(sDO, 2048, 128), sdesc(sW3, 128, 256), idesc(128, 64, 0, 1), 0);
            // dW3^T += [H2 | 1]^T dO over this tile's 128 rows (K = rows)
            for (uint32_t c = 0; c < 8; ++c)
                mma(tmem + kTmDW3, sdesc(sH2 + c * 256, 128, 2048), sdesc(sDO + c * 256, 128, 2048),
                    idesc(128, 16, 1, 1), (it > 0 || c > 0) ? 1u : 0u);
            mma_commit(&bar[2]);
        }
        if (!__syncthreads_and(mbar_wait(&bar[2], mma_phase))) { ok = false; break; }
        mma_phase ^= 1u;
        tc_after_sync();
        for (uint32_t c = 0; c < 64; c += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + kTmDH2 + c, v);
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if (!((mask2[(c + k) >> 5] >> ((c + k) & 31u)) & 1u)) v[k] = 0.0f;
            store8(sm + kSmDZ2, tile_offset(row, c), v);
            store8(sm + kSmDZ2, tile_offset(row, c + 8), v + 8);
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc_after_sync();
            // dH1 = dZ2 W2[:, :64]   (B = W2 viewed MN-major), K = 64
            for (uint32_t c = 0; c < 4; ++c)
                mma(tmem + kTmDH1, sdesc(sDZ2 + c * 4096, 2048, 128), sdesc(sW2 + c * 256, 128, 1024),
                    idesc(128, 64, 0, 1), c > 0);
            // dW2 += dZ2^T [H1 | 1]  (M = hidden rows, padded to 128; N = 80)
            for (uint32_t c = 0; c < 8; ++c)
                mma(tmem + kTmDW2, sdesc(sDZ2 + c * 256, 128, 2048), sdesc(sH1 + c * 256, 128, 2048),
                    idesc(128, 80, 1, 1), (it > 0 || c > 0) ? 1u : 0u);
            mma_commit(&bar[2]);
        }
        if (!__syncthreads_and(mbar_wait(&bar[2], mma_phase))) { ok = false; break; }
        mma_phase ^= 1u;
        tc_after_sync();
        for (uint32_t c = 0; c < 64; c += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + kTmDH1 + c, v);
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if (!((mask1[(c + k) >> 5] >> ((c + k) & 31u)) & 1u)) v[k] = 0.0f;
            store8(sm + kSmDZ1, tile_offset(row, c), v);
            store8(sm + kSmDZ1, tile_offset(row, c + 8), v + 8);
        }
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc_after_sync();
            // dW1 += dZ1^T X  (N = 16 input columns, bias gradient in column 8)
            for (uint32_t c = 0; c < 8; ++c)
                mma(tmem + kTmDW1, sdesc(sDZ1 + c * 256, 128, 2048), sdesc(sX + c * 256, 128, 2048),
                    idesc(128, 16, 1, 1), (it > 0 || c > 0) ? 1u : 0u);
            mma_commit(&bar[2]);
        }
        if (!__syncthreads_and(mbar_wait(&bar[2], mma_phase))) { ok = false; break; }
        mma_phase ^= 1u;
        tc_after_sync();
    }

    if (kTrain) {
        // Partial gradients of this CTA (zero when it had no tile).
        float* p = a.partial + size_t(blockIdx.x) * kMlpPartial;
        const bool any = it > 0 && ok;
        float v[16] = {};
        if (any) tmem_ld16(tmem + lane_base + kTmDW3, v);
        if (row < kMlpHiddenK)
            for (uint32_t o = 0; o < kMlpOutN; ++o)
                p[kMlpW3 + o * kMlpHiddenK + row] = (any && o < kMlpOut) ? v[o] : 0.0f;
        for (uint32_t c = 0; c < kMlpHiddenK; c += 16) {
            if (any) tmem_ld16(tmem + lane_base + kTmDW2 + c, v);
            if (row < kMlpHidden)
                for (int k = 0; k < 16; ++k) p[kMlpW2 + row * kMlpHiddenK + c + k] = any ? v[k] : 0.0f;
        }
        if (any) tmem_ld16(tmem + lane_base + kTmDW1, v);
        if (row < kMlpHidden)
            for (int k = 0; k < 16; ++k) p[kMlpW1 + row * kMlpIn + k] = any ? v[k] : 0.0f;
        red[row] = loss;
        __syncthreads();
        if (tid == 0) {
            float s = 0.0f;
            for (int k = 0; k < 128; ++k) s += red[k];
            p[kMlpParams] = s;
        }
        __syncthreads();
        red[row] = base;
        __syncthreads();
        if (tid == 0) {
            float s = 0.0f;
            for (int k = 0; k < 128; ++k) s += red[k];
            p[kMlpParams + 1] = s;
        }
    }
    if (!ok) {
        // Leave no bulk copy in flight: wait (bounded) for the prefetch of
        // the buffer the next iteration would have used.
        if (pending) mbar_wait(&bar[it & 1u ^ 1u], ((it + 1) >> 1) & 1u);
        if (tid == 0) atomicOr(a.status, a.status_bit);
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTrain ? kTmCols : 256u));
}

// ---------------------------------------------------------------- features
// One row per contact point, written into its tile's canonical position
// (each feature scaled to order one and clipped to [-5, 5]):
//  0 normal error at the start of the tick / 0.1 m
//  1 closing speed (m/s)
//  2 log1p(plain warm-start lambda / scale) / 2, scale = |g| m_eff,
//    m_eff = 1/(w_a+w_b)
//  3 (log10(plain warm-start penalty) - 6.5) / 0.3
//  4 2 w_b / (w_a + w_b) - 1
//  5 1 if the contact was matched in the cache
//  6 normal . up (up = -g/|g|)
//  7 (log10(m_eff) - 2.7) / 0.25
//  8 constant one (bias)
// The row's metadata keeps the plain warm start in the model's log space in
// FP32 (y0 = log1p(lambda / scale), y1 = log10(penalty)) and the scale: the
// network predicts scaled corrections of them (see kLamOut, kPenOut), so an
// all-zero output layer reproduces the plain warm start exactly.
__global__ void k_mlp_features(Dev d, StepParams sp, uint8_t* x, MlpMeta* meta) {
    const uint32_t nc = d.ctr->n_contacts;
    const uint32_t tiles = (nc + kMlpTile - 1) / kMlpTile;
    const float g = sqrtf(sp.gx * sp.gx + sp.gy * sp.gy + sp.gz * sp.gz);
    const float inv_g = g > 0.0f ? 1.0f / g : 0.0f;
    const V3 up{-sp.gx * inv_g, -sp.gy * inv_g, -sp.gz * inv_g};
    const uint32_t rows = tiles * kMlpTile;
    for (uint32_t c = grid_stride_begin(); c < rows; c += grid_stride()) {
        float f[16] = {};
        MlpMeta m{0.0f, 0.0f, 0.0f, 0.0f};
        if (c < nc) {
            const uint2 ab = d.c_bodies[c];
            const float wa = d.p0[ab.x].x, wb = d.p0[ab.y].x;
            const float wsum = wa + wb;
            const float meff = wsum > 0.0f ? 1.0f / wsum : 1.0f;
            const float scale = fmaxf(g * meff, 1.0e-6f);
            const float4 e = d.c_e[c], lam = d.c_lam[c], pen = d.c_pen[c], n = d.c_n[c], aa = d.c_aa[c];
            const float llam = log1pf(fmaxf(lam.x, 0.0f) / scale), lpen = log10f(fmaxf(pen.x, 1.0f));
            f[0] = e.x * 10.0f;
            f[1] = e.w;
            f[2] = llam * 0.5f;
            f[3] = (lpen - 6.5f) * (1.0f / 0.3f);
            f[4] = wsum > 0.0f ? 2.0f * wb / wsum - 1.0f : 0.0f;
            f[5] = aa.w != 0.0f ? 1.0f : 0.0f;
            f[6] = n.x * up.x + n.y * up.y + n.z * up.z;
            f[7] = (log10f(meff) - 2.7f) * 4.0f;
            for (int k = 0; k < 8; ++k) f[k] = isfinite(f[k]) ? fminf(fmaxf(f[k], -5.0f), 5.0f) : 0.0f;
            f[8] = 1.0f;
            m.y0 = llam;
            m.y1 = lpen;
            m.scale = scale;
        }
        const uint32_t tile = c / kMlpTile, r = c % kMlpTile;
        uint8_t* t = x + size_t(tile) * 4096;
        store8(t, tile_offset(r, 0), f);
        store8(t, tile_offset(r, 8), f + 8);
        meta[c] = m;
    }
}

// Training targets from the tick's converged normal rows: the scaled
// corrections that turn the plain warm start into the converged
// (lambda, penalty): y0 = kLamOut * (log1p(lambda / scale) - plain),
// y1 = kPenOut * (log10(penalty) - plain).
__global__ void k_mlp_targets(Dev d, MlpMeta* meta) {
    const uint32_t nc = d.ctr->n_contacts;
    const float w = nc ? 1.0f / float(nc) : 0.0f;
    for (uint32_t c = grid_stride_begin(); c < nc; c += grid_stride()) {
        MlpMeta m = meta[c];
        const float lam = reinterpret_cast<const float*>(d.c_lam + c)[0];
        const float pen = reinterpret_cast<const float*>(d.c_pen + c)[0];
        m.y0 = kLamOut * (log1pf(fmaxf(lam, 0.0f) / m.scale) - m.y0);
        m.y1 = kPenOut * (log10f(fmaxf(pen, 1.0f)) - m.y1);
        m.weight = (isfinite(m.y0) && isfinite(m.y1)) ? w : 0.0f;
        if (m.weight == 0.0f) m.y0 = m.y1 = 0.0f;
        meta[c] = m;
    }
}

// Learned warm start from the network's outputs (scaled corrections of the
// plain warm start in log space, meta.y0/y1 from k_mlp_features):
//   lambda  = scale * expm1(y0 + o0 / kLamOut)   (mode bit 0)
//   penalty = 10^(y1 + o1 / kPenOut)             (mode bit 1)
// With mode bit 2 the lambda correction of every point of a manifold is the
// mean of its points' corrections, so the split of the pair's normal force
// between its points stays the one the plain warm start carries over.
// Nothing changes while the gate is closed or for non-finite values.
__global__ void k_mlp_apply(Dev d, const MlpMeta* meta, const float* out, uint32_t mode, const float* gate) {
    if (gate && *gate == 0.0f) return;
    const uint32_t n_act = d.ctr->n_act;
    for (uint32_t i = grid_stride_begin(); i < n_act; i += grid_stride()) {
        const uint32_t off = d.act_off[i], cnt = d.act_cnt[i];
        float mean0 = 0.0f;
        for (uint32_t p = 0; p < cnt; ++p) mean0 += out[2 * size_t(off + p)];
        mean0 /= float(cnt > 0 ? cnt : 1);
        for (uint32_t p = 0; p < cnt; ++p) {
            const uint32_t c = off + p;
            const MlpMeta m = meta[c];
            // Trust region: a prediction moves the plain warm start by at most
            // kMaxCorrection in its log space (a factor of 10 in penalty), so
            // an input unlike the training contacts cannot soften or stiffen a
            // contact without bound.
            const float o0 = (mode & 4u) ? mean0 : out[2 * size_t(c)], o1 = out[2 * size_t(c) + 1];
            if (mode & 1u) {
                const float dl = fminf(fmaxf(o0 * (1.0f / kLamOut), -kMaxCorrection), kMaxCorrection);
                const float lam = fmaxf(m.scale * expm1f(m.y0 + dl), 0.0f);
                if (isfinite(lam)) reinterpret_cast<float*>(d.c_lam + c)[0] = lam;
            }
            if (mode & 2u) {
                const float dk = fminf(fmaxf(o1 * (1.0f / kPenOut), -kMaxCorrection), kMaxCorrection);
                const float pen = fminf(fmaxf(exp10f(m.y1 + dk), 1.0f), 1.0e10f);
                if (isfinite(pen)) reinterpret_cast<float*>(d.c_pen + c)[0] = pen;
            }
        }
    }
}

// Rows given directly (features already normalised), for gradient checks.
__global__ void k_mlp_pack_rows(const float* feat, const float* y, const float* weight, uint32_t n, uint8_t* x,
                                MlpMeta* meta, uint32_t tiles) {
    const uint32_t rows = tiles * kMlpTile;
    for (uint32_t c = grid_stride_begin(); c < rows; c += grid_stride()) {
        float f[16] = {};
        MlpMeta m{0.0f, 0.0f, 0.0f, 1.0f};
        if (c < n) {
            for (uint32_t k = 0; k < kMlpFeatures; ++k) f[k] = feat[kMlpFeatures * size_t(c) + k];
            f[8] = 1.0f;
            m.y0 = y[2 * size_t(c)];
            m.y1 = y[2 * size_t(c) + 1];
            m.weight = weight[c];
        }
        const uint32_t tile = c / kMlpTile, r = c % kMlpTile;
        uint8_t* t = x + size_t(tile) * 4096;
        store8(t, tile_offset(r, 0), f);
        store8(t, tile_offset(r, 8), f + 8);
        meta[c] = m;
    }
}

// BF16 images of the master weights in the shared-memory operand layout.
__global__ void k_mlp_images(const float* params, uint8_t* img) {
    for (uint32_t i = grid_stride_begin(); i < kMlpParams; i += grid_stride()) {
        uint32_t off;
        if (i < kMlpW2) {
            off = kImgW1 + img_offset(i / kMlpIn, i % kMlpIn, kMlpHidden);
        } else if (i < kMlpW3) {
            const uint32_t k = i - kMlpW2;
            off = kImgW2 + img_offset(k / kMlpHiddenK, k % kMlpHiddenK, kMlpHidden);
        } else {
            const uint32_t k = i - kMlpW3;
            off = kImgW3 + img_offset(k / kMlpHiddenK, k % kMlpHiddenK, kMlpOutN);
        }
        *reinterpret_cast<__nv_bfloat16*>(img + off) = __float2bfloat16_rn(params[i]);
    }
}

// Sum of the CTAs' partial gradients in CTA order, then one Adam step on the
// FP32 master weights (lr = 0 only sums). With gate set, also opens the
// learned warm start when this step's loss (measured before the update) is
// below 0.9 of the loss of the plain warm start (a zero correction).
__global__ void k_mlp_reduce_adam(const float* partial, uint32_t parts, float* grad, float* params, float* m,
                                  float* v, float lr, float b1, float b2, float c1, float c2, float eps, float* gate) {
    for (uint32_t i = grid_stride_begin(); i < kMlpPartial; i += grid_stride()) {
        float s = 0.0f;
        for (uint32_t p = 0; p < parts; ++p) s += partial[size_t(p) * kMlpPartial + i];
        grad[i] = s;
        if (i >= kMlpParams || lr == 0.0f) continue;
        const float mi = b1 * m[i] + (1.0f - b1) * s;
        const float vi = b2 * v[i] + (1.0f - b2) * s * s;
        m[i] = mi;
        v[i] = vi;
        params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
    if (gate && blockIdx.x == 0 && threadIdx.x == 0) {
        float loss = 0.0f, zero = 0.0f;
        for (uint32_t p = 0; p < parts; ++p) {
            loss += partial[size_t(p) * kMlpPartial + kMlpParams];
            zero += partial[size_t(p) * kMlpPartial + kMlpParams + 1];
        }
        *gate = (zero > 0.0f && loss < 0.9f * zero) ? 1.0f : 0.0f;
    }
}

}  // namespace

// ---------------------------------------------------------------- host side
size_t mlp_smem_bytes() { return kSmBytes; }

int mlp_configure_kernels() {
    if (cudaFuncSetAttribute(k_mlp_tiles<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmBytes)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_tiles<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmBytes)) !=
            cudaSuccess)
        return -1;
    return 0;
}

uint32_t mlp_grid(uint32_t tiles) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1u, std::min(tiles, uint32_t(sms)));
}

void launch_mlp_images(const float* params, uint8_t* img, cudaStream_t s) {
    k_mlp_images<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, img);
    note_launch((kMlpParams + 255) / 256);
}

void launch_mlp_features(const Dev& d, const StepParams& sp, uint8_t* x, MlpMeta* meta, cudaStream_t s) {
    k_mlp_features<<<cap_blocks(d.cap_contact), kBlock, 0, s>>>(d, sp, x, meta);
    note_launch(cap_blocks(d.cap_contact));
}

void launch_mlp_targets(const Dev& d, MlpMeta* meta, cudaStream_t s) {
    k_mlp_targets<<<cap_blocks(d.cap_contact), kBlock, 0, s>>>(d, meta);
    note_launch(cap_blocks(d.cap_contact));
}

void launch_mlp_pack_rows(const float* feat, const float* y, const float* w, uint32_t n, uint8_t* x, MlpMeta* meta,
                          uint32_t tiles, cudaStream_t s) {
    k_mlp_pack_rows<<<blocks_for(tiles * kMlpTile), kBlock, 0, s>>>(feat, y, w, n, x, meta, tiles);
    note_launch(blocks_for(tiles * kMlpTile));
}

void launch_mlp_tiles(bool train, const uint8_t* x, const MlpMeta* meta, const uint8_t* img, uint32_t rows,
                      uint32_t tiles, const uint32_t* rows_ptr, float* out, float* partial, uint32_t* status,
                      uint32_t status_bit, uint32_t grid, cudaStream_t s) {
    MlpArgs a{x, meta, img, rows, tiles, rows_ptr, out, partial, status, status_bit};
    if (train)
        k_mlp_tiles<true><<<grid, 128, kSmBytes, s>>>(a);
    else
        k_mlp_tiles<false><<<grid, 128, kSmBytes, s>>>(a);
    note_launch(grid);
}

void launch_mlp_apply(const Dev& d, const MlpMeta* meta, const float* out, uint32_t mode, const float* gate,
                      cudaStream_t s) {
    k_mlp_apply<<<cap_blocks(d.cap_pair), kBlock, 0, s>>>(d, meta, out, mode, gate);
    note_launch(cap_blocks(d.cap_pair));
}

void launch_mlp_reduce_adam(const float* partial, uint32_t parts, float* grad, float* params, float* m, float* v,
                            float lr, float b1, float b2, float c1, float c2, float eps, float* gate, cudaStream_t s) {
    k_mlp_reduce_adam<<<(kMlpPartial + 255) / 256, 256, 0, s>>>(partial, parts, grad, params, m, v, lr, b1, b2, c1,
                                                                 c2, eps, gate);
    note_launch((kMlpPartial + 255) / 256);
}

}  // namespace pmb

// SPDX-License-Identifier: MIT
// First-fit colouring of a caller-supplied graph that allocates no memory.
//
// Some callers of this library cannot call cudaMalloc: a pm* driver runs on
// memory the application binds to it (the application owns every memory
// object and the driver only receives ranges of it), and host threads with a
// real-time deadline cannot afford the device-wide synchronisation an
// allocation may imply. For them pmb_graph_color_noalloc colours a graph with
// working memory that lives in this file's static device array, so the call
// needs nothing but the caller's input and output buffers.
//
// The colouring is the one the tick computes for its constraint graph: every
// dynamic vertex, in index order, takes the smallest colour absent among its
// lower-index dynamic neighbours (the reference's serial greedy colouring,
// geometry_constraints.slang:1520-1558). It is found as the fixpoint of
// "colour(v) = mex(colours of lower neighbours)" by a cooperative kernel.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/pmb200_core.h"
#include "pmb_world.cuh"

namespace pmb {
namespace {

constexpr uint32_t kNoAllocMaxVertices = 1u << 20;  // 4 MiB of working colours
constexpr uint32_t kHeaderWords = 64;               // barrier, counters, status
enum : uint32_t { kHBarCount = 0, kHBarGen = 1, kHChanged = 2, kHRounds = 3, kHStatus = 4 };

// Working memory of every call on a device: header words, then one working
// colour per vertex. Every GPU that loads the library holds it until exit.
static __device__ __align__(256) uint32_t g_color_scratch[kHeaderWords + kNoAllocMaxVertices];

struct DeviceScratch {
    bool ready{};
    uint32_t* ptr{};
};
constexpr int kMaxDevices = 64;
DeviceScratch g_device_scratch[kMaxDevices];
std::mutex g_scratch_mutex;

// Bounded grid barrier over the header words (cooperative launch only).
__device__ bool barrier(uint32_t* h) {
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        ok = 1;
        volatile uint32_t* gen = h + kHBarGen;
        const uint32_t g = *gen;
        __threadfence();
        if (atomicAdd(h + kHBarCount, 1u) == gridDim.x - 1) {
            h[kHBarCount] = 0;
            __threadfence();
            atomicAdd(h + kHBarGen, 1u);
        } else {
            uint32_t spins = 0;
            while (*gen == g) {
                if (++spins > (1u << 26)) {
                    atomicOr(h + kHStatus, 2u);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

__global__ void k_color_noalloc(const uint32_t* offsets, const uint32_t* neighbors, const uint32_t* dynamic,
                                uint32_t n, uint32_t* colors, uint32_t* scratch) {
    uint32_t* h = scratch;
    volatile uint32_t* work = scratch + kHeaderWords;
    const uint32_t begin = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (uint32_t v = begin; v < n; v += stride) work[v] = dynamic[v] ? 0u : kInvalid;
    // The change counter is read by one thread per block and shared.
    __shared__ uint32_t s_before, s_after;
    for (uint32_t round = 0; round < n + 2; ++round) {
        if (threadIdx.x == 0) s_before = ((volatile uint32_t*)h)[kHChanged];
        if (!barrier(h)) return;
        const uint32_t before = s_before;
        uint32_t changes = 0;
        bool overflow = false;
        for (uint32_t v = begin; v < n; v += stride) {
            if (!dynamic[v]) continue;
            uint64_t mask[4] = {0, 0, 0, 0};
            for (uint32_t k = offsets[v]; k < offsets[v + 1]; ++k) {
                const uint32_t u = neighbors[k];
                if (u < v && u < n && dynamic[u]) {
                    const uint32_t c = work[u];
                    if (c < 256) mask[c >> 6] |= 1ull << (c & 63);
                }
            }
            uint32_t col = 255;
            bool found = false;
            for (int w = 0; w < 4 && !found; ++w)
                if (~mask[w]) {
                    col = uint32_t(w * 64 + __ffsll((long long)~mask[w]) - 1);
                    found = true;
                }
            overflow = overflow || !found;
            if (col != work[v]) {
                work[v] = col;
                ++changes;
            }
        }
        if (changes) atomicAdd(h + kHChanged, changes);
        if (!barrier(h)) return;
        if (threadIdx.x == 0) s_after = ((volatile uint32_t*)h)[kHChanged];
        __syncthreads();
        if (s_after == before) {
            // Converged: only this round's mex counts. A vertex may pass 255
            // lower-neighbour colours in an intermediate round of the
            // fixpoint and still settle below 256.
            if (overflow) atomicOr(h + kHStatus, 1u);
            if (begin == 0) h[kHRounds] = round + 1;
            for (uint32_t v = begin; v < n; v += stride) colors[v] = work[v];
            return;
        }
    }
    if (begin == 0) atomicOr(h + kHStatus, 4u);
}

}  // namespace
}  // namespace pmb

using namespace pmb;

extern "C" int pmb_graph_color_noalloc(const uint32_t* offsets, const uint32_t* neighbors, const uint32_t* dynamic,
                                       uint32_t vertex_count, uint32_t* colors, int32_t device, void* stream) {
    if (!offsets || !neighbors || !dynamic || !colors) return PMB_ERROR_INVALID_ARGUMENT;
    if (vertex_count > kNoAllocMaxVertices) {
        std::fprintf(stderr,
                     "pmb_graph_color_noalloc: %u vertices exceed the fixed working memory of %u vertices\n",
                     vertex_count, kNoAllocMaxVertices);
        return PMB_ERROR_CAPACITY_EXCEEDED;
    }
    if (device < 0 || device >= kMaxDevices) return PMB_ERROR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The call reads its status back and waits for the stream, which a stream
    // being captured into a graph cannot do: refuse before enqueuing anything
    // (enqueuing would invalidate the caller's capture).
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &capturing) != cudaSuccess || capturing != cudaStreamCaptureStatusNone)
        return PMB_ERROR_INVALID_ARGUMENT;
    // The caller's current device is put back on every return.
    int previous = -1;
    if (cudaGetDevice(&previous) != cudaSuccess) return PMB_ERROR_NO_DEVICE;
    struct Restore {
        int dev;
        ~Restore() { cudaSetDevice(dev); }
    } restore{previous};
    if (cudaSetDevice(device) != cudaSuccess) return PMB_ERROR_NO_DEVICE;
    uint32_t* scratch = nullptr;
    {
        // Once per device, with that device current: resolve the device
        // address of the static working array (host code cannot name it).
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        DeviceScratch& ds = g_device_scratch[device];
        if (!ds.ready) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_color_scratch) != cudaSuccess || !p) {
                std::fprintf(stderr, "pmb_graph_color_noalloc: cannot resolve the working array on device %d\n",
                             device);
                return PMB_ERROR_DEVICE_LOST;
            }
            ds.ptr = static_cast<uint32_t*>(p);
            ds.ready = true;
        }
        scratch = ds.ptr;
    }
    if (vertex_count == 0) return PMB_SUCCESS;
    // The header (barrier, counters, status) must start at zero; the working
    // colours are initialised by the kernel.
    if (cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * kHeaderWords, s) != cudaSuccess) return PMB_ERROR_DEVICE_LOST;
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_color_noalloc, kBlock, 0);
    const uint32_t want = (vertex_count + kBlock - 1) / kBlock;
    const int blocks = int(std::min<uint32_t>(want, uint32_t(std::max(1, per) * sms)));
    uint32_t n = vertex_count;
    void* args[] = {const_cast<uint32_t**>(&offsets), const_cast<uint32_t**>(&neighbors),
                    const_cast<uint32_t**>(&dynamic), &n, &colors, &scratch};
    if (cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&k_color_noalloc), dim3(blocks), dim3(kBlock), args,
                                    0, s) != cudaSuccess)
        return PMB_ERROR_DEVICE_LOST;
    note_launch(uint32_t(blocks));
    uint32_t status = 0;
    if (cudaMemcpyAsync(&status, scratch + kHStatus, sizeof(status), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return PMB_ERROR_DEVICE_LOST;
    if (status & 1u) return PMB_ERROR_CAPACITY_EXCEEDED;  // more than 256 colours
    if (status & 6u) return PMB_ERROR_DEVICE_LOST;        // barrier or round limit reached
    return PMB_SUCCESS;
}

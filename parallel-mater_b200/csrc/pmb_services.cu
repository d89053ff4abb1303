// SPDX-License-Identifier: MIT
// Device services for the pm* driver: device enumeration, memory objects,
// copies, streams and events. The driver reaches CUDA only through these so
// that one CUDA runtime (this library's) serves the whole process; they play
// the part of the reference's device::Services (src/device/services.hpp).
#include <cstring>

#include "../../include/pmb200_core.h"
#include "pmb_world.cuh"

namespace {
int status_of(cudaError_t e) {
    if (e == cudaSuccess) return PMB_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return PMB_ERROR_OUT_OF_DEVICE_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return PMB_ERROR_NO_DEVICE;
    if (e == cudaErrorInvalidValue || e == cudaErrorInvalidDevice) return PMB_ERROR_INVALID_ARGUMENT;
    return PMB_ERROR_DEVICE_LOST;
}
}  // namespace

extern "C" {

int pmb_device_count(int32_t* count) {
    if (!count) return PMB_ERROR_INVALID_ARGUMENT;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
    *count = n;
    return PMB_SUCCESS;
}

int pmb_device_info(int32_t device, pmb_device_info_t* info) {
    if (!info) return PMB_ERROR_INVALID_ARGUMENT;
    cudaDeviceProp p{};
    int r = status_of(cudaGetDeviceProperties(&p, device));
    if (r != PMB_SUCCESS) return r;
    std::memset(info, 0, sizeof(*info));
    std::strncpy(info->name, p.name, sizeof(info->name) - 1);
    std::memcpy(info->uuid, &p.uuid, 16);
    info->total_memory = p.totalGlobalMem;
    info->multiprocessors = uint32_t(p.multiProcessorCount);
    info->compute_major = uint32_t(p.major);
    info->compute_minor = uint32_t(p.minor);
    info->pci_device = uint32_t(p.pciDeviceID);
    int driver = 0;
    cudaDriverGetVersion(&driver);
    info->driver_version = uint32_t(driver);
    return PMB_SUCCESS;
}

int pmb_device_memory_info(int32_t device, uint64_t* free_bytes, uint64_t* total_bytes) {
    if (!free_bytes || !total_bytes) return PMB_ERROR_INVALID_ARGUMENT;
    int r = status_of(cudaSetDevice(device));
    if (r != PMB_SUCCESS) return r;
    size_t f = 0, t = 0;
    r = status_of(cudaMemGetInfo(&f, &t));
    *free_bytes = f;
    *total_bytes = t;
    return r;
}

int pmb_device_alloc(int32_t device, uint64_t bytes, int host_visible, void** out) {
    if (!out || bytes == 0) return PMB_ERROR_INVALID_ARGUMENT;
    *out = nullptr;
    int r = status_of(cudaSetDevice(device));
    if (r != PMB_SUCCESS) return r;
    // Host-visible memory is managed memory: device-local when the GPU
    // touches it, readable and writable by host code through one pointer.
    cudaError_t e = host_visible ? cudaMallocManaged(out, size_t(bytes), cudaMemAttachGlobal)
                                 : cudaMalloc(out, size_t(bytes));
    if (e != cudaSuccess) {
        *out = nullptr;
        return e == cudaErrorMemoryAllocation ? PMB_ERROR_OUT_OF_DEVICE_MEMORY : status_of(e);
    }
    return PMB_SUCCESS;
}

int pmb_device_free(int32_t device, void* ptr) {
    if (!ptr) return PMB_SUCCESS;
    cudaSetDevice(device);
    return status_of(cudaFree(ptr));
}

int pmb_stream_create(int32_t device, void** stream) {
    if (!stream) return PMB_ERROR_INVALID_ARGUMENT;
    int r = status_of(cudaSetDevice(device));
    if (r != PMB_SUCCESS) return r;
    cudaStream_t s = nullptr;
    r = status_of(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream = s;
    return r;
}

int pmb_stream_destroy(int32_t device, void* stream) {
    cudaSetDevice(device);
    return status_of(cudaStreamDestroy(static_cast<cudaStream_t>(stream)));
}

int pmb_stream_synchronize(int32_t device, void* stream) {
    cudaSetDevice(device);
    return status_of(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
}

int pmb_copy_async(int32_t device, void* dst, const void* src, uint64_t bytes, void* stream) {
    if (bytes == 0) return PMB_SUCCESS;
    if (!dst || !src) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(device);
    return status_of(cudaMemcpyAsync(dst, src, size_t(bytes), cudaMemcpyDefault, static_cast<cudaStream_t>(stream)));
}

int pmb_event_create(int32_t device, void** event) {
    if (!event) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(device);
    cudaEvent_t e = nullptr;
    int r = status_of(cudaEventCreate(&e));
    *event = e;
    return r;
}

int pmb_event_destroy(int32_t device, void* event) {
    cudaSetDevice(device);
    return status_of(cudaEventDestroy(static_cast<cudaEvent_t>(event)));
}

int pmb_event_record(int32_t device, void* event, void* stream) {
    cudaSetDevice(device);
    return status_of(cudaEventRecord(static_cast<cudaEvent_t>(event), static_cast<cudaStream_t>(stream)));
}

int pmb_event_query(int32_t device, void* event, int* ready) {
    if (!ready) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(device);
    cudaError_t e = cudaEventQuery(static_cast<cudaEvent_t>(event));
    *ready = e == cudaSuccess;
    if (e == cudaErrorNotReady) {
        cudaGetLastError();
        return PMB_SUCCESS;
    }
    return status_of(e);
}

int pmb_event_elapsed_ms(int32_t device, void* start, void* end, float* ms) {
    if (!ms) return PMB_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(device);
    cudaEventSynchronize(static_cast<cudaEvent_t>(end));
    return status_of(cudaEventElapsedTime(ms, static_cast<cudaEvent_t>(start), static_cast<cudaEvent_t>(end)));
}

}  // extern "C"

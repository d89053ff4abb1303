// SPDX-License-Identifier: MIT
// libpm_b200_driver.so: a Parallel Mater 0.3 driver for B200 GPUs, rigid
// domain. Exports exactly the four loader entry points of the reference's
// driver ABI (include/parallel_mater/pm_driver.h:34-41, implemented in the
// reference at src/driver/slang/entry.cpp:30-56); every pm* command is
// resolved by name through them.
//
// This file: instance, physical device, device and queue, memory, buffers,
// geometry, physics pipelines, command pools and buffers, submission,
// fences, timeline semaphores, queries. The simulation and the rigid
// commands are in pm_rigid.cpp. Validation and error codes follow the
// reference's src/api/*.cpp command by command.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include "pm_objects.hpp"

#define PM_EXPORT extern "C" PM_B200_DRIVER_API

namespace pmd {

// ---------------------------------------------------------------- worker
void Worker::start() {
    stopping_ = false;
    thread_ = std::thread([this] { run(); });
}

void Worker::stop() {
    {
        std::lock_guard<std::mutex> lock(mutex_);
        stopping_ = true;
    }
    cv_.notify_all();
    if (thread_.joinable()) thread_.join();
}

void Worker::enqueue(std::function<PmResult()> job, CompletionPtr completion) {
    {
        std::lock_guard<std::mutex> lock(mutex_);
        jobs_.emplace_back(std::move(job), std::move(completion));
    }
    cv_.notify_all();
}

void Worker::wait_idle() {
    std::unique_lock<std::mutex> lock(mutex_);
    idle_cv_.wait(lock, [&] { return jobs_.empty() && !busy_; });
}

void Worker::run() {
    for (;;) {
        std::pair<std::function<PmResult()>, CompletionPtr> job;
        {
            std::unique_lock<std::mutex> lock(mutex_);
            cv_.wait(lock, [&] { return stopping_ || !jobs_.empty(); });
            if (jobs_.empty()) return;  // stopping and drained
            job = std::move(jobs_.front());
            jobs_.pop_front();
            busy_ = true;
        }
        PmResult r = PM_ERROR_INVALID_STATE;
        try {
            r = job.first();
        } catch (const std::bad_alloc&) {
            r = PM_ERROR_OUT_OF_HOST_MEMORY;
        } catch (...) {
            r = PM_ERROR_INVALID_STATE;
        }
        if (job.second) job.second->finish(r);
        {
            std::lock_guard<std::mutex> lock(mutex_);
            busy_ = false;
        }
        idle_cv_.notify_all();
    }
}

PmResult from_core(int status) {
    switch (status) {
    case PMB_SUCCESS: return PM_SUCCESS;
    case PMB_ERROR_INVALID_ARGUMENT: return PM_ERROR_INVALID_ARGUMENT;
    case PMB_ERROR_OUT_OF_DEVICE_MEMORY: return PM_ERROR_OUT_OF_DEVICE_MEMORY;
    case PMB_ERROR_FEATURE_NOT_PRESENT: return PM_ERROR_FEATURE_NOT_PRESENT;
    case PMB_ERROR_CAPACITY_EXCEEDED: return PM_ERROR_CAPACITY_EXCEEDED;
    case PMB_ERROR_NO_DEVICE: return PM_ERROR_DEVICE_LOST;
    default: return PM_ERROR_DEVICE_LOST;
    }
}

// A command buffer whose submission completed is executable again (or
// initial, for one-time buffers).
void refresh_command_state(PmCommandBuffer_T* buffer) {
    if (!buffer || buffer->state != CommandState::pending || !buffer->completion) return;
    if (buffer->completion->status() == PM_NOT_READY) return;
    buffer->state = (buffer->usage & PM_COMMAND_BUFFER_ONE_TIME_BIT) ? CommandState::initial : CommandState::executable;
    buffer->completion.reset();
}

PmResult require_recording(PmCommandBuffer_T* buffer) {
    if (buffer == nullptr) return PM_ERROR_INVALID_ARGUMENT;
    if (buffer->state != CommandState::recording) return PM_ERROR_INVALID_STATE;
    if (buffer->latched != PM_SUCCESS) return buffer->latched;
    return PM_SUCCESS;
}

PmResult record(PmCommandBuffer_T* buffer, std::function<PmResult()> command) {
#if defined(PMB_TEST_FAILURE_DRIVER)
    // Test build only (reference src/api/internal.hpp:375-381): a recording
    // allocation failure, latched until the buffer is begun again.
    if (std::getenv("PM_TEST_FAIL_RECORDING") != nullptr) {
        buffer->latched = PM_ERROR_OUT_OF_HOST_MEMORY;
        return buffer->latched;
    }
#endif
    try {
        buffer->commands.push_back(std::move(command));
    } catch (const std::bad_alloc&) {
        buffer->latched = PM_ERROR_OUT_OF_HOST_MEMORY;
        return buffer->latched;
    }
    return PM_SUCCESS;
}

PmResult record_simulation(PmCommandBuffer_T* buffer, PmSimulation_T* simulation, std::function<PmResult()> command) {
    const PmResult r = record(buffer, std::move(command));
    if (r != PM_SUCCESS) return r;
    if (std::find(buffer->simulations.begin(), buffer->simulations.end(), simulation) == buffer->simulations.end())
        buffer->simulations.push_back(simulation);
    return PM_SUCCESS;
}

PmResult record_query(PmCommandBuffer_T* buffer, PmQueryPool_T* pool, uint32_t first, uint32_t count,
                      std::function<PmResult()> command) {
    const PmResult r = record(buffer, std::move(command));
    if (r != PM_SUCCESS) return r;
    buffer->query_writes.push_back({pool, first, count});
    return PM_SUCCESS;
}

namespace {

Clock::time_point deadline_after(uint64_t timeout_ns) {
    if (timeout_ns == PM_TIMEOUT_INFINITE || timeout_ns > uint64_t(INT64_MAX) / 2) return Clock::time_point::max();
    return Clock::now() + std::chrono::nanoseconds(int64_t(timeout_ns));
}

// Timeline bookkeeping: completed signals advance the value.
void refresh_timeline_locked(PmSemaphore_T* s) {
    while (!s->signals.empty()) {
        auto first = s->signals.begin();
        if (first->second->status() != PM_SUCCESS) break;
        s->value = std::max(s->value, first->first);
        s->signals.erase(first);
    }
}

PmResult timeline_status(PmSemaphore_T* s, uint64_t value) {
    std::lock_guard<std::mutex> lock(s->mutex);
    refresh_timeline_locked(s);
    if (s->value >= value) return PM_SUCCESS;
    auto found = s->signals.lower_bound(value);
    if (found == s->signals.end()) return PM_NOT_READY;
    const PmResult r = found->second->status();
    if (r == PM_SUCCESS) s->value = found->first;
    return r;
}

void copy_name(char (&dst)[256], const char* src) {
    const size_t n = strnlen(src, sizeof(dst) - 1);
    std::memcpy(dst, src, n);
    dst[n] = '\0';
}

PmPhysicalDeviceFeatures supported_features() {
    PmPhysicalDeviceFeatures f{};
    f.rigidBodies = PM_TRUE;
    f.rigidConstraints = PM_TRUE;
    f.timelineSemaphores = PM_TRUE;
    f.timestampQueries = PM_TRUE;
    f.statisticsQueries = PM_TRUE;
    f.memoryBudget = PM_TRUE;
    f.contactEvents = PM_TRUE;
    return f;
}

}  // namespace
}  // namespace pmd

using namespace pmd;

// ====================================================================
// instance and physical devices (reference src/api/instance.cpp:420-520,
// src/api/device.cpp)
// ====================================================================
namespace {

PmResult PMAPI_CALL pmEnumerateInstanceVersion(uint32_t* version) {
    if (!version) return PM_ERROR_INVALID_ARGUMENT;
    *version = PM_API_VERSION_0_3;
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmCreateInstance(const PmInstanceCreateInfo* info, const PmAllocationCallbacks* allocator,
                                     PmInstance* instance) {
    if (!instance) return PM_ERROR_INVALID_ARGUMENT;
    *instance = nullptr;
    if (!info || !valid_structure(info->sType, PM_STRUCTURE_TYPE_INSTANCE_CREATE_INFO, info->pNext))
        return PM_ERROR_INVALID_ARGUMENT;
    if (info->apiVersion != 0u && info->apiVersion != PM_API_VERSION_0_3) return PM_ERROR_INCOMPATIBLE_VERSION;
    if (allocator && (!allocator->pfnAllocate || !allocator->pfnFree)) return PM_ERROR_INVALID_ARGUMENT;
    auto* created = new (std::nothrow) PmInstance_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    if (allocator) {
        created->allocator = *allocator;
        created->has_allocator = true;
    }
    int32_t count = 0;
    pmb_device_count(&count);
    try {
        for (int32_t d = 0; d < count; ++d) {
            auto p = std::make_unique<PmPhysicalDevice_T>();
            p->instance = created;
            p->ordinal = d;
            if (pmb_device_info(d, &p->info) != PMB_SUCCESS) continue;
            created->physical.push_back(std::move(p));
        }
    } catch (const std::bad_alloc&) {
        delete created;
        return PM_ERROR_OUT_OF_HOST_MEMORY;
    }
    *instance = created;
    return PM_SUCCESS;
}

void PMAPI_CALL pmDestroyInstance(PmInstance instance) { delete instance; }

PmResult PMAPI_CALL pmEnumeratePhysicalDevices(PmInstance instance, uint32_t* count, PmPhysicalDevice* devices) {
    if (!instance || !count) return PM_ERROR_INVALID_ARGUMENT;
    const uint32_t available = uint32_t(instance->physical.size());
    if (!devices) {
        *count = available;
        return PM_SUCCESS;
    }
    const uint32_t written = std::min(*count, available);
    for (uint32_t i = 0; i < written; ++i) devices[i] = instance->physical[i].get();
    *count = written;
    return written == available ? PM_SUCCESS : PM_INCOMPLETE;
}

void PMAPI_CALL pmGetPhysicalDeviceProperties(PmPhysicalDevice physical, PmPhysicalDeviceProperties* properties) {
    if (!properties) return;
    *properties = {};
    if (!physical) return;
    properties->apiVersion = PM_API_VERSION_0_3;
    properties->driverVersion = physical->info.driver_version;
    properties->vendorId = 0x10deu;
    properties->deviceId = physical->info.pci_device;
    std::memcpy(properties->deviceUuid, physical->info.uuid, 16);
    copy_name(properties->deviceName, physical->info.name);
}

PmResult PMAPI_CALL pmGetPhysicalDeviceQueueFamilies(PmPhysicalDevice physical, uint32_t* count,
                                                     PmQueueFamilyProperties* properties) {
    if (!physical || !count) return PM_ERROR_INVALID_ARGUMENT;
    if (!properties) {
        *count = 1;
        return PM_SUCCESS;
    }
    if (*count == 0) return PM_INCOMPLETE;
    properties[0] = {PM_QUEUE_PHYSICS_BIT | PM_QUEUE_TRANSFER_BIT, 1u, 64u, 1.0f};
    *count = 1;
    return PM_SUCCESS;
}

void PMAPI_CALL pmGetPhysicalDeviceFeatures(PmPhysicalDevice physical, PmPhysicalDeviceFeatures* features) {
    if (!features) return;
    *features = {};
    if (!physical) return;
    *features = supported_features();
}

void PMAPI_CALL pmGetPhysicalDeviceMemoryProperties(PmPhysicalDevice physical, PmMemoryProperties* properties) {
    if (!properties) return;
    *properties = {};
    if (!physical) return;
    // One HBM heap; type 0 device-local, type 1 device-local and host-visible
    // (managed memory), as the reference's CUDA backend advertises
    // (src/api/device.cpp:101-114).
    properties->heapCount = 1;
    properties->heaps[0] = {physical->info.total_memory, PM_MEMORY_DEVICE_LOCAL_BIT};
    properties->typeCount = 2;
    properties->types[0] = {PM_MEMORY_DEVICE_LOCAL_BIT, 0u};
    properties->types[1] = {PM_MEMORY_DEVICE_LOCAL_BIT | PM_MEMORY_HOST_VISIBLE_BIT | PM_MEMORY_HOST_COHERENT_BIT, 0u};
}

PmResult PMAPI_CALL pmCreateDevice(PmPhysicalDevice physical, const PmDeviceCreateInfo* info, PmDevice* device) {
    if (!device) return PM_ERROR_INVALID_ARGUMENT;
    *device = nullptr;
    if (!physical || !info || !valid_structure(info->sType, PM_STRUCTURE_TYPE_DEVICE_CREATE_INFO, info->pNext))
        return PM_ERROR_INVALID_ARGUMENT;
    if (info->queueCreateInfoCount > 1 || (info->queueCreateInfoCount == 1 && !info->pQueueInfos))
        return PM_ERROR_INVALID_ARGUMENT;
    if (info->queueCreateInfoCount == 1 &&
        (info->pQueueInfos[0].queueFamilyIndex != 0u || info->pQueueInfos[0].queueCount != 1u))
        return PM_ERROR_INVALID_ARGUMENT;
    if (info->enabledExtensionCount != 0) return PM_ERROR_EXTENSION_NOT_PRESENT;
    // Every requested feature must be supported.
    const PmPhysicalDeviceFeatures have = supported_features();
    const PmBool32* want = &info->enabledFeatures.rigidBodies;
    const PmBool32* can = &have.rigidBodies;
    for (size_t k = 0; k < sizeof(PmPhysicalDeviceFeatures) / sizeof(PmBool32); ++k)
        if (want[k] == PM_TRUE && can[k] != PM_TRUE) return PM_ERROR_FEATURE_NOT_PRESENT;
    auto* created = new (std::nothrow) PmDevice_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    created->physical = physical;
    created->ordinal = physical->ordinal;
    created->enabled = info->enabledFeatures;
    created->queue.device = created;
    if (pmb_stream_create(created->ordinal, &created->stream) != PMB_SUCCESS ||
        pmb_event_create(created->ordinal, &created->epoch) != PMB_SUCCESS ||
        pmb_event_record(created->ordinal, created->epoch, created->stream) != PMB_SUCCESS) {
        if (created->epoch) pmb_event_destroy(created->ordinal, created->epoch);
        if (created->stream) pmb_stream_destroy(created->ordinal, created->stream);
        delete created;
        return PM_ERROR_DEVICE_LOST;
    }
    created->worker.start();
    *device = created;
    return PM_SUCCESS;
}

void PMAPI_CALL pmDestroyDevice(PmDevice device) {
    if (!device) return;
    device->worker.wait_idle();
    device->worker.stop();
    pmb_stream_synchronize(device->ordinal, device->stream);
    pmb_event_destroy(device->ordinal, device->epoch);
    pmb_stream_destroy(device->ordinal, device->stream);
    delete device;
}

void PMAPI_CALL pmGetDeviceQueue(PmDevice device, uint32_t family, uint32_t index, PmQueue* queue) {
    if (!queue) return;
    *queue = (device && family == 0u && index == 0u) ? &device->queue : nullptr;
}

// ====================================================================
// memory and buffers (reference src/api/memory.cpp)
// ====================================================================
PmResult PMAPI_CALL pmAllocateMemory(PmDevice device, const PmMemoryAllocateInfo* info, PmDeviceMemory* memory) {
    if (!memory) return PM_ERROR_INVALID_ARGUMENT;
    *memory = nullptr;
    if (!device || !info || !valid_structure(info->sType, PM_STRUCTURE_TYPE_MEMORY_ALLOCATE_INFO, info->pNext) ||
        info->allocationSize == 0u || info->memoryTypeIndex > 1u)
        return PM_ERROR_INVALID_ARGUMENT;
#if defined(PMB_TEST_FAILURE_DRIVER)
    // Test build only (reference src/device/cpu_device.cpp:119-122): a device
    // allocation failure that publishes no handle.
    if (std::getenv("PM_TEST_FAIL_ALLOCATION") != nullptr) return PM_ERROR_OUT_OF_DEVICE_MEMORY;
#endif
    auto* created = new (std::nothrow) PmDeviceMemory_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    const int r = pmb_device_alloc(device->ordinal, info->allocationSize, info->memoryTypeIndex == 1u ? 1 : 0,
                                   &created->ptr);
    if (r != PMB_SUCCESS) {
        delete created;
        return r == PMB_ERROR_OUT_OF_DEVICE_MEMORY ? PM_ERROR_OUT_OF_DEVICE_MEMORY : from_core(r);
    }
    created->device = device;
    created->size = info->allocationSize;
    created->type = info->memoryTypeIndex;
    device->application_bytes += info->allocationSize;
    *memory = created;
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmDeviceWaitIdle(PmDevice device);

void PMAPI_CALL pmFreeMemory(PmDevice device, PmDeviceMemory memory) {
    if (!device || !memory || memory->device != device) return;
    (void)pmDeviceWaitIdle(device);
    pmb_device_free(device->ordinal, memory->ptr);
    device->application_bytes -= memory->size;
    delete memory;
}

PmResult PMAPI_CALL pmMapMemory(PmDevice device, PmDeviceMemory memory, PmDeviceSize offset, PmDeviceSize size,
                                void** data) {
    if (!data) return PM_ERROR_INVALID_ARGUMENT;
    *data = nullptr;
    if (!device || !memory || memory->device != device || memory->type != 1u) return PM_ERROR_INVALID_ARGUMENT;
    size = resolved_size(offset, size, memory->size);
    if (!range_fits(offset, size, memory->size)) return PM_ERROR_INVALID_ARGUMENT;
    if (memory->mapped) return PM_ERROR_INVALID_STATE;
    memory->mapped = true;
    *data = static_cast<char*>(memory->ptr) + offset;
    return PM_SUCCESS;
}

void PMAPI_CALL pmUnmapMemory(PmDevice device, PmDeviceMemory memory) {
    if (device && memory && memory->device == device) memory->mapped = false;
}

PmResult check_ranges(PmDevice device, uint32_t count, const PmMappedMemoryRange* ranges, bool need_mapped) {
    if (!device || (count && !ranges)) return PM_ERROR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < count; ++i) {
        const PmMappedMemoryRange& r = ranges[i];
        if (!r.memory || r.memory->device != device || r.memory->type != 1u ||
            (need_mapped && !r.memory->mapped) ||
            !range_fits(r.offset, resolved_size(r.offset, r.size, r.memory->size), r.memory->size))
            return PM_ERROR_INVALID_ARGUMENT;
    }
    return PM_SUCCESS;
}

// Host-visible memory is coherent managed memory: flushing and invalidating
// only validate their ranges.
PmResult PMAPI_CALL pmFlushMappedMemoryRanges(PmDevice device, uint32_t count, const PmMappedMemoryRange* ranges) {
    return check_ranges(device, count, ranges, false);
}

PmResult PMAPI_CALL pmInvalidateMappedMemoryRanges(PmDevice device, uint32_t count,
                                                   const PmMappedMemoryRange* ranges) {
    return check_ranges(device, count, ranges, true);
}

PmResult PMAPI_CALL pmCreateBuffer(PmDevice device, const PmBufferCreateInfo* info, PmBuffer* buffer) {
    if (!buffer) return PM_ERROR_INVALID_ARGUMENT;
    *buffer = nullptr;
    if (!device || !info || !valid_structure(info->sType, PM_STRUCTURE_TYPE_BUFFER_CREATE_INFO, info->pNext) ||
        info->size == 0u || info->initialQueueFamilyIndex != 0u)
        return PM_ERROR_INVALID_ARGUMENT;
    auto* created = new (std::nothrow) PmBuffer_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    created->device = device;
    created->size = info->size;
    created->usage = info->usage;
    created->queue_family = info->initialQueueFamilyIndex;
    *buffer = created;
    return PM_SUCCESS;
}

void PMAPI_CALL pmDestroyBuffer(PmDevice device, PmBuffer buffer) {
    if (!device || !buffer || buffer->device != device) return;
    (void)pmDeviceWaitIdle(device);
    delete buffer;
}

void PMAPI_CALL pmGetBufferMemoryRequirements(PmDevice device, PmBuffer buffer, PmMemoryRequirements* req) {
    if (!req) return;
    *req = {};
    if (!device || !buffer || buffer->device != device) return;
    req->size = buffer->size;
    req->alignment = 256u;
    req->memoryTypeBits = 0x3u;
}

PmResult PMAPI_CALL pmBindBufferMemory(PmDevice device, PmBuffer buffer, PmDeviceMemory memory, PmDeviceSize offset) {
    if (!device || !buffer || !memory || buffer->device != device || memory->device != device || offset % 256u ||
        !range_fits(offset, buffer->size, memory->size))
        return PM_ERROR_INVALID_ARGUMENT;
    if (buffer->memory) return PM_ERROR_INVALID_STATE;
    buffer->memory = memory;
    buffer->offset = offset;
    buffer->ptr = static_cast<char*>(memory->ptr) + offset;
    return PM_SUCCESS;
}

// ====================================================================
// geometry (reference src/api/resources.cpp:182-203, 456-533)
// ====================================================================
bool view_fits(PmDevice device, const PmBufferView& view, PmFormat format, uint32_t element) {
    const PmBuffer_T* b = view.range.buffer;
    if (!b || b->device != device || !b->memory || view.format != format || view.count == 0u ||
        (view.stride != 0u && view.stride != element))
        return false;
    const PmDeviceSize size = resolved_size(view.range.offset, view.range.size, b->size);
    return range_fits(view.range.offset, size, b->size) && PmDeviceSize(view.count) * element <= size;
}

PmResult PMAPI_CALL pmCreateGeometry(PmDevice device, const PmGeometryCreateInfo* info, PmGeometry* geometry) {
    if (!geometry) return PM_ERROR_INVALID_ARGUMENT;
    *geometry = nullptr;
    if (!device || !info || !valid_structure(info->sType, PM_STRUCTURE_TYPE_GEOMETRY_CREATE_INFO, info->pNext) ||
        info->queueFamilyIndex != 0u || !view_fits(device, info->vertices, PM_FORMAT_R32G32B32_SFLOAT, 12u) ||
        !view_fits(device, info->indices, PM_FORMAT_R32_UINT, 4u) || info->indices.count % 3u)
        return PM_ERROR_INVALID_ARGUMENT;
    auto* created = new (std::nothrow) PmGeometry_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    created->device = device;
    created->info = *info;
    // Room for the vertices, the reordered indices and one plane per
    // triangle; host-visible like the reference's geometry storage.
    const PmDeviceSize bytes = PmDeviceSize(info->vertices.count) * 16u + PmDeviceSize(info->indices.count) * 4u +
                               PmDeviceSize(info->indices.count / 3u) * 16u + 256u;
    created->requirements = {(bytes + 255u) & ~PmDeviceSize(255u), 256u, 0x2u, PM_FALSE};
    *geometry = created;
    return PM_SUCCESS;
}

void PMAPI_CALL pmDestroyGeometry(PmDevice device, PmGeometry geometry) {
    if (!device || !geometry || geometry->device != device) return;
    (void)pmDeviceWaitIdle(device);
    delete geometry;
}

void PMAPI_CALL pmGetGeometryMemoryRequirements(PmDevice device, PmGeometry geometry, PmMemoryRequirements* req) {
    if (!req) return;
    *req = {};
    if (!device || !geometry || geometry->device != device) return;
    *req = geometry->requirements;
}

PmResult PMAPI_CALL pmBindGeometryMemory(PmDevice device, PmGeometry geometry, PmDeviceMemory memory,
                                         PmDeviceSize offset) {
    if (!device || !geometry || !memory || geometry->device != device || memory->device != device || offset % 256u)
        return PM_ERROR_INVALID_ARGUMENT;
    if (!(geometry->requirements.memoryTypeBits & (1u << memory->type)) ||
        !range_fits(offset, geometry->requirements.size, memory->size))
        return PM_ERROR_INVALID_ARGUMENT;
    if (geometry->memory) return PM_ERROR_INVALID_STATE;
    geometry->memory = memory;
    geometry->offset = offset;
    return PM_SUCCESS;
}

// Reads the two views at execution time, checks the indices, and records the
// mesh bounds the rigid bodies' default inertia is derived from.
PmResult PMAPI_CALL pmCmdBuildGeometry(PmCommandBuffer buffer, PmGeometry geometry) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!geometry || geometry->device != buffer->device || !geometry->memory) return PM_ERROR_INVALID_ARGUMENT;
    PmDevice_T* device = buffer->device;
    return record(buffer, [geometry, device]() -> PmResult {
        const PmGeometryCreateInfo& info = geometry->info;
        const uint32_t nv = info.vertices.count, ni = info.indices.count;
        std::vector<float> v(3 * size_t(nv));
        std::vector<uint32_t> idx(ni);
        int r = pmb_stream_synchronize(device->ordinal, device->stream);
        if (r == PMB_SUCCESS)
            r = pmb_copy_async(device->ordinal, v.data(), info.vertices.range.buffer->ptr + info.vertices.range.offset,
                               12u * uint64_t(nv), device->stream);
        if (r == PMB_SUCCESS)
            r = pmb_copy_async(device->ordinal, idx.data(), info.indices.range.buffer->ptr + info.indices.range.offset,
                               4u * uint64_t(ni), device->stream);
        if (r == PMB_SUCCESS) r = pmb_stream_synchronize(device->ordinal, device->stream);
        if (r != PMB_SUCCESS) return from_core(r);
        for (uint32_t k = 0; k < ni; ++k)
            if (idx[k] >= nv) return PM_ERROR_INVALID_ARGUMENT;
        for (float x : v)
            if (!std::isfinite(x)) return PM_ERROR_INVALID_ARGUMENT;
        std::vector<uint32_t> order(ni);
        std::vector<float> planes(4 * size_t(ni / 3 + 1));
        float bounds[10];
        int convex = 0;
        r = pmb_prepare_mesh(v.data(), nv, idx.data(), ni, order.data(), planes.data(), bounds, &convex);
        if (r != PMB_SUCCESS) return from_core(r);
        geometry->vertices = std::move(v);
        geometry->indices = std::move(idx);
        for (int k = 0; k < 3; ++k) {
            geometry->lo[k] = bounds[k];
            geometry->hi[k] = bounds[3 + k];
        }
        geometry->built = true;
        return PM_SUCCESS;
    });
}

// ====================================================================
// physics pipelines (reference src/api/pipeline.cpp)
// ====================================================================
PmResult PMAPI_CALL pmCreatePhysicsPipeline(PmDevice device, const PmPhysicsPipelineCreateInfo* info,
                                            PmPhysicsPipeline* pipeline) {
    if (!pipeline) return PM_ERROR_INVALID_ARGUMENT;
    *pipeline = nullptr;
    if (!device || !info ||
        !valid_structure(info->sType, PM_STRUCTURE_TYPE_PHYSICS_PIPELINE_CREATE_INFO, info->pNext))
        return PM_ERROR_INVALID_ARGUMENT;
    if (info->fluidMaterialCount || info->couplingCount || info->clothMaterialCount || info->ropeMaterialCount ||
        info->softBodyMaterialCount || info->smokeMaterialCount)
        return PM_ERROR_FEATURE_NOT_PRESENT;
    PmRigidSolverState rigid{10u, PM_FALSE, 0.02f, 0.02f, 0.5f};
    if (info->pRigidState) {
        rigid = *info->pRigidState;
        if (rigid.rigidIterations == 0u || rigid.rigidIterations > 64u || !std::isfinite(rigid.sleepLinearThreshold) ||
            !std::isfinite(rigid.sleepAngularThreshold) || !std::isfinite(rigid.sleepTimeSeconds) ||
            rigid.sleepLinearThreshold < 0.0f || rigid.sleepAngularThreshold < 0.0f || rigid.sleepTimeSeconds < 0.0f)
            return PM_ERROR_INVALID_ARGUMENT;
    }
    auto* created = new (std::nothrow) PmPhysicsPipeline_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    created->device = device;
    created->rigid = rigid;
    *pipeline = created;
    return PM_SUCCESS;
}

void PMAPI_CALL pmDestroyPhysicsPipeline(PmDevice device, PmPhysicsPipeline pipeline) {
    if (!device || !pipeline || pipeline->device != device) return;
    (void)pmDeviceWaitIdle(device);
    delete pipeline;
}

// ====================================================================
// command pools and buffers (reference src/api/commands.cpp)
// ====================================================================
void clear_recording(PmCommandBuffer_T* b) {
    b->commands.clear();
    b->query_writes.clear();
    b->simulations.clear();
    b->latched = PM_SUCCESS;
    b->bound_pipeline = nullptr;
    b->statistics_open = false;
    b->statistics_pool = nullptr;
    b->statistics_simulation = nullptr;
}

PmResult PMAPI_CALL pmCreateCommandPool(PmDevice device, const PmCommandPoolCreateInfo* info, PmCommandPool* pool) {
    if (!pool) return PM_ERROR_INVALID_ARGUMENT;
    *pool = nullptr;
    if (!device || !info || !valid_structure(info->sType, PM_STRUCTURE_TYPE_COMMAND_POOL_CREATE_INFO, info->pNext) ||
        info->queueFamilyIndex != 0u)
        return PM_ERROR_INVALID_ARGUMENT;
    auto* created = new (std::nothrow) PmCommandPool_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    created->device = device;
    created->flags = info->flags;
    *pool = created;
    return PM_SUCCESS;
}

void PMAPI_CALL pmDestroyCommandPool(PmDevice device, PmCommandPool pool) {
    if (!device || !pool || pool->device != device) return;
    (void)pmDeviceWaitIdle(device);
    for (auto* b : pool->buffers) delete b;
    delete pool;
}

PmResult PMAPI_CALL pmResetCommandPool(PmDevice device, PmCommandPool pool) {
    if (!device || !pool || pool->device != device) return PM_ERROR_INVALID_ARGUMENT;
    for (auto* b : pool->buffers) {
        refresh_command_state(b);
        if (b->state == CommandState::recording || b->state == CommandState::pending) return PM_ERROR_INVALID_STATE;
    }
    for (auto* b : pool->buffers) {
        clear_recording(b);
        b->state = CommandState::initial;
    }
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmAllocateCommandBuffers(PmDevice device, PmCommandPool pool, uint32_t count,
                                             PmCommandBuffer* buffers) {
    if (!device || !pool || pool->device != device || count == 0u || !buffers) return PM_ERROR_INVALID_ARGUMENT;
    std::fill_n(buffers, count, nullptr);
    const size_t previous = pool->buffers.size();
    for (uint32_t i = 0; i < count; ++i) {
        auto* b = new (std::nothrow) PmCommandBuffer_T;
        if (!b) {
            for (size_t k = previous; k < pool->buffers.size(); ++k) delete pool->buffers[k];
            pool->buffers.resize(previous);
            std::fill_n(buffers, count, nullptr);
            return PM_ERROR_OUT_OF_HOST_MEMORY;
        }
        b->device = device;
        b->pool = pool;
        pool->buffers.push_back(b);
        buffers[i] = b;
    }
    return PM_SUCCESS;
}

void PMAPI_CALL pmFreeCommandBuffers(PmDevice device, PmCommandPool pool, uint32_t count,
                                     const PmCommandBuffer* buffers) {
    if (!device || !pool || pool->device != device || (count && !buffers)) return;
    for (uint32_t i = 0; i < count; ++i) {
        PmCommandBuffer_T* b = buffers[i];
        refresh_command_state(b);
        if (!b || b->pool != pool || b->state == CommandState::pending) continue;
        auto found = std::find(pool->buffers.begin(), pool->buffers.end(), b);
        if (found == pool->buffers.end()) continue;
        delete b;
        pool->buffers.erase(found);
    }
}

PmResult PMAPI_CALL pmBeginCommandBuffer(PmCommandBuffer buffer, const PmCommandBufferBeginInfo* info) {
    refresh_command_state(buffer);
    if (!buffer || !info ||
        !valid_structure(info->sType, PM_STRUCTURE_TYPE_COMMAND_BUFFER_BEGIN_INFO, info->pNext) ||
        buffer->state == CommandState::recording || buffer->state == CommandState::pending)
        return PM_ERROR_INVALID_STATE;
    clear_recording(buffer);
    buffer->usage = info->flags;
    buffer->state = CommandState::recording;
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmEndCommandBuffer(PmCommandBuffer buffer) {
    if (!buffer || buffer->state != CommandState::recording) return PM_ERROR_INVALID_STATE;
    if (buffer->latched != PM_SUCCESS) return buffer->latched;
    if (buffer->statistics_open) return PM_ERROR_INVALID_STATE;
    buffer->state = CommandState::executable;
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmResetCommandBuffer(PmCommandBuffer buffer) {
    refresh_command_state(buffer);
    if (!buffer || !buffer->pool || !(buffer->pool->flags & PM_COMMAND_POOL_RESET_BUFFER_BIT) ||
        buffer->state == CommandState::pending)
        return PM_ERROR_INVALID_STATE;
    clear_recording(buffer);
    buffer->state = CommandState::initial;
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmCmdBindPhysicsPipeline(PmCommandBuffer buffer, PmPhysicsPipeline pipeline) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!pipeline || pipeline->device != buffer->device) return PM_ERROR_INVALID_ARGUMENT;
    buffer->bound_pipeline = pipeline;
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmCmdCopyBuffer(PmCommandBuffer buffer, PmBuffer src, PmBuffer dst, uint32_t count,
                                    const PmBufferCopy* regions) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!src || !dst || src->device != buffer->device || dst->device != buffer->device || count == 0u || !regions ||
        !src->ptr || !dst->ptr)
        return PM_ERROR_INVALID_ARGUMENT;
    std::vector<PmBufferCopy> copied(regions, regions + count);
    for (const PmBufferCopy& r : copied)
        if (!range_fits(r.srcOffset, r.size, src->size) || !range_fits(r.dstOffset, r.size, dst->size))
            return PM_ERROR_INVALID_ARGUMENT;
    PmDevice_T* device = buffer->device;
    return record(buffer, [device, src, dst, copied]() -> PmResult {
        if (src->queue_family != 0u || dst->queue_family != 0u) return PM_ERROR_INVALID_STATE;
        for (const PmBufferCopy& r : copied) {
            const int rc = pmb_copy_async(device->ordinal, dst->ptr + r.dstOffset, src->ptr + r.srcOffset, r.size,
                                          device->stream);
            if (rc != PMB_SUCCESS) return from_core(rc);
        }
        return PM_SUCCESS;
    });
}

// The worker runs every command of a submission in order on one CUDA
// stream, so memory barriers only carry queue-family ownership transfers.
PmResult PMAPI_CALL pmCmdPipelineBarrier(PmCommandBuffer buffer, uint32_t memory_count,
                                         const PmMemoryBarrier* memory_barriers, uint32_t buffer_count,
                                         const PmBufferMemoryBarrier* buffer_barriers) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if ((memory_count && !memory_barriers) || (buffer_count && !buffer_barriers)) return PM_ERROR_INVALID_ARGUMENT;
    std::vector<PmBufferMemoryBarrier> copied;
    if (buffer_count) copied.assign(buffer_barriers, buffer_barriers + buffer_count);
    for (const auto& b : copied) {
        const bool ignored =
            b.srcQueueFamilyIndex == PM_QUEUE_FAMILY_IGNORED && b.dstQueueFamilyIndex == PM_QUEUE_FAMILY_IGNORED;
        const auto family_ok = [](uint32_t f) { return f == 0u || f == PM_QUEUE_FAMILY_EXTERNAL; };
        if (!b.range.buffer || b.range.buffer->device != buffer->device ||
            !range_fits(b.range.offset, resolved_size(b.range.offset, b.range.size, b.range.buffer->size),
                        b.range.buffer->size) ||
            (!ignored && (!family_ok(b.srcQueueFamilyIndex) || !family_ok(b.dstQueueFamilyIndex))))
            return PM_ERROR_INVALID_ARGUMENT;
    }
    if (copied.empty()) return PM_SUCCESS;
    return record(buffer, [copied]() -> PmResult {
        for (const auto& b : copied) {
            if (b.srcQueueFamilyIndex == PM_QUEUE_FAMILY_IGNORED) continue;
            if (b.range.buffer->queue_family != b.srcQueueFamilyIndex) return PM_ERROR_INVALID_STATE;
            b.range.buffer->queue_family = b.dstQueueFamilyIndex;
        }
        return PM_SUCCESS;
    });
}

// ====================================================================
// semaphores, submission, fences (reference src/api/synchronization.cpp)
// ====================================================================
PmResult PMAPI_CALL pmCreateSemaphore(PmDevice device, const PmSemaphoreCreateInfo* info, PmSemaphore* semaphore) {
    if (!semaphore) return PM_ERROR_INVALID_ARGUMENT;
    *semaphore = nullptr;
    if (!device || !info || !valid_structure(info->sType, PM_STRUCTURE_TYPE_SEMAPHORE_CREATE_INFO, info->pNext))
        return PM_ERROR_INVALID_ARGUMENT;
    auto* created = new (std::nothrow) PmSemaphore_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    created->device = device;
    created->value = info->initialValue;
    *semaphore = created;
    return PM_SUCCESS;
}

void PMAPI_CALL pmDestroySemaphore(PmDevice device, PmSemaphore semaphore) {
    if (!device || !semaphore || semaphore->device != device) return;
    (void)pmDeviceWaitIdle(device);
    delete semaphore;
}

PmResult PMAPI_CALL pmGetSemaphoreCounterValue(PmDevice device, PmSemaphore semaphore, uint64_t* value) {
    if (!device || !semaphore || !value || semaphore->device != device) return PM_ERROR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(semaphore->mutex);
    refresh_timeline_locked(semaphore);
    if (!semaphore->signals.empty()) {
        const PmResult r = semaphore->signals.begin()->second->status();
        if (r < PM_SUCCESS) return r;
    }
    *value = semaphore->value;
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmWaitSemaphore(PmDevice device, PmSemaphore semaphore, uint64_t value, uint64_t timeout) {
    if (!device || !semaphore || semaphore->device != device) return PM_ERROR_INVALID_ARGUMENT;
    const auto deadline = deadline_after(timeout);
    for (;;) {
        const PmResult r = timeline_status(semaphore, value);
        if (r != PM_NOT_READY) return r;
        CompletionPtr next;
        {
            std::lock_guard<std::mutex> lock(semaphore->mutex);
            auto found = semaphore->signals.lower_bound(value);
            if (found != semaphore->signals.end()) next = found->second;
        }
        if (!next) return PM_TIMEOUT;  // nothing submitted will ever signal it
        if (Clock::now() >= deadline) return PM_TIMEOUT;
        next->wait_until(deadline);
    }
}

PmResult PMAPI_CALL pmQueueSubmit(PmQueue queue, const PmSubmitInfo* info, PmFence fence) {
    if (!queue || !info || !valid_structure(info->sType, PM_STRUCTURE_TYPE_SUBMIT_INFO, info->pNext) ||
        (info->waitCount && !info->pWaits) || (info->commandBufferCount && !info->pCommandBuffers) ||
        (info->signalCount && !info->pSignals) || (fence && fence->device != queue->device))
        return PM_ERROR_INVALID_ARGUMENT;
    PmDevice_T* device = queue->device;
    std::lock_guard<std::mutex> submit_lock(device->submit_mutex);
    if (fence && (fence->submitted || fence->initially_signaled)) return PM_ERROR_INVALID_STATE;
    for (uint32_t i = 0; i < info->commandBufferCount; ++i) {
        PmCommandBuffer_T* b = info->pCommandBuffers[i];
        refresh_command_state(b);
        if (!b || b->device != device || b->state != CommandState::executable) return PM_ERROR_INVALID_STATE;
        for (uint32_t k = 0; k < i; ++k)
            if (info->pCommandBuffers[k] == b) return PM_ERROR_INVALID_ARGUMENT;
    }
    for (uint32_t i = 0; i < info->waitCount; ++i) {
        const PmSemaphoreSubmitInfo& w = info->pWaits[i];
        if (!w.semaphore || w.semaphore->device != device) return PM_ERROR_INVALID_ARGUMENT;
        std::lock_guard<std::mutex> lock(w.semaphore->mutex);
        const bool submitted =
            w.semaphore->value >= w.value || w.semaphore->signals.lower_bound(w.value) != w.semaphore->signals.end();
        // One ordered queue: a wait nothing earlier will signal can never be
        // satisfied.
        if (!submitted) return PM_ERROR_INVALID_ARGUMENT;
    }
    for (uint32_t i = 0; i < info->signalCount; ++i) {
        const PmSemaphoreSubmitInfo& s = info->pSignals[i];
        if (!s.semaphore || s.semaphore->device != device || s.stages != PM_STAGE_ALL_COMMANDS_BIT)
            return PM_ERROR_INVALID_ARGUMENT;
        std::lock_guard<std::mutex> lock(s.semaphore->mutex);
        refresh_timeline_locked(s.semaphore);
        uint64_t greatest = s.semaphore->value;
        if (!s.semaphore->signals.empty()) greatest = std::max(greatest, s.semaphore->signals.rbegin()->first);
        for (uint32_t k = 0; k < i; ++k)
            if (info->pSignals[k].semaphore == s.semaphore) greatest = std::max(greatest, info->pSignals[k].value);
        if (s.value <= greatest) return PM_ERROR_INVALID_ARGUMENT;
    }
#if defined(PMB_TEST_FAILURE_DRIVER)
    // Test build only (reference src/device/submission.cpp:45-48): the
    // submission fails before acceptance, so nothing becomes pending.
    if (std::getenv("PM_TEST_FAIL_SUBMISSION") != nullptr) return PM_ERROR_OUT_OF_HOST_MEMORY;
#endif
    auto completion = std::make_shared<Completion>();
    std::vector<std::function<PmResult()>> commands;
    std::vector<PmSimulation_T*> simulations;
    std::vector<std::pair<PmSemaphore_T*, uint64_t>> waits;
    for (uint32_t i = 0; i < info->waitCount; ++i) waits.push_back({info->pWaits[i].semaphore, info->pWaits[i].value});
    for (uint32_t i = 0; i < info->commandBufferCount; ++i) {
        PmCommandBuffer_T* b = info->pCommandBuffers[i];
        commands.insert(commands.end(), b->commands.begin(), b->commands.end());
        for (auto* s : b->simulations)
            if (std::find(simulations.begin(), simulations.end(), s) == simulations.end()) simulations.push_back(s);
        for (const QueryWrite& q : b->query_writes) {
            std::lock_guard<std::mutex> lock(q.pool->mutex);
            for (uint32_t slot = q.first; slot < q.first + q.count; ++slot) {
                q.pool->slots[slot].completion = completion;
                q.pool->slots[slot].available = false;
            }
        }
        b->completion = completion;
        b->state = CommandState::pending;
    }
    for (auto* s : simulations) s->pending.fetch_add(1u);
    for (uint32_t i = 0; i < info->signalCount; ++i) {
        std::lock_guard<std::mutex> lock(info->pSignals[i].semaphore->mutex);
        info->pSignals[i].semaphore->signals.emplace(info->pSignals[i].value, completion);
    }
    if (fence) {
        fence->completion = completion;
        fence->submitted = true;
    }
    device->worker.enqueue(
        [device, commands = std::move(commands), simulations, waits]() -> PmResult {
            PmResult result = PM_SUCCESS;
            for (const auto& w : waits)
                if (result == PM_SUCCESS) result = timeline_status(w.first, w.second);
            for (const auto& command : commands) {
                if (result != PM_SUCCESS) break;
                result = command();
            }
            const int drained = pmb_stream_synchronize(device->ordinal, device->stream);
            if (result == PM_SUCCESS && drained != PMB_SUCCESS) result = PM_ERROR_DEVICE_LOST;
            for (auto* s : simulations) {
                if (result != PM_SUCCESS) s->execution_result.store(result);
                s->pending.fetch_sub(1u);
            }
            return result;
        },
        completion);
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmQueueWaitIdle(PmQueue queue) {
    if (!queue) return PM_ERROR_INVALID_ARGUMENT;
    queue->device->worker.wait_idle();
    return from_core(pmb_stream_synchronize(queue->device->ordinal, queue->device->stream));
}

PmResult PMAPI_CALL pmDeviceWaitIdle(PmDevice device) {
    return device ? pmQueueWaitIdle(&device->queue) : PM_ERROR_INVALID_ARGUMENT;
}

PmResult PMAPI_CALL pmCreateFence(PmDevice device, PmFlags flags, PmFence* fence) {
    if (!fence) return PM_ERROR_INVALID_ARGUMENT;
    *fence = nullptr;
    if (!device || (flags & ~PmFlags(PM_FENCE_SIGNALED_BIT))) return PM_ERROR_INVALID_ARGUMENT;
    auto* created = new (std::nothrow) PmFence_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    created->device = device;
    created->initially_signaled = (flags & PM_FENCE_SIGNALED_BIT) != 0u;
    *fence = created;
    return PM_SUCCESS;
}

void PMAPI_CALL pmDestroyFence(PmDevice device, PmFence fence) {
    if (!device || !fence || fence->device != device) return;
    if (fence->completion) fence->completion->wait_until(Clock::time_point::max());
    delete fence;
}

PmResult PMAPI_CALL pmGetFenceStatus(PmDevice device, PmFence fence) {
    if (!device || !fence || fence->device != device) return PM_ERROR_INVALID_ARGUMENT;
    if (fence->initially_signaled) return PM_SUCCESS;
    if (!fence->submitted) return PM_NOT_READY;
    return fence->completion->status();
}

PmResult PMAPI_CALL pmResetFences(PmDevice device, uint32_t count, const PmFence* fences) {
    if (!device || count == 0u || !fences) return PM_ERROR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < count; ++i)
        if (!fences[i] || fences[i]->device != device ||
            (fences[i]->submitted && pmGetFenceStatus(device, fences[i]) == PM_NOT_READY))
            return PM_ERROR_INVALID_STATE;
    for (uint32_t i = 0; i < count; ++i) {
        fences[i]->completion.reset();
        fences[i]->submitted = false;
        fences[i]->initially_signaled = false;
    }
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmWaitForFences(PmDevice device, uint32_t count, const PmFence* fences, PmBool32 wait_all,
                                    uint64_t timeout) {
    if (!device || count == 0u || !fences) return PM_ERROR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < count; ++i)
        if (!fences[i] || fences[i]->device != device) return PM_ERROR_INVALID_ARGUMENT;
    const auto deadline = deadline_after(timeout);
    for (;;) {
        uint32_t ready = 0;
        CompletionPtr pending;
        for (uint32_t i = 0; i < count; ++i) {
            const PmResult s = pmGetFenceStatus(device, fences[i]);
            if (s == PM_SUCCESS)
                ++ready;
            else if (s != PM_NOT_READY)
                return s;
            else if (!pending && fences[i]->submitted)
                pending = fences[i]->completion;
        }
        if ((wait_all == PM_TRUE && ready == count) || (wait_all != PM_TRUE && ready != 0u)) return PM_SUCCESS;
        if (Clock::now() >= deadline) return PM_TIMEOUT;
        if (!pending) {
            // Only unsubmitted fences remain: nothing can signal them
            // before the deadline except a later submission; poll.
            std::this_thread::sleep_for(std::chrono::microseconds(200));
            continue;
        }
        pending->wait_until(std::min(deadline, Clock::now() + std::chrono::milliseconds(50)));
    }
}

// ====================================================================
// queries (reference src/api/queries.cpp)
// ====================================================================
PmResult PMAPI_CALL pmCreateQueryPool(PmDevice device, const PmQueryPoolCreateInfo* info, PmQueryPool* pool) {
    if (!pool) return PM_ERROR_INVALID_ARGUMENT;
    *pool = nullptr;
    if (!device || !info || !valid_structure(info->sType, PM_STRUCTURE_TYPE_QUERY_POOL_CREATE_INFO, info->pNext) ||
        info->queryCount == 0u || info->queryCount > 65536u ||
        (info->queryType != PM_QUERY_TIMESTAMP && info->queryType != PM_QUERY_STEP_STATISTICS &&
         info->queryType != PM_QUERY_REALTIME_STEP_STATISTICS))
        return PM_ERROR_INVALID_ARGUMENT;
    auto* created = new (std::nothrow) PmQueryPool_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    created->device = device;
    created->type = info->queryType;
    created->slots.resize(info->queryCount);
    if (info->queryType == PM_QUERY_TIMESTAMP)
        for (auto& slot : created->slots)
            if (pmb_event_create(device->ordinal, &slot.event) != PMB_SUCCESS) {
                for (auto& s : created->slots)
                    if (s.event) pmb_event_destroy(device->ordinal, s.event);
                delete created;
                return PM_ERROR_DEVICE_LOST;
            }
    *pool = created;
    return PM_SUCCESS;
}

void PMAPI_CALL pmDestroyQueryPool(PmDevice device, PmQueryPool pool) {
    if (!device || !pool || pool->device != device) return;
    (void)pmDeviceWaitIdle(device);
    for (auto& s : pool->slots)
        if (s.event) pmb_event_destroy(device->ordinal, s.event);
    delete pool;
}

PmResult PMAPI_CALL pmCmdResetQueryPool(PmCommandBuffer buffer, PmQueryPool pool, uint32_t first, uint32_t count) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!pool || pool->device != buffer->device || count == 0u || first > pool->slots.size() ||
        count > pool->slots.size() - first)
        return PM_ERROR_INVALID_ARGUMENT;
    return record_query(buffer, pool, first, count, [pool, first, count]() -> PmResult {
        std::lock_guard<std::mutex> lock(pool->mutex);
        for (uint32_t i = first; i < first + count; ++i) {
            pool->slots[i].available = false;
            pool->slots[i].statistics = {};
            pool->slots[i].realtime = {};
        }
        return PM_SUCCESS;
    });
}

PmResult PMAPI_CALL pmCmdWriteTimestamp(PmCommandBuffer buffer, PmStageFlags, PmQueryPool pool, uint32_t query) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!pool || pool->device != buffer->device || pool->type != PM_QUERY_TIMESTAMP || query >= pool->slots.size())
        return PM_ERROR_INVALID_ARGUMENT;
    PmDevice_T* device = buffer->device;
    return record_query(buffer, pool, query, 1u, [device, pool, query]() -> PmResult {
        std::lock_guard<std::mutex> lock(pool->mutex);
        const int r = pmb_event_record(device->ordinal, pool->slots[query].event, device->stream);
        if (r != PMB_SUCCESS) return from_core(r);
        pool->slots[query].available = true;
        return PM_SUCCESS;
    });
}

PmResult PMAPI_CALL pmCmdBeginStatisticsQuery(PmCommandBuffer buffer, PmQueryPool pool, uint32_t query) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!pool || pool->device != buffer->device ||
        (pool->type != PM_QUERY_STEP_STATISTICS && pool->type != PM_QUERY_REALTIME_STEP_STATISTICS) ||
        query >= pool->slots.size() || buffer->statistics_open)
        return PM_ERROR_INVALID_ARGUMENT;
    buffer->statistics_open = true;
    buffer->statistics_pool = pool;
    buffer->statistics_query = query;
    buffer->statistics_simulation = nullptr;
    buffer->statistics_step_count = 0;
    return record_query(buffer, pool, query, 1u, [pool, query]() -> PmResult {
        std::lock_guard<std::mutex> lock(pool->mutex);
        pool->slots[query].statistics = {};
        pool->slots[query].realtime = {};
        pool->slots[query].available = false;
        return PM_SUCCESS;
    });
}

PmResult PMAPI_CALL pmCmdEndStatisticsQuery(PmCommandBuffer buffer, PmQueryPool pool, uint32_t query) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    // A realtime statistics query brackets exactly one step
    // (reference src/api/queries.cpp:159-172).
    if (!pool || pool->device != buffer->device ||
        (pool->type != PM_QUERY_STEP_STATISTICS && pool->type != PM_QUERY_REALTIME_STEP_STATISTICS) ||
        query >= pool->slots.size() || !buffer->statistics_open || buffer->statistics_pool != pool ||
        buffer->statistics_query != query || !buffer->statistics_simulation ||
        (pool->type == PM_QUERY_REALTIME_STEP_STATISTICS && buffer->statistics_step_count != 1u))
        return PM_ERROR_INVALID_ARGUMENT;
    PmSimulation_T* simulation = buffer->statistics_simulation;
    buffer->statistics_open = false;
    buffer->statistics_pool = nullptr;
    buffer->statistics_simulation = nullptr;
    buffer->statistics_step_count = 0;
    return record_query(buffer, pool, query, 1u, [pool, query, simulation]() -> PmResult {
        std::lock_guard<std::mutex> lock(pool->mutex);
        auto& slot = pool->slots[query];
        fill_statistics(simulation, slot.statistics);
        if (pool->type == PM_QUERY_REALTIME_STEP_STATISTICS) {
            const PmResult r = fill_realtime_statistics(simulation, slot.realtime);
            if (r != PM_SUCCESS) return r;
            slot.realtime.step = slot.statistics;
            slot.realtime.step.stepCount = 1;  // query-local, as the reference reports it
        }
        slot.available = true;
        return PM_SUCCESS;
    });
}

PmResult PMAPI_CALL pmGetQueryPoolResults(PmDevice device, PmQueryPool pool, uint32_t first, uint32_t count,
                                          size_t data_size, void* data, PmDeviceSize stride, PmFlags flags) {
    if (!device || !pool || pool->device != device || count == 0u || !data || first > pool->slots.size() ||
        count > pool->slots.size() - first)
        return PM_ERROR_INVALID_ARGUMENT;
    const size_t value_size = pool->type == PM_QUERY_TIMESTAMP                   ? sizeof(uint64_t)
                              : pool->type == PM_QUERY_REALTIME_STEP_STATISTICS ? sizeof(PmRealtimeStepStatistics)
                                                                                : sizeof(PmStepStatistics);
    const size_t record_size = value_size + ((flags & PM_QUERY_RESULT_WITH_AVAILABILITY_BIT) ? sizeof(uint64_t) : 0);
    if (stride < record_size || data_size < record_size + size_t(count - 1u) * size_t(stride))
        return PM_ERROR_INVALID_ARGUMENT;
    bool incomplete = false;
    for (uint32_t k = 0; k < count; ++k) {
        CompletionPtr completion;
        {
            std::lock_guard<std::mutex> lock(pool->mutex);
            completion = pool->slots[first + k].completion;
        }
        if (completion && (flags & PM_QUERY_RESULT_WAIT_BIT)) completion->wait_until(Clock::time_point::max());
        const PmResult status = completion ? completion->status() : PM_SUCCESS;
        if (status < PM_SUCCESS) return status;
        std::lock_guard<std::mutex> lock(pool->mutex);
        auto& slot = pool->slots[first + k];
        bool available = status == PM_SUCCESS && slot.available;
        char* dst = static_cast<char*>(data) + size_t(k) * size_t(stride);
        if (available && pool->type == PM_QUERY_TIMESTAMP) {
            int ready = 0;
            if (pmb_event_query(device->ordinal, slot.event, &ready) != PMB_SUCCESS) return PM_ERROR_DEVICE_LOST;
            if (!ready && (flags & PM_QUERY_RESULT_WAIT_BIT)) ready = 1;  // elapsed_ms waits on the event
            available = ready != 0;
        }
        if (available) {
            if (pool->type == PM_QUERY_TIMESTAMP) {
                float ms = 0.0f;
                if (pmb_event_elapsed_ms(device->ordinal, device->epoch, slot.event, &ms) != PMB_SUCCESS)
                    return PM_ERROR_DEVICE_LOST;
                const uint64_t ns = uint64_t(double(ms) * 1.0e6);
                std::memcpy(dst, &ns, sizeof(ns));
            } else if (pool->type == PM_QUERY_REALTIME_STEP_STATISTICS) {
                std::memcpy(dst, &slot.realtime, sizeof(PmRealtimeStepStatistics));
            } else {
                std::memcpy(dst, &slot.statistics, sizeof(PmStepStatistics));
            }
        } else {
            std::memset(dst, 0, value_size);
            incomplete = true;
        }
        if (flags & PM_QUERY_RESULT_WITH_AVAILABILITY_BIT) {
            const uint64_t a = available ? 1u : 0u;
            std::memcpy(dst + value_size, &a, sizeof(a));
        }
    }
    return incomplete ? PM_NOT_READY : PM_SUCCESS;
}

PmResult PMAPI_CALL pmGetDeviceMemoryBudget(PmDevice device, PmMemoryBudget* budget) {
    if (!device || !budget) return PM_ERROR_INVALID_ARGUMENT;
    *budget = {};
    uint64_t free_bytes = 0, total = 0;
    const int r = pmb_device_memory_info(device->ordinal, &free_bytes, &total);
    if (r != PMB_SUCCESS) return from_core(r);
    budget->heapCount = 1;
    budget->budget[0] = free_bytes + device->application_bytes.load();
    budget->usage[0] = total - free_bytes;
    budget->confidence[0] = PM_MEMORY_BUDGET_CONFIDENCE_DRIVER_REPORTED;
    budget->applicationAllocationBytes = device->application_bytes.load();
    return PM_SUCCESS;
}

PFN_pmVoidFunction lookup(const char* name) {
    if (!name) return nullptr;
#define PM_ENTRY(fn) \
    if (std::strcmp(name, #fn) == 0) return reinterpret_cast<PFN_pmVoidFunction>(&fn);
    PM_ENTRY(pmEnumerateInstanceVersion)
    PM_ENTRY(pmCreateInstance)
    PM_ENTRY(pmDestroyInstance)
    PM_ENTRY(pmEnumeratePhysicalDevices)
    PM_ENTRY(pmGetPhysicalDeviceProperties)
    PM_ENTRY(pmGetPhysicalDeviceQueueFamilies)
    PM_ENTRY(pmGetPhysicalDeviceFeatures)
    PM_ENTRY(pmGetPhysicalDeviceMemoryProperties)
    PM_ENTRY(pmCreateDevice)
    PM_ENTRY(pmDestroyDevice)
    PM_ENTRY(pmGetDeviceQueue)
    PM_ENTRY(pmAllocateMemory)
    PM_ENTRY(pmFreeMemory)
    PM_ENTRY(pmMapMemory)
    PM_ENTRY(pmUnmapMemory)
    PM_ENTRY(pmFlushMappedMemoryRanges)
    PM_ENTRY(pmInvalidateMappedMemoryRanges)
    PM_ENTRY(pmCreateBuffer)
    PM_ENTRY(pmDestroyBuffer)
    PM_ENTRY(pmGetBufferMemoryRequirements)
    PM_ENTRY(pmBindBufferMemory)
    PM_ENTRY(pmCreateGeometry)
    PM_ENTRY(pmDestroyGeometry)
    PM_ENTRY(pmGetGeometryMemoryRequirements)
    PM_ENTRY(pmBindGeometryMemory)
    PM_ENTRY(pmCmdBuildGeometry)
    PM_ENTRY(pmCreatePhysicsPipeline)
    PM_ENTRY(pmDestroyPhysicsPipeline)
    PM_ENTRY(pmCreateCommandPool)
    PM_ENTRY(pmDestroyCommandPool)
    PM_ENTRY(pmResetCommandPool)
    PM_ENTRY(pmAllocateCommandBuffers)
    PM_ENTRY(pmFreeCommandBuffers)
    PM_ENTRY(pmBeginCommandBuffer)
    PM_ENTRY(pmEndCommandBuffer)
    PM_ENTRY(pmResetCommandBuffer)
    PM_ENTRY(pmCmdBindPhysicsPipeline)
    PM_ENTRY(pmCmdCopyBuffer)
    PM_ENTRY(pmCmdPipelineBarrier)
    PM_ENTRY(pmCreateSemaphore)
    PM_ENTRY(pmDestroySemaphore)
    PM_ENTRY(pmGetSemaphoreCounterValue)
    PM_ENTRY(pmWaitSemaphore)
    PM_ENTRY(pmQueueSubmit)
    PM_ENTRY(pmQueueWaitIdle)
    PM_ENTRY(pmDeviceWaitIdle)
    PM_ENTRY(pmCreateFence)
    PM_ENTRY(pmDestroyFence)
    PM_ENTRY(pmGetFenceStatus)
    PM_ENTRY(pmResetFences)
    PM_ENTRY(pmWaitForFences)
    PM_ENTRY(pmCreateQueryPool)
    PM_ENTRY(pmDestroyQueryPool)
    PM_ENTRY(pmCmdResetQueryPool)
    PM_ENTRY(pmCmdWriteTimestamp)
    PM_ENTRY(pmCmdBeginStatisticsQuery)
    PM_ENTRY(pmCmdEndStatisticsQuery)
    PM_ENTRY(pmGetQueryPoolResults)
    PM_ENTRY(pmGetDeviceMemoryBudget)
#undef PM_ENTRY
    return lookup_rigid(name);
}

}  // namespace

// The proc-address lookups behave as the reference driver's
// (src/driver/slang/entry.cpp:30-56): without an instance only the
// bootstrapping commands resolve; device and physical-device lookups need a
// handle.
PM_EXPORT PmResult PMAPI_CALL pm_driverNegotiateLoaderInterfaceVersion(uint32_t* version) {
    if (!version || *version == 0u) return PM_ERROR_INVALID_ARGUMENT;
    *version = std::min(*version, PM_DRIVER_INTERFACE_VERSION);
    return PM_SUCCESS;
}

PM_EXPORT PFN_pmVoidFunction PMAPI_CALL pm_driverGetInstanceProcAddr(PmInstance instance, const char* name) {
    if (!instance && name && std::strcmp(name, "pmGetInstanceProcAddr") != 0 &&
        std::strcmp(name, "pmEnumerateInstanceVersion") != 0 && std::strcmp(name, "pmCreateInstance") != 0)
        return nullptr;
    if (name && std::strcmp(name, "pmGetInstanceProcAddr") == 0)
        return reinterpret_cast<PFN_pmVoidFunction>(&pm_driverGetInstanceProcAddr);
    if (name && std::strcmp(name, "pmGetDeviceProcAddr") == 0)
        return reinterpret_cast<PFN_pmVoidFunction>(&pm_driverGetDeviceProcAddr);
    return lookup(name);
}

PM_EXPORT PFN_pmVoidFunction PMAPI_CALL pm_driverGetDeviceProcAddr(PmDevice device, const char* name) {
    if (!device) return nullptr;
    if (name && std::strcmp(name, "pmGetDeviceProcAddr") == 0)
        return reinterpret_cast<PFN_pmVoidFunction>(&pm_driverGetDeviceProcAddr);
    return lookup(name);
}

PM_EXPORT PFN_pmVoidFunction PMAPI_CALL pm_driverGetPhysicalDeviceProcAddr(PmInstance instance, const char* name) {
    return instance ? lookup(name) : nullptr;
}

// SPDX-License-Identifier: MIT
// Objects behind the pm* handles of libpm_b200_driver.so.
//
// Execution model (the reference's, src/device/submission.hpp:34-73 and
// src/api/synchronization.cpp): commands are validated and recorded on the
// caller's thread as closures; pmQueueSubmit hands a submission to the
// device's single ordered worker thread, which runs the closures, drains the
// device's CUDA stream and then completes the submission's fence and
// semaphore signals. A simulation's rigid world (pmb_world) lives in the
// memory the application bound to it and is only touched by the worker.
#pragma once

#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/pm_b200.h"
#include "../../include/pmb200_core.h"

namespace pmd {

using Clock = std::chrono::steady_clock;

// Completion of one submission: PM_NOT_READY until the worker finishes it.
struct Completion {
    std::mutex mutex;
    std::condition_variable cv;
    bool done{};
    PmResult result{PM_SUCCESS};
    PmResult status() {
        std::lock_guard<std::mutex> lock(mutex);
        return done ? result : PM_NOT_READY;
    }
    void finish(PmResult r) {
        {
            std::lock_guard<std::mutex> lock(mutex);
            done = true;
            result = r;
        }
        cv.notify_all();
    }
    // Waits until done or the deadline; returns status().
    PmResult wait_until(Clock::time_point deadline) {
        std::unique_lock<std::mutex> lock(mutex);
        if (deadline == Clock::time_point::max())
            cv.wait(lock, [&] { return done; });
        else
            cv.wait_until(lock, deadline, [&] { return done; });
        return done ? result : PM_NOT_READY;
    }
};
using CompletionPtr = std::shared_ptr<Completion>;

// One ordered worker thread per device queue.
class Worker {
public:
    void start();
    void stop();
    void enqueue(std::function<PmResult()> job, CompletionPtr completion);
    void wait_idle();

private:
    void run();
    std::mutex mutex_;
    std::condition_variable cv_, idle_cv_;
    std::deque<std::pair<std::function<PmResult()>, CompletionPtr>> jobs_;
    bool busy_{}, stopping_{};
    std::thread thread_;
};

}  // namespace pmd

struct PmPhysicalDevice_T {
    PmInstance_T* instance{};
    int32_t ordinal{};
    pmb_device_info_t info{};
};

struct PmInstance_T {
    std::vector<std::unique_ptr<PmPhysicalDevice_T>> physical;
    PmAllocationCallbacks allocator{};
    bool has_allocator{};
};

struct PmQueue_T {
    PmDevice_T* device{};
};

struct PmDevice_T {
    PmPhysicalDevice_T* physical{};
    int32_t ordinal{};
    PmPhysicalDeviceFeatures enabled{};
    PmQueue_T queue{};
    void* stream{};  // cudaStream_t, used only by the worker
    void* epoch{};   // cudaEvent_t recorded at creation: timestamp origin
    pmd::Worker worker;
    std::mutex submit_mutex;
    std::atomic<uint64_t> application_bytes{0};
};

struct PmDeviceMemory_T {
    PmDevice_T* device{};
    void* ptr{};
    PmDeviceSize size{};
    uint32_t type{};  // 0 device-local, 1 device-local + host-visible (managed)
    bool mapped{};
};

struct PmBuffer_T {
    PmDevice_T* device{};
    PmDeviceSize size{};
    PmFlags usage{};
    uint32_t queue_family{};
    PmDeviceMemory_T* memory{};
    PmDeviceSize offset{};
    char* ptr{};  // device (or managed) address of byte 0, once bound
};

struct PmGeometry_T {
    PmDevice_T* device{};
    PmGeometryCreateInfo info{};
    PmMemoryRequirements requirements{};
    PmDeviceMemory_T* memory{};
    PmDeviceSize offset{};
    // Filled by pmCmdBuildGeometry on the worker.
    bool built{};
    std::vector<float> vertices;
    std::vector<uint32_t> indices;
    float lo[3]{}, hi[3]{};
};

struct PmPhysicsPipeline_T {
    PmDevice_T* device{};
    PmRigidSolverState rigid{};
};

struct PmSimulation_T {
    PmDevice_T* device{};
    PmSimulationCreateInfo info{};
    PmSimulationMemoryRequirements requirements{};
    pmb_world_capacity capacity{};
    PmSimulationMemoryBinding binding{};
    bool bound{};
    // Worker-side runtime state.
    struct Body {
        bool active{};
        PmRigidBodyInfo info{};
    };
    struct Constraint {
        bool active{};
        PmRigidConstraintInfo info{};
    };
    std::vector<Body> bodies;             // by slot
    std::vector<Constraint> constraints;  // by slot
    std::vector<uint8_t> fresh;           // slot written since the world was built
    pmb_world* world{};
    bool dirty{true};
    std::vector<uint32_t> dense_of_slot;  // PM_INVALID_INDEX when inactive
    std::vector<uint32_t> joint_of_slot;
    std::map<uint32_t, std::array<float, 12>> inputs;  // by dense index
    std::map<uint32_t, PmRigidState> targets;          // by dense index
    pmb_step_stats last{};
    uint64_t submitted_steps{};
    uint32_t last_substeps{};
    std::atomic<uint32_t> pending{0};
    std::atomic<int32_t> execution_result{PM_SUCCESS};
};

struct PmCommandBuffer_T;

struct PmCommandPool_T {
    PmDevice_T* device{};
    PmFlags flags{};
    std::vector<PmCommandBuffer_T*> buffers;
};

enum class CommandState { initial, recording, executable, pending };

struct QueryWrite {
    PmQueryPool_T* pool{};
    uint32_t first{}, count{};
};

struct PmCommandBuffer_T {
    PmDevice_T* device{};
    PmCommandPool_T* pool{};
    CommandState state{CommandState::initial};
    PmFlags usage{};
    PmResult latched{PM_SUCCESS};
    std::vector<std::function<PmResult()>> commands;
    std::vector<QueryWrite> query_writes;
    std::vector<PmSimulation_T*> simulations;
    PmPhysicsPipeline_T* bound_pipeline{};
    bool statistics_open{};
    PmQueryPool_T* statistics_pool{};
    uint32_t statistics_query{};
    PmSimulation_T* statistics_simulation{};
    uint32_t statistics_step_count{};  // steps recorded inside an open statistics query
    pmd::CompletionPtr completion;
};

struct PmSemaphore_T {
    PmDevice_T* device{};
    std::mutex mutex;
    uint64_t value{};
    std::map<uint64_t, pmd::CompletionPtr> signals;  // pending signal value -> submission
};

struct PmFence_T {
    PmDevice_T* device{};
    bool initially_signaled{}, submitted{};
    pmd::CompletionPtr completion;
};

struct PmQueryPool_T {
    PmDevice_T* device{};
    PmQueryType type{};
    std::mutex mutex;
    struct Slot {
        bool available{};
        void* event{};  // timestamps
        PmStepStatistics statistics{};
        PmRealtimeStepStatistics realtime{};
        pmd::CompletionPtr completion;
    };
    std::vector<Slot> slots;
};

namespace pmd {

// Helpers shared by the command translation units.
inline bool range_fits(PmDeviceSize offset, PmDeviceSize size, PmDeviceSize total) {
    return offset <= total && size <= total - offset;
}
inline PmDeviceSize resolved_size(PmDeviceSize offset, PmDeviceSize size, PmDeviceSize total) {
    return size == PM_WHOLE_SIZE ? (offset <= total ? total - offset : 0) : size;
}
inline bool valid_structure(PmStructureType got, PmStructureType want, const void* next) {
    return got == want && next == nullptr;
}
PmResult from_core(int status);
// Fails unless the buffer is in the recording state.
PmResult require_recording(PmCommandBuffer_T* buffer);
// Appends a closure the worker runs at submission time.
PmResult record(PmCommandBuffer_T* buffer, std::function<PmResult()> command);
PmResult record_simulation(PmCommandBuffer_T* buffer, PmSimulation_T* simulation, std::function<PmResult()> command);
PmResult record_query(PmCommandBuffer_T* buffer, PmQueryPool_T* pool, uint32_t first, uint32_t count,
                      std::function<PmResult()> command);
// Resolved command table of the rigid translation unit.
PFN_pmVoidFunction lookup_rigid(const char* name);
// Statistics of a simulation's last tick, for step-statistics queries.
void fill_statistics(PmSimulation_T* simulation, PmStepStatistics& out);
PmResult fill_realtime_statistics(PmSimulation_T* simulation, PmRealtimeStepStatistics& out);

}  // namespace pmd

/* SPDX-License-Identifier: MIT
 * pm_b200: the rigid-body subset of the Parallel Mater 0.3 command API as
 * implemented by libpm_b200_driver.so, plus the four loader-to-driver entry
 * points that library exports.
 *
 * Binary compatibility is the point of this header: every type below has the
 * size, field order and field types of the declaration with the same name in
 * the reference's include/parallel_mater/parallel_mater.h (and the driver ABI
 * of include/parallel_mater/pm_driver.h:22-41), so an application or loader
 * built against the reference talks to this driver unchanged. Line numbers
 * in the comments name the reference declaration each block matches.
 *
 * Only the rigid domain is implemented. Every command of another domain
 * (fluids, cloth, rope, soft bodies, smoke, paint, couplings, native interop)
 * resolves to NULL from the proc-address entry points, which the reference
 * loader reports to the application as PM_ERROR_FEATURE_NOT_PRESENT
 * (reference src/loader/entry.cpp:521-524); the matching feature bits of
 * PmPhysicalDeviceFeatures read PM_FALSE. Types those commands need are
 * declared opaque here.
 */
#ifndef PM_B200_H
#define PM_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef PMAPI_CALL
#define PMAPI_CALL
#endif

/* ---- versions and scalar types (parallel_mater.h:31-51) ---- */
#define PM_MAKE_API_VERSION(major, minor, patch) \
    ((((uint32_t)(major)) << 22) | (((uint32_t)(minor)) << 12) | ((uint32_t)(patch)))
#define PM_API_VERSION_0_3 PM_MAKE_API_VERSION(0, 3, 0)
#define PM_WHOLE_SIZE UINT64_MAX
#define PM_TIMEOUT_INFINITE UINT64_MAX
#define PM_INVALID_INDEX UINT32_MAX
#define PM_QUEUE_FAMILY_IGNORED UINT32_MAX
#define PM_QUEUE_FAMILY_EXTERNAL (UINT32_MAX - 1u)
#define PM_FALSE 0u
#define PM_TRUE 1u
typedef uint32_t PmBool32;
typedef uint32_t PmFlags;
typedef uint64_t PmDeviceSize;
typedef uint64_t PmStageFlags;
typedef uint64_t PmAccessFlags;

/* ---- handles (parallel_mater.h:52-65) ---- */
typedef struct PmInstance_T* PmInstance;
typedef struct PmPhysicalDevice_T* PmPhysicalDevice;
typedef struct PmDevice_T* PmDevice;
typedef struct PmQueue_T* PmQueue;
typedef struct PmDeviceMemory_T* PmDeviceMemory;
typedef struct PmBuffer_T* PmBuffer;
typedef struct PmGeometry_T* PmGeometry;
typedef struct PmSimulation_T* PmSimulation;
typedef struct PmPhysicsPipeline_T* PmPhysicsPipeline;
typedef struct PmCommandPool_T* PmCommandPool;
typedef struct PmCommandBuffer_T* PmCommandBuffer;
typedef struct PmSemaphore_T* PmSemaphore;
typedef struct PmFence_T* PmFence;
typedef struct PmQueryPool_T* PmQueryPool;

/* ---- structure types and results (parallel_mater.h:66-110) ---- */
typedef enum PmStructureType {
    PM_STRUCTURE_TYPE_UNDEFINED = 0,
    PM_STRUCTURE_TYPE_INSTANCE_CREATE_INFO = 1,
    PM_STRUCTURE_TYPE_DEVICE_CREATE_INFO = 2,
    PM_STRUCTURE_TYPE_MEMORY_ALLOCATE_INFO = 3,
    PM_STRUCTURE_TYPE_BUFFER_CREATE_INFO = 4,
    PM_STRUCTURE_TYPE_GEOMETRY_CREATE_INFO = 5,
    PM_STRUCTURE_TYPE_SIMULATION_CREATE_INFO = 6,
    PM_STRUCTURE_TYPE_PHYSICS_PIPELINE_CREATE_INFO = 7,
    PM_STRUCTURE_TYPE_COMMAND_POOL_CREATE_INFO = 8,
    PM_STRUCTURE_TYPE_COMMAND_BUFFER_BEGIN_INFO = 9,
    PM_STRUCTURE_TYPE_SEMAPHORE_CREATE_INFO = 10,
    PM_STRUCTURE_TYPE_SUBMIT_INFO = 11,
    PM_STRUCTURE_TYPE_NATIVE_DEVICE_IMPORT_INFO = 12,
    PM_STRUCTURE_TYPE_QUERY_POOL_CREATE_INFO = 13,
    PM_STRUCTURE_TYPE_VALIDATION_DIAGNOSTICS_CREATE_INFO = 14
} PmStructureType;

typedef enum PmResult {
    PM_SUCCESS = 0,
    PM_NOT_READY = 1,
    PM_TIMEOUT = 2,
    PM_INCOMPLETE = 3,
    PM_ERROR_INVALID_ARGUMENT = -1,
    PM_ERROR_INVALID_STATE = -2,
    PM_ERROR_OUT_OF_HOST_MEMORY = -3,
    PM_ERROR_OUT_OF_DEVICE_MEMORY = -4,
    PM_ERROR_FEATURE_NOT_PRESENT = -5,
    PM_ERROR_FORMAT_NOT_SUPPORTED = -6,
    PM_ERROR_CAPACITY_EXCEEDED = -7,
    PM_ERROR_DEVICE_LOST = -8,
    PM_ERROR_INCOMPATIBLE_VERSION = -9,
    PM_ERROR_DRIVER_NOT_FOUND = -10,
    PM_ERROR_LAYER_NOT_PRESENT = -11,
    PM_ERROR_EXTENSION_NOT_PRESENT = -12
} PmResult;

typedef void(PMAPI_CALL* PFN_pmVoidFunction)(void);

/* ---- instance (parallel_mater.h:115-135, 178-182) ---- */
typedef struct PmLayerProperties {
    char layerName[256];
    uint32_t specificationVersion;
    uint32_t implementationVersion;
    char description[256];
} PmLayerProperties;
typedef struct PmExtensionProperties {
    char extensionName[256];
    uint32_t specificationVersion;
} PmExtensionProperties;
typedef struct PmInstanceCreateInfo {
    PmStructureType sType;
    const void* pNext;
    uint32_t apiVersion;
    const char* pApplicationName;
    PmBool32 enableValidation;
    uint32_t enabledLayerCount;
    const char* const* ppEnabledLayerNames;
    uint32_t enabledExtensionCount;
    const char* const* ppEnabledExtensionNames;
} PmInstanceCreateInfo;
typedef void*(PMAPI_CALL* PmAllocateFn)(void* user, size_t size, size_t alignment);
typedef void(PMAPI_CALL* PmFreeFn)(void* user, void* allocation);
typedef struct PmAllocationCallbacks {
    void* pUserData;
    PmAllocateFn pfnAllocate;
    PmFreeFn pfnFree;
} PmAllocationCallbacks;

/* ---- physical device and device (parallel_mater.h:184-239) ---- */
typedef struct PmPhysicalDeviceProperties {
    uint32_t apiVersion;
    uint32_t driverVersion;
    uint32_t vendorId;
    uint32_t deviceId;
    uint8_t deviceUuid[16];
    char deviceName[256];
} PmPhysicalDeviceProperties;
enum { PM_QUEUE_PHYSICS_BIT = 0x1, PM_QUEUE_TRANSFER_BIT = 0x2 };
typedef struct PmQueueFamilyProperties {
    PmFlags queueFlags;
    uint32_t queueCount;
    uint32_t timestampValidBits;
    float timestampPeriodNanoseconds;
} PmQueueFamilyProperties;
typedef struct PmPhysicalDeviceFeatures {
    PmBool32 rigidBodies;
    PmBool32 rigidConstraints;
    PmBool32 particleLiquids;
    PmBool32 liquidRigidCoupling;
    PmBool32 liquidLiquidCoupling;
    PmBool32 cloth;
    PmBool32 rope;
    PmBool32 softBodies;
    PmBool32 smoke;
    PmBool32 domainCouplings;
    PmBool32 particleEmitters;
    PmBool32 paint;
    PmBool32 contactEvents;
    PmBool32 debugData;
    PmBool32 timelineSemaphores;
    PmBool32 timestampQueries;
    PmBool32 statisticsQueries;
    PmBool32 memoryBudget;
    PmBool32 vulkanInterop;
} PmPhysicalDeviceFeatures;
typedef struct PmDeviceQueueCreateInfo {
    uint32_t queueFamilyIndex;
    uint32_t queueCount;
    const float* pPriorities;
} PmDeviceQueueCreateInfo;
typedef struct PmDeviceCreateInfo {
    PmStructureType sType;
    const void* pNext;
    uint32_t queueCreateInfoCount;
    const PmDeviceQueueCreateInfo* pQueueInfos;
    PmPhysicalDeviceFeatures enabledFeatures;
    uint32_t enabledExtensionCount;
    const char* const* ppEnabledExtensionNames;
} PmDeviceCreateInfo;

/* ---- memory and buffers (parallel_mater.h:241-301) ---- */
enum {
    PM_MEMORY_DEVICE_LOCAL_BIT = 0x1,
    PM_MEMORY_HOST_VISIBLE_BIT = 0x2,
    PM_MEMORY_HOST_COHERENT_BIT = 0x4,
    PM_MEMORY_HOST_CACHED_BIT = 0x8
};
typedef struct PmMemoryHeap {
    PmDeviceSize size;
    PmFlags flags;
} PmMemoryHeap;
typedef struct PmMemoryType {
    PmFlags propertyFlags;
    uint32_t heapIndex;
} PmMemoryType;
typedef struct PmMemoryProperties {
    uint32_t heapCount;
    PmMemoryHeap heaps[16];
    uint32_t typeCount;
    PmMemoryType types[32];
} PmMemoryProperties;
typedef struct PmMemoryRequirements {
    PmDeviceSize size;
    PmDeviceSize alignment;
    uint32_t memoryTypeBits;
    PmBool32 requiresDedicatedAllocation;
} PmMemoryRequirements;
typedef struct PmMemoryAllocateInfo {
    PmStructureType sType;
    const void* pNext;
    PmDeviceSize allocationSize;
    uint32_t memoryTypeIndex;
} PmMemoryAllocateInfo;
typedef struct PmMappedMemoryRange {
    PmDeviceMemory memory;
    PmDeviceSize offset;
    PmDeviceSize size;
} PmMappedMemoryRange;
enum {
    PM_BUFFER_TRANSFER_SRC_BIT = 0x1,
    PM_BUFFER_TRANSFER_DST_BIT = 0x2,
    PM_BUFFER_GEOMETRY_INPUT_BIT = 0x4,
    PM_BUFFER_PARTICLE_INPUT_BIT = 0x8,
    PM_BUFFER_SIMULATION_OUTPUT_BIT = 0x10
};
typedef struct PmBufferCreateInfo {
    PmStructureType sType;
    const void* pNext;
    PmDeviceSize size;
    PmFlags usage;
    uint32_t initialQueueFamilyIndex;
} PmBufferCreateInfo;
typedef struct PmBufferRange {
    PmBuffer buffer;
    PmDeviceSize offset;
    PmDeviceSize size;
} PmBufferRange;

/* ---- geometry (parallel_mater.h:303-326) ---- */
typedef enum PmFormat {
    PM_FORMAT_UNDEFINED = 0,
    PM_FORMAT_R32_UINT = 1,
    PM_FORMAT_R32_SFLOAT = 2,
    PM_FORMAT_R32G32B32_SFLOAT = 3,
    PM_FORMAT_R32G32B32A32_SFLOAT = 4,
    PM_FORMAT_PARTICLE_STATE = 5,
    PM_FORMAT_RIGID_STATE = 6,
    PM_FORMAT_FLUID_PARTICLE_OUTPUT = 7
} PmFormat;
typedef struct PmBufferView {
    PmBufferRange range;
    PmFormat format;
    uint32_t count;
    uint32_t stride;
} PmBufferView;
typedef struct PmGeometryCreateInfo {
    PmStructureType sType;
    const void* pNext;
    PmBufferView vertices;
    PmBufferView indices;
    uint32_t queueFamilyIndex;
} PmGeometryCreateInfo;

/* ---- simulation (parallel_mater.h:328-390); the per-domain capacity
 * records of other domains are opaque here. ---- */
typedef struct PmFluidCapacity PmFluidCapacity;
typedef struct PmClothCapacity PmClothCapacity;
typedef struct PmRopeCapacity PmRopeCapacity;
typedef struct PmSoftBodyCapacity PmSoftBodyCapacity;
typedef struct PmSmokeCapacity PmSmokeCapacity;
typedef struct PmPaintFieldCapacity PmPaintFieldCapacity;
typedef struct PmSimulationCreateInfo {
    PmStructureType sType;
    const void* pNext;
    uint32_t queueFamilyIndex;
    uint32_t rigidBodyCapacity;
    uint32_t constraintCapacity;
    uint32_t contactCapacity;
    uint32_t fluidCount;
    const PmFluidCapacity* pFluidCapacities;
    uint32_t clothCount;
    const PmClothCapacity* pClothCapacities;
    uint32_t ropeCount;
    const PmRopeCapacity* pRopeCapacities;
    uint32_t softBodyCount;
    const PmSoftBodyCapacity* pSoftBodyCapacities;
    uint32_t smokeCount;
    const PmSmokeCapacity* pSmokeCapacities;
    uint32_t couplingCapacity;
    uint32_t emitterCapacity;
    uint32_t destroyerCapacity;
    uint32_t paintFieldCount;
    const PmPaintFieldCapacity* pPaintFieldCapacities;
    uint32_t paintRuleCapacity;
    uint32_t debugFrameCapacity;
} PmSimulationCreateInfo;
typedef struct PmSimulationMemoryRequirements {
    PmMemoryRequirements persistent;
    PmMemoryRequirements scratch;
} PmSimulationMemoryRequirements;
typedef struct PmSimulationMemoryBinding {
    PmDeviceMemory persistentMemory;
    PmDeviceSize persistentOffset;
    PmDeviceMemory scratchMemory;
    PmDeviceSize scratchOffset;
} PmSimulationMemoryBinding;

/* ---- rigid bodies, inputs, constraints (parallel_mater.h:392-500) ---- */
typedef struct PmRigidState {
    float position[3];
    float orientation[4];
    float linearVelocity[3];
    float angularVelocity[3];
} PmRigidState;
typedef enum PmMotionType { PM_MOTION_STATIC = 0, PM_MOTION_KINEMATIC = 1, PM_MOTION_DYNAMIC = 2 } PmMotionType;
typedef struct PmRigidBodyInfo {
    PmBool32 active;
    PmMotionType motionType;
    PmGeometry geometry;
    PmRigidState state;
    float mass;
    float inertiaDiagonal[3];
    float friction;
    float restitution;
    float linearDamping;
    float angularDamping;
    float maximumLinearSpeed;
    float maximumAngularSpeed;
    float collisionMargin;
    uint64_t userData;
} PmRigidBodyInfo;
typedef struct PmRigidInput {
    uint32_t bodyIndex;
    float force[3];
    float torque[3];
    float linearImpulse[3];
    float angularImpulse[3];
} PmRigidInput;
typedef enum PmConstraintType {
    PM_CONSTRAINT_FIXED = 0,
    PM_CONSTRAINT_POINT = 1,
    PM_CONSTRAINT_HINGE = 2,
    PM_CONSTRAINT_SLIDER = 3,
    PM_CONSTRAINT_PISTON = 4,
    PM_CONSTRAINT_GENERIC = 5,
    PM_CONSTRAINT_GENERIC_SPRING = 6,
    PM_CONSTRAINT_MOTOR = 7
} PmConstraintType;
typedef struct PmConstraintFrame {
    float position[3];
    float orientation[4];
} PmConstraintFrame;
typedef struct PmAxisLimit {
    PmBool32 enabled;
    float lower;
    float upper;
} PmAxisLimit;
typedef struct PmAxisSpring {
    PmBool32 enabled;
    float stiffness;
    float damping;
    float equilibrium;
} PmAxisSpring;
typedef struct PmAxisMotor {
    PmBool32 enabled;
    float targetVelocity;
    float maximumForce;
} PmAxisMotor;
typedef struct PmRigidConstraintInfo {
    PmBool32 active;
    PmConstraintType type;
    uint32_t bodyA;
    uint32_t bodyB;
    PmConstraintFrame frameA;
    PmConstraintFrame frameB;
    PmAxisLimit linearLimits[3];
    PmAxisLimit angularLimits[3];
    PmAxisSpring linearSprings[3];
    PmAxisSpring angularSprings[3];
    PmAxisMotor linearMotors[3];
    PmAxisMotor angularMotors[3];
    PmBool32 collideConnected;
    float breakingImpulseThreshold;
    uint32_t solverIterations;
} PmRigidConstraintInfo;
typedef struct PmRigidSolverState {
    uint32_t rigidIterations;
    PmBool32 enableSleeping;
    float sleepLinearThreshold;
    float sleepAngularThreshold;
    float sleepTimeSeconds;
} PmRigidSolverState;

/* ---- physics pipeline (parallel_mater.h:741-757); material records of
 * other domains are opaque. ---- */
typedef struct PmLiquidMaterialState PmLiquidMaterialState;
typedef struct PmCouplingState PmCouplingState;
typedef struct PmClothMaterialState PmClothMaterialState;
typedef struct PmRopeMaterialState PmRopeMaterialState;
typedef struct PmSoftBodyMaterialState PmSoftBodyMaterialState;
typedef struct PmSmokeMaterialState PmSmokeMaterialState;
typedef struct PmPhysicsPipelineCreateInfo {
    PmStructureType sType;
    const void* pNext;
    const PmRigidSolverState* pRigidState;
    uint32_t fluidMaterialCount;
    const PmLiquidMaterialState* pFluidMaterials;
    uint32_t couplingCount;
    const PmCouplingState* pCouplings;
    uint32_t clothMaterialCount;
    const PmClothMaterialState* pClothMaterials;
    uint32_t ropeMaterialCount;
    const PmRopeMaterialState* pRopeMaterials;
    uint32_t softBodyMaterialCount;
    const PmSoftBodyMaterialState* pSoftBodyMaterials;
    uint32_t smokeMaterialCount;
    const PmSmokeMaterialState* pSmokeMaterials;
} PmPhysicsPipelineCreateInfo;

/* ---- command pools, buffers, steps, copies (parallel_mater.h:985-1030) ---- */
enum { PM_COMMAND_POOL_RESET_BUFFER_BIT = 0x1, PM_COMMAND_BUFFER_ONE_TIME_BIT = 0x1 };
typedef struct PmCommandPoolCreateInfo {
    PmStructureType sType;
    const void* pNext;
    PmFlags flags;
    uint32_t queueFamilyIndex;
} PmCommandPoolCreateInfo;
typedef struct PmCommandBufferBeginInfo {
    PmStructureType sType;
    const void* pNext;
    PmFlags flags;
} PmCommandBufferBeginInfo;
enum { PM_STEP_COLLECT_CONTACT_EVENTS_BIT = 0x1 };
typedef struct PmStepInfo {
    float timestep;
    uint32_t substeps;
    float gravity[3];
    PmFlags flags;
} PmStepInfo;
typedef struct PmBufferCopy {
    PmDeviceSize srcOffset;
    PmDeviceSize dstOffset;
    PmDeviceSize size;
} PmBufferCopy;

/* ---- constraint state records (parallel_mater.h:950-954) ---- */
typedef struct PmConstraintState {
    PmBool32 enabled;
    PmBool32 broken;
    float appliedImpulse;
} PmConstraintState;

/* ---- contact events (parallel_mater.h:759-774, 955-968) ---- */
typedef struct PmFloat3 { float x; float y; float z; } PmFloat3;
typedef struct PmDomainOutputHeader {
    uint32_t activeCount;
    uint32_t capacity;
    uint64_t revision;
} PmDomainOutputHeader;
typedef enum PmContactEventType { PM_CONTACT_RIGID_RIGID = 0, PM_CONTACT_LIQUID_RIGID = 1 } PmContactEventType;
typedef struct PmContactEvent {
    PmContactEventType type;
    uint32_t first;
    uint32_t second;
    PmFloat3 position;
    PmFloat3 normal;
    float penetration;
    float normalImpulse;
    PmFloat3 frictionImpulse;
} PmContactEvent;

/* ---- barriers and synchronisation (parallel_mater.h:1032-1078) ---- */
#define PM_STAGE_HOST_BIT UINT64_C(0x1)
#define PM_STAGE_TRANSFER_BIT UINT64_C(0x2)
#define PM_STAGE_UPDATE_BIT UINT64_C(0x4)
#define PM_STAGE_GEOMETRY_BUILD_BIT UINT64_C(0x8)
#define PM_STAGE_PHYSICS_BIT UINT64_C(0x10)
#define PM_STAGE_ALL_COMMANDS_BIT UINT64_C(0x1e)
#define PM_ACCESS_HOST_READ_BIT UINT64_C(0x1)
#define PM_ACCESS_HOST_WRITE_BIT UINT64_C(0x2)
#define PM_ACCESS_READ_BIT UINT64_C(0x4)
#define PM_ACCESS_WRITE_BIT UINT64_C(0x8)
typedef struct PmMemoryBarrier {
    PmStageFlags srcStages;
    PmAccessFlags srcAccess;
    PmStageFlags dstStages;
    PmAccessFlags dstAccess;
} PmMemoryBarrier;
typedef struct PmBufferMemoryBarrier {
    PmMemoryBarrier memory;
    PmBufferRange range;
    uint32_t srcQueueFamilyIndex;
    uint32_t dstQueueFamilyIndex;
} PmBufferMemoryBarrier;
typedef struct PmSemaphoreCreateInfo {
    PmStructureType sType;
    const void* pNext;
    uint64_t initialValue;
} PmSemaphoreCreateInfo;
typedef struct PmSemaphoreSubmitInfo {
    PmSemaphore semaphore;
    uint64_t value;
    PmStageFlags stages;
} PmSemaphoreSubmitInfo;
typedef struct PmSubmitInfo {
    PmStructureType sType;
    const void* pNext;
    uint32_t waitCount;
    const PmSemaphoreSubmitInfo* pWaits;
    uint32_t commandBufferCount;
    const PmCommandBuffer* pCommandBuffers;
    uint32_t signalCount;
    const PmSemaphoreSubmitInfo* pSignals;
} PmSubmitInfo;
enum { PM_FENCE_SIGNALED_BIT = 0x1 };

/* ---- queries (parallel_mater.h:1127-1163) ---- */
typedef enum PmQueryType {
    PM_QUERY_TIMESTAMP = 0,
    PM_QUERY_STEP_STATISTICS = 1,
    PM_QUERY_REALTIME_STEP_STATISTICS = 2
} PmQueryType;
typedef struct PmQueryPoolCreateInfo {
    PmStructureType sType;
    const void* pNext;
    PmQueryType queryType;
    uint32_t queryCount;
} PmQueryPoolCreateInfo;
typedef struct PmStepStatistics {
    uint64_t stepCount;
    uint64_t substepsExecuted;
    uint64_t poseIterations;
    uint64_t impactIterations;
    uint64_t peakContactCount;
    uint64_t peakActiveBodies;
    uint64_t peakAwakeBodies;
    uint64_t peakParticleCount;
    uint64_t scratchHighWaterBytes;
    uint64_t overflowCount;
    int32_t executionResult;
    uint32_t earlyExitCount;
} PmStepStatistics;
/* ---- realtime step statistics (parallel_mater.h:1154-1193) ---- */
enum { PM_REALTIME_WORK_PHASE_COUNT = 7, PM_REALTIME_DOMAIN_COUNT = 6 };
typedef enum PmRealtimeWorkPhase {
    PM_REALTIME_WORK_PHASE_BOUNDARY = 0,
    PM_REALTIME_WORK_PHASE_PREDICT = 1,
    PM_REALTIME_WORK_PHASE_INDEX = 2,
    PM_REALTIME_WORK_PHASE_CANDIDATES = 3,
    PM_REALTIME_WORK_PHASE_DOMAIN = 4,
    PM_REALTIME_WORK_PHASE_COUPLING = 5,
    PM_REALTIME_WORK_PHASE_COMMIT = 6
} PmRealtimeWorkPhase;
typedef struct PmRealtimeWorkStatistics {
    uint64_t dispatches;
    uint64_t workgroups;
    uint64_t bytesMoved;
    uint64_t spatialIndexBuilds;
    uint64_t spatialIndexRefits;
    uint64_t spatialIndexPublications;
    uint64_t numericalIterations;
    uint64_t barriers;
    uint64_t queueSubmissions;
    uint64_t intraTickHostReadbacks;
    uint64_t intraTickHostWaits;
} PmRealtimeWorkStatistics;
typedef struct PmRealtimeStepStatistics {
    PmStepStatistics step;
    uint32_t schemaVersion;
    uint32_t profileVersion;
    uint32_t budgetVersion;
    uint32_t phaseCount;
    uint64_t tick;
    PmRealtimeWorkStatistics total;
    PmRealtimeWorkStatistics phases[PM_REALTIME_WORK_PHASE_COUNT];
    uint64_t timeAdvances;
    uint64_t domainIterations[PM_REALTIME_DOMAIN_COUNT];
    uint64_t couplingEdgeCount;
    uint64_t couplingSweeps;
} PmRealtimeStepStatistics;
enum { PM_QUERY_RESULT_WAIT_BIT = 0x1, PM_QUERY_RESULT_WITH_AVAILABILITY_BIT = 0x2 };

/* ---- memory budget (parallel_mater.h:1200-1215) ---- */
typedef enum PmMemoryBudgetConfidence {
    PM_MEMORY_BUDGET_CONFIDENCE_UNKNOWN = 0,
    PM_MEMORY_BUDGET_CONFIDENCE_IMPLEMENTATION_ESTIMATE = 1,
    PM_MEMORY_BUDGET_CONFIDENCE_DRIVER_REPORTED = 2,
    PM_MEMORY_BUDGET_CONFIDENCE_OS_REPORTED = 3
} PmMemoryBudgetConfidence;
typedef struct PmMemoryBudget {
    uint32_t heapCount;
    PmDeviceSize budget[16];
    PmDeviceSize usage[16];
    PmMemoryBudgetConfidence confidence[16];
    PmDeviceSize applicationAllocationBytes;
    PmDeviceSize libraryDeviceBytes;
    PmDeviceSize libraryHostBytes;
    PmDeviceSize borrowedBufferBytes;
} PmMemoryBudget;

/* ---- the driver's only exported symbols (pm_driver.h:22-41) ----
 * Every pm* command above is reached through these proc-address lookups,
 * as the reference loader does (src/loader/driver.cpp); none is exported by
 * name. */
#define PM_DRIVER_INTERFACE_VERSION 2u
#define PM_DRIVER_MANIFEST_FILE_VERSION "1.0.0"
#define PM_B200_DRIVER_API __attribute__((visibility("default")))
typedef PmResult(PMAPI_CALL* PFN_pmDriverNegotiateLoaderInterfaceVersion)(uint32_t* pVersion);
typedef PFN_pmVoidFunction(PMAPI_CALL* PFN_pmDriverGetInstanceProcAddr)(PmInstance instance, const char* pName);
typedef PFN_pmVoidFunction(PMAPI_CALL* PFN_pmDriverGetDeviceProcAddr)(PmDevice device, const char* pName);
typedef PFN_pmVoidFunction(PMAPI_CALL* PFN_pmDriverGetPhysicalDeviceProcAddr)(PmInstance instance, const char* pName);
PM_B200_DRIVER_API PmResult PMAPI_CALL pm_driverNegotiateLoaderInterfaceVersion(uint32_t* pVersion);
PM_B200_DRIVER_API PFN_pmVoidFunction PMAPI_CALL pm_driverGetInstanceProcAddr(PmInstance instance, const char* pName);
PM_B200_DRIVER_API PFN_pmVoidFunction PMAPI_CALL pm_driverGetDeviceProcAddr(PmDevice device, const char* pName);
PM_B200_DRIVER_API PFN_pmVoidFunction PMAPI_CALL pm_driverGetPhysicalDeviceProcAddr(PmInstance instance,
                                                                                  const char* pName);

/* ---- the commands this driver resolves (signatures of
 * parallel_mater.h:1726-2128 for these names) ---- */
typedef PmResult(PMAPI_CALL* PFN_pmEnumerateInstanceVersion)(uint32_t* pApiVersion);
typedef PmResult(PMAPI_CALL* PFN_pmCreateInstance)(const PmInstanceCreateInfo* pInfo,
                                                   const PmAllocationCallbacks* pAllocator, PmInstance* pInstance);
typedef void(PMAPI_CALL* PFN_pmDestroyInstance)(PmInstance instance);
typedef PmResult(PMAPI_CALL* PFN_pmEnumeratePhysicalDevices)(PmInstance instance, uint32_t* pCount,
                                                             PmPhysicalDevice* pDevices);
typedef void(PMAPI_CALL* PFN_pmGetPhysicalDeviceProperties)(PmPhysicalDevice physicalDevice,
                                                           PmPhysicalDeviceProperties* pProperties);
typedef PmResult(PMAPI_CALL* PFN_pmGetPhysicalDeviceQueueFamilies)(PmPhysicalDevice physicalDevice, uint32_t* pCount,
                                                                   PmQueueFamilyProperties* pProperties);
typedef void(PMAPI_CALL* PFN_pmGetPhysicalDeviceFeatures)(PmPhysicalDevice physicalDevice,
                                                         PmPhysicalDeviceFeatures* pFeatures);
typedef void(PMAPI_CALL* PFN_pmGetPhysicalDeviceMemoryProperties)(PmPhysicalDevice physicalDevice,
                                                                 PmMemoryProperties* pProperties);
typedef PmResult(PMAPI_CALL* PFN_pmCreateDevice)(PmPhysicalDevice physicalDevice, const PmDeviceCreateInfo* pInfo,
                                                 PmDevice* pDevice);
typedef void(PMAPI_CALL* PFN_pmDestroyDevice)(PmDevice device);
typedef void(PMAPI_CALL* PFN_pmGetDeviceQueue)(PmDevice device, uint32_t family, uint32_t index, PmQueue* pQueue);
typedef PmResult(PMAPI_CALL* PFN_pmAllocateMemory)(PmDevice device, const PmMemoryAllocateInfo* pInfo,
                                                   PmDeviceMemory* pMemory);
typedef void(PMAPI_CALL* PFN_pmFreeMemory)(PmDevice device, PmDeviceMemory memory);
typedef PmResult(PMAPI_CALL* PFN_pmMapMemory)(PmDevice device, PmDeviceMemory memory, PmDeviceSize offset,
                                              PmDeviceSize size, void** ppData);
typedef void(PMAPI_CALL* PFN_pmUnmapMemory)(PmDevice device, PmDeviceMemory memory);
typedef PmResult(PMAPI_CALL* PFN_pmFlushMappedMemoryRanges)(PmDevice device, uint32_t count,
                                                            const PmMappedMemoryRange* pRanges);
typedef PmResult(PMAPI_CALL* PFN_pmInvalidateMappedMemoryRanges)(PmDevice device, uint32_t count,
                                                                 const PmMappedMemoryRange* pRanges);
typedef PmResult(PMAPI_CALL* PFN_pmCreateBuffer)(PmDevice device, const PmBufferCreateInfo* pInfo, PmBuffer* pBuffer);
typedef void(PMAPI_CALL* PFN_pmDestroyBuffer)(PmDevice device, PmBuffer buffer);
typedef void(PMAPI_CALL* PFN_pmGetBufferMemoryRequirements)(PmDevice device, PmBuffer buffer,
                                                           PmMemoryRequirements* pRequirements);
typedef PmResult(PMAPI_CALL* PFN_pmBindBufferMemory)(PmDevice device, PmBuffer buffer, PmDeviceMemory memory,
                                                     PmDeviceSize offset);
typedef PmResult(PMAPI_CALL* PFN_pmCreateGeometry)(PmDevice device, const PmGeometryCreateInfo* pInfo,
                                                   PmGeometry* pGeometry);
typedef void(PMAPI_CALL* PFN_pmDestroyGeometry)(PmDevice device, PmGeometry geometry);
typedef void(PMAPI_CALL* PFN_pmGetGeometryMemoryRequirements)(PmDevice device, PmGeometry geometry,
                                                             PmMemoryRequirements* pRequirements);
typedef PmResult(PMAPI_CALL* PFN_pmBindGeometryMemory)(PmDevice device, PmGeometry geometry, PmDeviceMemory memory,
                                                       PmDeviceSize offset);
typedef PmResult(PMAPI_CALL* PFN_pmCmdBuildGeometry)(PmCommandBuffer commandBuffer, PmGeometry geometry);
typedef PmResult(PMAPI_CALL* PFN_pmCreateSimulation)(PmDevice device, const PmSimulationCreateInfo* pInfo,
                                                     PmSimulation* pSimulation);
typedef void(PMAPI_CALL* PFN_pmDestroySimulation)(PmDevice device, PmSimulation simulation);
typedef void(PMAPI_CALL* PFN_pmGetSimulationMemoryRequirements)(PmDevice device, PmSimulation simulation,
                                                               PmSimulationMemoryRequirements* pInfo);
typedef PmResult(PMAPI_CALL* PFN_pmBindSimulationMemory)(PmDevice device, PmSimulation simulation,
                                                         const PmSimulationMemoryBinding* pBinding);
typedef PmResult(PMAPI_CALL* PFN_pmCmdWriteRigidBodies)(PmCommandBuffer commandBuffer, PmSimulation simulation,
                                                        uint32_t firstBody, uint32_t count,
                                                        const PmRigidBodyInfo* pBodies);
typedef PmResult(PMAPI_CALL* PFN_pmCmdApplyRigidInputs)(PmCommandBuffer commandBuffer, PmSimulation simulation,
                                                        uint32_t count, const PmRigidInput* pInputs);
typedef PmResult(PMAPI_CALL* PFN_pmCmdSetRigidStates)(PmCommandBuffer commandBuffer, PmSimulation simulation,
                                                      uint32_t firstBody, uint32_t count,
                                                      const PmRigidState* pStates);
typedef PmResult(PMAPI_CALL* PFN_pmCmdSetKinematicTargets)(PmCommandBuffer commandBuffer, PmSimulation simulation,
                                                           uint32_t firstBody, uint32_t count,
                                                           const PmRigidState* pTargets);
typedef PmResult(PMAPI_CALL* PFN_pmCmdWriteRigidConstraints)(PmCommandBuffer commandBuffer, PmSimulation simulation,
                                                             uint32_t firstConstraint, uint32_t count,
                                                             const PmRigidConstraintInfo* pConstraints);
typedef PmResult(PMAPI_CALL* PFN_pmCreatePhysicsPipeline)(PmDevice device, const PmPhysicsPipelineCreateInfo* pInfo,
                                                          PmPhysicsPipeline* pPipeline);
typedef void(PMAPI_CALL* PFN_pmDestroyPhysicsPipeline)(PmDevice device, PmPhysicsPipeline pipeline);
typedef PmResult(PMAPI_CALL* PFN_pmCmdCopyConstraintStates)(PmCommandBuffer commandBuffer, PmSimulation simulation,
                                                            uint32_t firstConstraint, uint32_t count,
                                                            const PmBufferRange* pDestination);
typedef PmResult(PMAPI_CALL* PFN_pmCmdCopyContactEvents)(PmCommandBuffer commandBuffer, PmSimulation simulation,
                                                         const PmBufferRange* pDestination);
typedef PmResult(PMAPI_CALL* PFN_pmCreateCommandPool)(PmDevice device, const PmCommandPoolCreateInfo* pInfo,
                                                      PmCommandPool* pPool);
typedef void(PMAPI_CALL* PFN_pmDestroyCommandPool)(PmDevice device, PmCommandPool pool);
typedef PmResult(PMAPI_CALL* PFN_pmResetCommandPool)(PmDevice device, PmCommandPool pool);
typedef PmResult(PMAPI_CALL* PFN_pmAllocateCommandBuffers)(PmDevice device, PmCommandPool pool, uint32_t count,
                                                           PmCommandBuffer* pBuffers);
typedef void(PMAPI_CALL* PFN_pmFreeCommandBuffers)(PmDevice device, PmCommandPool pool, uint32_t count,
                                                  const PmCommandBuffer* pBuffers);
typedef PmResult(PMAPI_CALL* PFN_pmBeginCommandBuffer)(PmCommandBuffer commandBuffer,
                                                       const PmCommandBufferBeginInfo* pInfo);
typedef PmResult(PMAPI_CALL* PFN_pmEndCommandBuffer)(PmCommandBuffer commandBuffer);
typedef PmResult(PMAPI_CALL* PFN_pmResetCommandBuffer)(PmCommandBuffer commandBuffer);
typedef PmResult(PMAPI_CALL* PFN_pmCmdResetSimulation)(PmCommandBuffer commandBuffer, PmSimulation simulation);
typedef PmResult(PMAPI_CALL* PFN_pmCmdBindPhysicsPipeline)(PmCommandBuffer commandBuffer, PmPhysicsPipeline pipeline);
typedef PmResult(PMAPI_CALL* PFN_pmCmdStepSimulation)(PmCommandBuffer commandBuffer, PmSimulation simulation,
                                                      const PmStepInfo* pStep);
typedef PmResult(PMAPI_CALL* PFN_pmCmdCopyBuffer)(PmCommandBuffer commandBuffer, PmBuffer src, PmBuffer dst,
                                                  uint32_t count, const PmBufferCopy* pRegions);
typedef PmResult(PMAPI_CALL* PFN_pmCmdCopyRigidStates)(PmCommandBuffer commandBuffer, PmSimulation simulation,
                                                       uint32_t firstBody, uint32_t count,
                                                       const PmBufferRange* pDestination);
typedef PmResult(PMAPI_CALL* PFN_pmCmdPipelineBarrier)(PmCommandBuffer commandBuffer, uint32_t memoryBarrierCount,
                                                       const PmMemoryBarrier* pMemoryBarriers,
                                                       uint32_t bufferBarrierCount,
                                                       const PmBufferMemoryBarrier* pBufferBarriers);
typedef PmResult(PMAPI_CALL* PFN_pmCreateSemaphore)(PmDevice device, const PmSemaphoreCreateInfo* pInfo,
                                                    PmSemaphore* pSemaphore);
typedef void(PMAPI_CALL* PFN_pmDestroySemaphore)(PmDevice device, PmSemaphore semaphore);
typedef PmResult(PMAPI_CALL* PFN_pmGetSemaphoreCounterValue)(PmDevice device, PmSemaphore semaphore,
                                                             uint64_t* pValue);
typedef PmResult(PMAPI_CALL* PFN_pmWaitSemaphore)(PmDevice device, PmSemaphore semaphore, uint64_t value,
                                                  uint64_t timeoutNanoseconds);
typedef PmResult(PMAPI_CALL* PFN_pmQueueSubmit)(PmQueue queue, const PmSubmitInfo* pInfo, PmFence fence);
typedef PmResult(PMAPI_CALL* PFN_pmQueueWaitIdle)(PmQueue queue);
typedef PmResult(PMAPI_CALL* PFN_pmDeviceWaitIdle)(PmDevice device);
typedef PmResult(PMAPI_CALL* PFN_pmCreateFence)(PmDevice device, PmFlags flags, PmFence* pFence);
typedef void(PMAPI_CALL* PFN_pmDestroyFence)(PmDevice device, PmFence fence);
typedef PmResult(PMAPI_CALL* PFN_pmGetFenceStatus)(PmDevice device, PmFence fence);
typedef PmResult(PMAPI_CALL* PFN_pmResetFences)(PmDevice device, uint32_t count, const PmFence* pFences);
typedef PmResult(PMAPI_CALL* PFN_pmWaitForFences)(PmDevice device, uint32_t count, const PmFence* pFences,
                                                  PmBool32 waitAll, uint64_t timeoutNanoseconds);
typedef PmResult(PMAPI_CALL* PFN_pmCreateQueryPool)(PmDevice device, const PmQueryPoolCreateInfo* pInfo,
                                                    PmQueryPool* pPool);
typedef void(PMAPI_CALL* PFN_pmDestroyQueryPool)(PmDevice device, PmQueryPool pool);
typedef PmResult(PMAPI_CALL* PFN_pmCmdResetQueryPool)(PmCommandBuffer commandBuffer, PmQueryPool pool, uint32_t first,
                                                      uint32_t count);
typedef PmResult(PMAPI_CALL* PFN_pmCmdWriteTimestamp)(PmCommandBuffer commandBuffer, PmStageFlags stage,
                                                      PmQueryPool pool, uint32_t query);
typedef PmResult(PMAPI_CALL* PFN_pmCmdBeginStatisticsQuery)(PmCommandBuffer commandBuffer, PmQueryPool pool,
                                                            uint32_t query);
typedef PmResult(PMAPI_CALL* PFN_pmCmdEndStatisticsQuery)(PmCommandBuffer commandBuffer, PmQueryPool pool,
                                                          uint32_t query);
typedef PmResult(PMAPI_CALL* PFN_pmGetSimulationStatus)(PmDevice device, PmSimulation simulation,
                                                        PmResult* pExecutionResult);
typedef PmResult(PMAPI_CALL* PFN_pmGetQueryPoolResults)(PmDevice device, PmQueryPool pool, uint32_t first,
                                                        uint32_t count, size_t dataSize, void* pData,
                                                        PmDeviceSize stride, PmFlags flags);
typedef PmResult(PMAPI_CALL* PFN_pmGetDeviceMemoryBudget)(PmDevice device, PmMemoryBudget* pBudget);

#ifdef __cplusplus
}
#endif
#endif

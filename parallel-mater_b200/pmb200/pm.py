# SPDX-License-Identifier: MIT
"""ctypes binding of the pm* command API through libpm_b200_driver.so.

The driver exports only the four loader entry points; like the reference
loader (src/loader/driver.cpp) this module negotiates the interface version
and resolves every command with pm_driverGetInstanceProcAddr /
pm_driverGetDeviceProcAddr. Structures mirror include/pm_b200.h, which is
binary compatible with the reference's include/parallel_mater/parallel_mater.h.

``RigidSession`` runs a ``pmb200.scenes.Scene`` through the API the way an
application would: geometry in host-visible memory, a simulation bound to
application memory, bodies and constraints written by commands, one
submission per tick, states copied into a mapped buffer.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

from .scenes import DYNAMIC, KINEMATIC, STATE_DTYPE, Scene

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER_PATH = os.path.join(PKG_DIR, "libpm_b200_driver.so")

u32, i32, u64, f32, vp = C.c_uint32, C.c_int32, C.c_uint64, C.c_float, C.c_void_p

# PmResult
SUCCESS, NOT_READY, TIMEOUT, INCOMPLETE = 0, 1, 2, 3
ERROR_INVALID_ARGUMENT, ERROR_INVALID_STATE, ERROR_FEATURE_NOT_PRESENT = -1, -2, -5
ERROR_CAPACITY_EXCEEDED, ERROR_INCOMPATIBLE_VERSION = -7, -9
# PmStructureType
ST_INSTANCE, ST_DEVICE, ST_MEMORY, ST_BUFFER, ST_GEOMETRY, ST_SIMULATION = 1, 2, 3, 4, 5, 6
ST_PIPELINE, ST_POOL, ST_BEGIN, ST_SEMAPHORE, ST_SUBMIT, ST_QUERY_POOL = 7, 8, 9, 10, 11, 13
API_VERSION_0_3 = (0 << 22) | (3 << 12)
WHOLE_SIZE = 2**64 - 1
TIMEOUT_INFINITE = 2**64 - 1
INVALID_INDEX = 2**32 - 1
FORMAT_R32_UINT, FORMAT_R32G32B32_SFLOAT = 1, 3
STAGE_ALL_COMMANDS = 0x1E
QUERY_TIMESTAMP, QUERY_STEP_STATISTICS, QUERY_REALTIME_STEP_STATISTICS = 0, 1, 2
QUERY_RESULT_WAIT = 1


class PmError(RuntimeError):
    def __init__(self, what, code):
        super().__init__(f"{what} -> {code}")
        self.code = code


def S(name, fields):
    return type(name, (C.Structure,), {"_fields_": fields})


InstanceCreateInfo = S("PmInstanceCreateInfo", [
    ("sType", i32), ("pNext", vp), ("apiVersion", u32), ("pApplicationName", C.c_char_p),
    ("enableValidation", u32), ("enabledLayerCount", u32), ("ppEnabledLayerNames", vp),
    ("enabledExtensionCount", u32), ("ppEnabledExtensionNames", vp)])
FEATURE_NAMES = ["rigidBodies", "rigidConstraints", "particleLiquids", "liquidRigidCoupling",
                 "liquidLiquidCoupling", "cloth", "rope", "softBodies", "smoke", "domainCouplings",
                 "particleEmitters", "paint", "contactEvents", "debugData", "timelineSemaphores",
                 "timestampQueries", "statisticsQueries", "memoryBudget", "vulkanInterop"]
PhysicalDeviceFeatures = S("PmPhysicalDeviceFeatures", [(n, u32) for n in FEATURE_NAMES])
PhysicalDeviceProperties = S("PmPhysicalDeviceProperties", [
    ("apiVersion", u32), ("driverVersion", u32), ("vendorId", u32), ("deviceId", u32),
    ("deviceUuid", C.c_uint8 * 16), ("deviceName", C.c_char * 256)])
QueueFamilyProperties = S("PmQueueFamilyProperties", [
    ("queueFlags", u32), ("queueCount", u32), ("timestampValidBits", u32),
    ("timestampPeriodNanoseconds", f32)])
DeviceQueueCreateInfo = S("PmDeviceQueueCreateInfo", [
    ("queueFamilyIndex", u32), ("queueCount", u32), ("pPriorities", vp)])
DeviceCreateInfo = S("PmDeviceCreateInfo", [
    ("sType", i32), ("pNext", vp), ("queueCreateInfoCount", u32), ("pQueueInfos", vp),
    ("enabledFeatures", PhysicalDeviceFeatures), ("enabledExtensionCount", u32),
    ("ppEnabledExtensionNames", vp)])
MemoryHeap = S("PmMemoryHeap", [("size", u64), ("flags", u32)])
MemoryType = S("PmMemoryType", [("propertyFlags", u32), ("heapIndex", u32)])
MemoryProperties = S("PmMemoryProperties", [
    ("heapCount", u32), ("heaps", MemoryHeap * 16), ("typeCount", u32), ("types", MemoryType * 32)])
MemoryRequirements = S("PmMemoryRequirements", [
    ("size", u64), ("alignment", u64), ("memoryTypeBits", u32), ("requiresDedicatedAllocation", u32)])
MemoryAllocateInfo = S("PmMemoryAllocateInfo", [
    ("sType", i32), ("pNext", vp), ("allocationSize", u64), ("memoryTypeIndex", u32)])
BufferCreateInfo = S("PmBufferCreateInfo", [
    ("sType", i32), ("pNext", vp), ("size", u64), ("usage", u32), ("initialQueueFamilyIndex", u32)])
BufferRange = S("PmBufferRange", [("buffer", vp), ("offset", u64), ("size", u64)])
BufferView = S("PmBufferView", [("range", BufferRange), ("format", i32), ("count", u32), ("stride", u32)])
GeometryCreateInfo = S("PmGeometryCreateInfo", [
    ("sType", i32), ("pNext", vp), ("vertices", BufferView), ("indices", BufferView),
    ("queueFamilyIndex", u32)])
# PmContactEvent (parallel_mater.h:959-968)
PM_EVENT_DTYPE = np.dtype([("type", "<u4"), ("first", "<u4"), ("second", "<u4"), ("position", "<f4", 3),
                           ("normal", "<f4", 3), ("penetration", "<f4"), ("normalImpulse", "<f4"),
                           ("frictionImpulse", "<f4", 3)])
assert PM_EVENT_DTYPE.itemsize == 56

SimulationCreateInfo = S("PmSimulationCreateInfo", [
    ("sType", i32), ("pNext", vp), ("queueFamilyIndex", u32), ("rigidBodyCapacity", u32),
    ("constraintCapacity", u32), ("contactCapacity", u32), ("fluidCount", u32), ("pFluidCapacities", vp),
    ("clothCount", u32), ("pClothCapacities", vp), ("ropeCount", u32), ("pRopeCapacities", vp),
    ("softBodyCount", u32), ("pSoftBodyCapacities", vp), ("smokeCount", u32), ("pSmokeCapacities", vp),
    ("couplingCapacity", u32), ("emitterCapacity", u32), ("destroyerCapacity", u32),
    ("paintFieldCount", u32), ("pPaintFieldCapacities", vp), ("paintRuleCapacity", u32),
    ("debugFrameCapacity", u32)])
SimulationMemoryRequirements = S("PmSimulationMemoryRequirements", [
    ("persistent", MemoryRequirements), ("scratch", MemoryRequirements)])
SimulationMemoryBinding = S("PmSimulationMemoryBinding", [
    ("persistentMemory", vp), ("persistentOffset", u64), ("scratchMemory", vp), ("scratchOffset", u64)])
RigidState = S("PmRigidState", [
    ("position", f32 * 3), ("orientation", f32 * 4), ("linearVelocity", f32 * 3), ("angularVelocity", f32 * 3)])
RigidBodyInfo = S("PmRigidBodyInfo", [
    ("active", u32), ("motionType", i32), ("geometry", vp), ("state", RigidState), ("mass", f32),
    ("inertiaDiagonal", f32 * 3), ("friction", f32), ("restitution", f32), ("linearDamping", f32),
    ("angularDamping", f32), ("maximumLinearSpeed", f32), ("maximumAngularSpeed", f32),
    ("collisionMargin", f32), ("userData", u64)])
RigidInput = S("PmRigidInput", [
    ("bodyIndex", u32), ("force", f32 * 3), ("torque", f32 * 3), ("linearImpulse", f32 * 3),
    ("angularImpulse", f32 * 3)])
ConstraintFrame = S("PmConstraintFrame", [("position", f32 * 3), ("orientation", f32 * 4)])
AxisLimit = S("PmAxisLimit", [("enabled", u32), ("lower", f32), ("upper", f32)])
AxisSpring = S("PmAxisSpring", [("enabled", u32), ("stiffness", f32), ("damping", f32), ("equilibrium", f32)])
AxisMotor = S("PmAxisMotor", [("enabled", u32), ("targetVelocity", f32), ("maximumForce", f32)])
RigidConstraintInfo = S("PmRigidConstraintInfo", [
    ("active", u32), ("type", i32), ("bodyA", u32), ("bodyB", u32), ("frameA", ConstraintFrame),
    ("frameB", ConstraintFrame), ("linearLimits", AxisLimit * 3), ("angularLimits", AxisLimit * 3),
    ("linearSprings", AxisSpring * 3), ("angularSprings", AxisSpring * 3), ("linearMotors", AxisMotor * 3),
    ("angularMotors", AxisMotor * 3), ("collideConnected", u32), ("breakingImpulseThreshold", f32),
    ("solverIterations", u32)])
RigidSolverState = S("PmRigidSolverState", [
    ("rigidIterations", u32), ("enableSleeping", u32), ("sleepLinearThreshold", f32),
    ("sleepAngularThreshold", f32), ("sleepTimeSeconds", f32)])
PhysicsPipelineCreateInfo = S("PmPhysicsPipelineCreateInfo", [
    ("sType", i32), ("pNext", vp), ("pRigidState", vp), ("fluidMaterialCount", u32), ("pFluidMaterials", vp),
    ("couplingCount", u32), ("pCouplings", vp), ("clothMaterialCount", u32), ("pClothMaterials", vp),
    ("ropeMaterialCount", u32), ("pRopeMaterials", vp), ("softBodyMaterialCount", u32),
    ("pSoftBodyMaterials", vp), ("smokeMaterialCount", u32), ("pSmokeMaterials", vp)])
CommandPoolCreateInfo = S("PmCommandPoolCreateInfo", [
    ("sType", i32), ("pNext", vp), ("flags", u32), ("queueFamilyIndex", u32)])
CommandBufferBeginInfo = S("PmCommandBufferBeginInfo", [("sType", i32), ("pNext", vp), ("flags", u32)])
StepInfo = S("PmStepInfo", [("timestep", f32), ("substeps", u32), ("gravity", f32 * 3), ("flags", u32)])
SemaphoreCreateInfo = S("PmSemaphoreCreateInfo", [("sType", i32), ("pNext", vp), ("initialValue", u64)])
SemaphoreSubmitInfo = S("PmSemaphoreSubmitInfo", [("semaphore", vp), ("value", u64), ("stages", u64)])
SubmitInfo = S("PmSubmitInfo", [
    ("sType", i32), ("pNext", vp), ("waitCount", u32), ("pWaits", vp), ("commandBufferCount", u32),
    ("pCommandBuffers", vp), ("signalCount", u32), ("pSignals", vp)])
QueryPoolCreateInfo = S("PmQueryPoolCreateInfo", [
    ("sType", i32), ("pNext", vp), ("queryType", i32), ("queryCount", u32)])
StepStatistics = S("PmStepStatistics", [(n, u64) for n in (
    "stepCount", "substepsExecuted", "poseIterations", "impactIterations", "peakContactCount",
    "peakActiveBodies", "peakAwakeBodies", "peakParticleCount", "scratchHighWaterBytes",
    "overflowCount")] + [("executionResult", i32), ("earlyExitCount", u32)])
REALTIME_PHASES = ("boundary", "predict", "index", "candidates", "domain", "coupling", "commit")
RealtimeWorkStatistics = S("PmRealtimeWorkStatistics", [(n, u64) for n in (
    "dispatches", "workgroups", "bytesMoved", "spatialIndexBuilds", "spatialIndexRefits",
    "spatialIndexPublications", "numericalIterations", "barriers", "queueSubmissions",
    "intraTickHostReadbacks", "intraTickHostWaits")])
RealtimeStepStatistics = S("PmRealtimeStepStatistics", [
    ("step", StepStatistics), ("schemaVersion", u32), ("profileVersion", u32), ("budgetVersion", u32),
    ("phaseCount", u32), ("tick", u64), ("total", RealtimeWorkStatistics),
    ("phases", RealtimeWorkStatistics * len(REALTIME_PHASES)), ("timeAdvances", u64),
    ("domainIterations", u64 * 6), ("couplingEdgeCount", u64), ("couplingSweeps", u64)])
ConstraintState = S("PmConstraintState", [("enabled", u32), ("broken", u32), ("appliedImpulse", f32)])

R = i32  # PmResult
V = None
P = vp
# name -> (restype, argtypes)
SIGNATURES = {
    "pmEnumerateInstanceVersion": (R, [P]),
    "pmCreateInstance": (R, [P, P, P]),
    "pmDestroyInstance": (V, [P]),
    "pmEnumeratePhysicalDevices": (R, [P, P, P]),
    "pmGetPhysicalDeviceProperties": (V, [P, P]),
    "pmGetPhysicalDeviceQueueFamilies": (R, [P, P, P]),
    "pmGetPhysicalDeviceFeatures": (V, [P, P]),
    "pmGetPhysicalDeviceMemoryProperties": (V, [P, P]),
    "pmCreateDevice": (R, [P, P, P]),
    "pmDestroyDevice": (V, [P]),
    "pmGetDeviceQueue": (V, [P, u32, u32, P]),
    "pmAllocateMemory": (R, [P, P, P]),
    "pmFreeMemory": (V, [P, P]),
    "pmMapMemory": (R, [P, P, u64, u64, P]),
    "pmUnmapMemory": (V, [P, P]),
    "pmCreateBuffer": (R, [P, P, P]),
    "pmDestroyBuffer": (V, [P, P]),
    "pmGetBufferMemoryRequirements": (V, [P, P, P]),
    "pmBindBufferMemory": (R, [P, P, P, u64]),
    "pmCreateGeometry": (R, [P, P, P]),
    "pmDestroyGeometry": (V, [P, P]),
    "pmGetGeometryMemoryRequirements": (V, [P, P, P]),
    "pmBindGeometryMemory": (R, [P, P, P, u64]),
    "pmCmdBuildGeometry": (R, [P, P]),
    "pmCreateSimulation": (R, [P, P, P]),
    "pmDestroySimulation": (V, [P, P]),
    "pmGetSimulationMemoryRequirements": (V, [P, P, P]),
    "pmBindSimulationMemory": (R, [P, P, P]),
    "pmGetSimulationStatus": (R, [P, P, P]),
    "pmCmdResetSimulation": (R, [P, P]),
    "pmCmdWriteRigidBodies": (R, [P, P, u32, u32, P]),
    "pmCmdApplyRigidInputs": (R, [P, P, u32, P]),
    "pmCmdSetRigidStates": (R, [P, P, u32, u32, P]),
    "pmCmdSetKinematicTargets": (R, [P, P, u32, u32, P]),
    "pmCmdWriteRigidConstraints": (R, [P, P, u32, u32, P]),
    "pmCreatePhysicsPipeline": (R, [P, P, P]),
    "pmDestroyPhysicsPipeline": (V, [P, P]),
    "pmCmdCopyConstraintStates": (R, [P, P, u32, u32, P]),
    "pmCmdCopyContactEvents": (R, [P, P, P]),
    "pmCreateCommandPool": (R, [P, P, P]),
    "pmDestroyCommandPool": (V, [P, P]),
    "pmResetCommandPool": (R, [P, P]),
    "pmAllocateCommandBuffers": (R, [P, P, u32, P]),
    "pmFreeCommandBuffers": (V, [P, P, u32, P]),
    "pmBeginCommandBuffer": (R, [P, P]),
    "pmEndCommandBuffer": (R, [P]),
    "pmResetCommandBuffer": (R, [P]),
    "pmCmdBindPhysicsPipeline": (R, [P, P]),
    "pmCmdStepSimulation": (R, [P, P, P]),
    "pmCmdCopyBuffer": (R, [P, P, P, u32, P]),
    "pmCmdCopyRigidStates": (R, [P, P, u32, u32, P]),
    "pmCreateSemaphore": (R, [P, P, P]),
    "pmDestroySemaphore": (V, [P, P]),
    "pmGetSemaphoreCounterValue": (R, [P, P, P]),
    "pmWaitSemaphore": (R, [P, P, u64, u64]),
    "pmQueueSubmit": (R, [P, P, P]),
    "pmQueueWaitIdle": (R, [P]),
    "pmDeviceWaitIdle": (R, [P]),
    "pmCreateFence": (R, [P, u32, P]),
    "pmDestroyFence": (V, [P, P]),
    "pmGetFenceStatus": (R, [P, P]),
    "pmResetFences": (R, [P, u32, P]),
    "pmWaitForFences": (R, [P, u32, P, u32, u64]),
    "pmCreateQueryPool": (R, [P, P, P]),
    "pmDestroyQueryPool": (V, [P, P]),
    "pmCmdResetQueryPool": (R, [P, P, u32, u32]),
    "pmCmdWriteTimestamp": (R, [P, u64, P, u32]),
    "pmCmdBeginStatisticsQuery": (R, [P, P, u32]),
    "pmCmdEndStatisticsQuery": (R, [P, P, u32]),
    "pmGetQueryPoolResults": (R, [P, P, u32, u32, C.c_size_t, P, u64, u32]),
    "pmGetDeviceMemoryBudget": (R, [P, P]),
}

_drv = None


def use_driver(path=None):
    """Load the driver from `path` (default: libpm_b200_driver.so) for the
    sessions created afterwards; the test build with failure injection is
    libpm_b200_driver_failtest.so."""
    global _drv, DRIVER_PATH
    DRIVER_PATH = path or os.path.join(PKG_DIR, "libpm_b200_driver.so")
    _drv = None


def driver():
    """The loaded driver with its four entry points typed."""
    global _drv
    if _drv is None:
        if not os.path.exists(DRIVER_PATH):
            raise PmError(f"{DRIVER_PATH} is not built", ERROR_FEATURE_NOT_PRESENT)
        L = C.CDLL(DRIVER_PATH)
        L.pm_driverNegotiateLoaderInterfaceVersion.restype = R
        L.pm_driverNegotiateLoaderInterfaceVersion.argtypes = [P]
        for n in ("pm_driverGetInstanceProcAddr", "pm_driverGetDeviceProcAddr",
                  "pm_driverGetPhysicalDeviceProcAddr"):
            getattr(L, n).restype = vp
            getattr(L, n).argtypes = [P, C.c_char_p]
        _drv = L
    return _drv


def _typed(addr, name):
    res, args = SIGNATURES[name]
    return C.CFUNCTYPE(res, *args)(addr)


class Api:
    """Commands resolved through the driver, as a loader would."""

    def __init__(self, instance=None, device=None):
        self.instance = instance
        self.device = device
        self._cache = {}

    def __getattr__(self, name):
        if not name.startswith("pm"):
            raise AttributeError(name)
        if name not in self._cache:
            L = driver()
            if self.device:
                addr = L.pm_driverGetDeviceProcAddr(self.device, name.encode())
            else:
                addr = L.pm_driverGetInstanceProcAddr(self.instance, name.encode())
            if not addr:
                raise AttributeError(f"{name} is not provided by the driver")
            self._cache[name] = _typed(addr, name)
        return self._cache[name]


def check(rc, what):
    if rc != SUCCESS:
        raise PmError(what, rc)


def ref(x):
    return C.byref(x)


class RigidSession:
    """A Scene driven through the pm* API on one device (realtime profile,
    dt = 1/60 s, one substep, as the reference's command path requires)."""

    def __init__(self, scene: Scene, physical_index=0, iterations=8, contact_capacity=4096, body_infos=None):
        """body_infos: optional {body: {PmRigidBodyInfo field: value}} written
        over the fields derived from the scene (e.g. mass and a zero inertia
        diagonal, which asks the driver for the mesh's box inertia)."""
        self.scene = scene
        boot = Api()
        inst = vp()
        check(boot.pmCreateInstance(ref(InstanceCreateInfo(ST_INSTANCE, None, API_VERSION_0_3)), None, ref(inst)),
              "pmCreateInstance")
        self.instance = inst
        api = Api(instance=inst)
        n = u32(0)
        check(api.pmEnumeratePhysicalDevices(inst, ref(n), None), "pmEnumeratePhysicalDevices")
        if n.value == 0:
            raise PmError("no physical device", ERROR_FEATURE_NOT_PRESENT)
        phys = (vp * n.value)()
        check(api.pmEnumeratePhysicalDevices(inst, ref(n), phys), "pmEnumeratePhysicalDevices")
        self.physical = phys[physical_index]
        feats = PhysicalDeviceFeatures()
        feats.rigidBodies = 1
        feats.rigidConstraints = 1
        feats.timelineSemaphores = 1
        feats.statisticsQueries = 1
        prio = (f32 * 1)(1.0)
        qci = DeviceQueueCreateInfo(0, 1, C.cast(prio, vp))
        dci = DeviceCreateInfo(ST_DEVICE, None, 1, C.cast(C.pointer(qci), vp), feats, 0, None)
        dev = vp()
        check(api.pmCreateDevice(self.physical, ref(dci), ref(dev)), "pmCreateDevice")
        self.dev = dev
        self.api = Api(instance=inst, device=dev)
        q = vp()
        self.api.pmGetDeviceQueue(dev, 0, 0, ref(q))
        self.queue = q
        self._memories = []
        self._buffers = []
        self.geometries = [self._geometry(m) for m in range(len(scene.mesh_vertex_offsets) - 1)]
        # simulation
        sci = SimulationCreateInfo(ST_SIMULATION, None, 0, scene.n, max(len(scene.joints), 0), contact_capacity)
        self.contact_capacity = contact_capacity
        sim = vp()
        check(self.api.pmCreateSimulation(dev, ref(sci), ref(sim)), "pmCreateSimulation")
        self.sim = sim
        req = SimulationMemoryRequirements()
        self.api.pmGetSimulationMemoryRequirements(dev, sim, ref(req))
        self.requirements = (req.persistent.size, req.scratch.size)
        pmem = self._alloc(req.persistent.size, 0)
        smem = self._alloc(req.scratch.size, 0)
        check(self.api.pmBindSimulationMemory(dev, sim, ref(SimulationMemoryBinding(pmem, 0, smem, 0))),
              "pmBindSimulationMemory")
        rs = RigidSolverState(iterations, 0, 0.02, 0.02, 0.5)
        pci = PhysicsPipelineCreateInfo(ST_PIPELINE, None, C.cast(C.pointer(rs), vp))
        pipe = vp()
        check(self.api.pmCreatePhysicsPipeline(dev, ref(pci), ref(pipe)), "pmCreatePhysicsPipeline")
        self.pipeline = pipe
        pool = vp()
        check(self.api.pmCreateCommandPool(dev, ref(CommandPoolCreateInfo(ST_POOL, None, 1, 0)), ref(pool)),
              "pmCreateCommandPool")
        self.pool = pool
        cb = vp()
        check(self.api.pmAllocateCommandBuffers(dev, pool, 1, ref(cb)), "pmAllocateCommandBuffers")
        self.cb = cb
        self.query_pools = {}
        # state read-back buffer in host-visible memory
        self.state_bytes = 52 * scene.n
        self.state_mem, self.state_buf, self.state_ptr = self._mapped_buffer(self.state_bytes)
        # contact-event read-back: PmDomainOutputHeader + PmContactEvent records
        self.event_bytes = 16 + 56 * contact_capacity
        self.event_mem, self.event_buf, self.event_ptr = self._mapped_buffer(self.event_bytes)
        fence = vp()
        check(self.api.pmCreateFence(dev, 0, ref(fence)), "pmCreateFence")
        self.fence = fence
        # constraint-state read-back
        self.constraint_count = len(scene.joints)
        self.cstate_bytes = 12 * max(1, self.constraint_count)
        self.cstate_mem, self.cstate_buf, self.cstate_ptr = self._mapped_buffer(self.cstate_bytes)
        # bodies and constraints
        self.body_infos = self._bodies()
        for i, fields in (body_infos or {}).items():
            for key, value in fields.items():
                if key == "inertiaDiagonal":
                    self.body_infos[i].inertiaDiagonal[:] = [float(v) for v in value]
                else:
                    setattr(self.body_infos[i], key, value)
        self._record(lambda: [
            *[check(self.api.pmCmdBuildGeometry(cb, g), "pmCmdBuildGeometry") for g in self.geometries],
            check(self.api.pmCmdWriteRigidBodies(cb, sim, 0, scene.n, self.body_infos), "pmCmdWriteRigidBodies"),
            self._write_constraints(),
        ])

    # ---- helpers
    def _alloc(self, size, type_index):
        mem = vp()
        check(self.api.pmAllocateMemory(self.dev, ref(MemoryAllocateInfo(ST_MEMORY, None, size, type_index)),
                                        ref(mem)), "pmAllocateMemory")
        self._memories.append(mem)
        return mem

    def _mapped_buffer(self, size):
        size = max(256, (size + 255) // 256 * 256)
        mem = self._alloc(size, 1)
        buf = vp()
        check(self.api.pmCreateBuffer(self.dev, ref(BufferCreateInfo(ST_BUFFER, None, size, 0x1F, 0)), ref(buf)),
              "pmCreateBuffer")
        self._buffers.append(buf)
        check(self.api.pmBindBufferMemory(self.dev, buf, mem, 0), "pmBindBufferMemory")
        ptr = vp()
        check(self.api.pmMapMemory(self.dev, mem, 0, WHOLE_SIZE, ref(ptr)), "pmMapMemory")
        return mem, buf, ptr.value

    def _geometry(self, m):
        s = self.scene
        v0, v1 = int(s.mesh_vertex_offsets[m]), int(s.mesh_vertex_offsets[m + 1])
        i0, i1 = int(s.mesh_index_offsets[m]), int(s.mesh_index_offsets[m + 1])
        verts = np.ascontiguousarray(s.vertices[v0:v1], np.float32)
        idx = np.ascontiguousarray(s.indices[i0:i1], np.uint32)
        vbytes, ibytes = verts.nbytes, idx.nbytes
        ioff = (vbytes + 255) // 256 * 256
        mem, buf, ptr = self._mapped_buffer(ioff + ibytes)
        C.memmove(ptr, verts.ctypes.data, vbytes)
        C.memmove(ptr + ioff, idx.ctypes.data, ibytes)
        gci = GeometryCreateInfo(ST_GEOMETRY, None,
                                 BufferView(BufferRange(buf, 0, vbytes), FORMAT_R32G32B32_SFLOAT, v1 - v0, 12),
                                 BufferView(BufferRange(buf, ioff, ibytes), FORMAT_R32_UINT, i1 - i0, 4), 0)
        g = vp()
        check(self.api.pmCreateGeometry(self.dev, ref(gci), ref(g)), "pmCreateGeometry")
        req = MemoryRequirements()
        self.api.pmGetGeometryMemoryRequirements(self.dev, g, ref(req))
        gmem = self._alloc(req.size, 1)
        check(self.api.pmBindGeometryMemory(self.dev, g, gmem, 0), "pmBindGeometryMemory")
        return g

    def _bodies(self):
        b, st = self.scene.bodies, self.scene.states
        infos = (RigidBodyInfo * self.scene.n)()
        for i in range(self.scene.n):
            x = infos[i]
            x.active = 1
            x.motionType = int(b["motion"][i])
            x.geometry = self.geometries[int(b["mesh"][i])]
            x.state = _state(st[i])
            dyn = int(b["motion"][i]) == DYNAMIC
            inv_m = float(b["inv_mass"][i])
            x.mass = float(np.float32(1.0) / np.float32(inv_m)) if dyn else 0.0
            inv_i = b["inv_inertia"][i]
            for k in range(3):
                x.inertiaDiagonal[k] = float(np.float32(1.0) / np.float32(inv_i[k])) if dyn else 0.0
            x.friction = float(b["friction"][i])
            x.restitution = float(b["restitution"][i])
            x.linearDamping = float(b["linear_damping"][i])
            x.angularDamping = float(b["angular_damping"][i])
            x.maximumLinearSpeed = float(b["max_linear_speed"][i])
            x.maximumAngularSpeed = float(b["max_angular_speed"][i])
            x.collisionMargin = float(b["margin"][i])
        return infos

    def _write_constraints(self, active=None):
        j = self.scene.joints
        if len(j) == 0:
            return
        infos = (RigidConstraintInfo * len(j))()
        for k in range(len(j)):
            c, x = j[k], infos[k]
            x.active = 1 if active is None else int(bool(active[k]))
            x.type = int(c["type"])
            x.bodyA, x.bodyB = int(c["body_a"]), int(c["body_b"])
            x.frameA.position[:] = [float(v) for v in c["anchor_a"]]
            x.frameB.position[:] = [float(v) for v in c["anchor_b"]]
            x.frameA.orientation[:] = [float(v) for v in c["frame_a"]]
            x.frameB.orientation[:] = [float(v) for v in c["frame_b"]]
            for a in range(3):
                x.linearLimits[a] = AxisLimit(int(c["lin_limit_axes"]) >> a & 1, float(c["lin_lower"][a]),
                                              float(c["lin_upper"][a]))
                x.angularLimits[a] = AxisLimit(int(c["ang_limit_axes"]) >> a & 1, float(c["ang_lower"][a]),
                                               float(c["ang_upper"][a]))
                x.linearSprings[a] = AxisSpring(int(c["lin_spring_axes"]) >> a & 1, float(c["lin_stiffness"][a]),
                                                float(c["lin_damping"][a]), 0.0)
                x.angularSprings[a] = AxisSpring(int(c["ang_spring_axes"]) >> a & 1, float(c["ang_stiffness"][a]),
                                                 float(c["ang_damping"][a]), 0.0)
            x.linearMotors[0] = AxisMotor(int(c["motor_linear"]), float(c["motor_linear_velocity"]),
                                          float(c["motor_linear_max_impulse"]))
            x.angularMotors[0] = AxisMotor(int(c["motor_angular"]), float(c["motor_angular_velocity"]),
                                           float(c["motor_angular_max_impulse"]))
            x.collideConnected = 0 if int(c["disable_collisions"]) else 1
            x.breakingImpulseThreshold = float(c["breaking_threshold"])
            x.solverIterations = int(c["solver_iterations"])
        check(self.api.pmCmdWriteRigidConstraints(self.cb, self.sim, 0, len(j), infos),
              "pmCmdWriteRigidConstraints")

    def _record(self, body):
        check(self.api.pmBeginCommandBuffer(self.cb, ref(CommandBufferBeginInfo(ST_BEGIN, None, 0))),
              "pmBeginCommandBuffer")
        body()
        check(self.api.pmEndCommandBuffer(self.cb), "pmEndCommandBuffer")
        return self.submit()

    def submit(self, wait=True):
        cbs = (vp * 1)(self.cb)
        si = SubmitInfo(ST_SUBMIT, None, 0, None, 1, C.cast(cbs, vp), 0, None)
        check(self.api.pmResetFences(self.dev, 1, ref(self.fence)), "pmResetFences")
        check(self.api.pmQueueSubmit(self.queue, ref(si), self.fence), "pmQueueSubmit")
        if wait:
            return self.api.pmWaitForFences(self.dev, 1, ref(self.fence), 1, TIMEOUT_INFINITE)
        return SUCCESS

    # ---- public
    def step(self, gravity=(0.0, -9.81, 0.0), inputs=None, targets=None, states=True, statistics=False,
             events=False, copy_events=None):
        """One tick; returns the submission result. inputs: list of
        (body, force, torque, linear impulse, angular impulse); targets:
        {body: state record}. statistics: wrap the step in a step-statistics
        query, read afterwards with step_statistics(); "realtime" uses a
        realtime query instead (realtime_statistics()). events: collect the
        tick's contact events; copy_events (default: events) records
        pmCmdCopyContactEvents after the step (read with contact_events())."""
        copy_events = events if copy_events is None else copy_events
        step = StepInfo(1.0 / 60.0, 1, (f32 * 3)(*gravity), 1 if events else 0)
        kind = QUERY_REALTIME_STEP_STATISTICS if statistics == "realtime" else QUERY_STEP_STATISTICS
        if statistics and self.query_pools.get(kind) is None:
            qp = vp()
            check(self.api.pmCreateQueryPool(self.dev, ref(QueryPoolCreateInfo(ST_QUERY_POOL, None, kind, 1)),
                                             ref(qp)), "pmCreateQueryPool")
            self.query_pools[kind] = qp
        pool = self.query_pools.get(kind)

        def rec():
            check(self.api.pmCmdBindPhysicsPipeline(self.cb, self.pipeline), "pmCmdBindPhysicsPipeline")
            if inputs:
                arr = (RigidInput * len(inputs))()
                for k, (b, f, t, li, ai) in enumerate(inputs):
                    arr[k] = RigidInput(b, (f32 * 3)(*f), (f32 * 3)(*t), (f32 * 3)(*li), (f32 * 3)(*ai))
                check(self.api.pmCmdApplyRigidInputs(self.cb, self.sim, len(inputs), arr), "pmCmdApplyRigidInputs")
            for b, s in (targets or {}).items():
                t = _state(s)
                check(self.api.pmCmdSetKinematicTargets(self.cb, self.sim, b, 1, ref(t)), "pmCmdSetKinematicTargets")
            if statistics:
                check(self.api.pmCmdResetQueryPool(self.cb, pool, 0, 1), "pmCmdResetQueryPool")
                check(self.api.pmCmdBeginStatisticsQuery(self.cb, pool, 0), "pmCmdBeginStatisticsQuery")
            check(self.api.pmCmdStepSimulation(self.cb, self.sim, ref(step)), "pmCmdStepSimulation")
            if statistics:
                check(self.api.pmCmdEndStatisticsQuery(self.cb, pool, 0), "pmCmdEndStatisticsQuery")
            if states:
                rng = BufferRange(self.state_buf, 0, self.state_bytes)
                check(self.api.pmCmdCopyRigidStates(self.cb, self.sim, 0, self.scene.n, ref(rng)),
                      "pmCmdCopyRigidStates")
            if copy_events:
                rng = BufferRange(self.event_buf, 0, self.event_bytes)
                check(self.api.pmCmdCopyContactEvents(self.cb, self.sim, ref(rng)), "pmCmdCopyContactEvents")
        return self._record(rec)

    def contact_events(self):
        """(activeCount, capacity, revision), PM_EVENT_DTYPE records of the
        last pmCmdCopyContactEvents."""
        raw = bytes((C.c_uint8 * self.event_bytes).from_address(self.event_ptr))
        count, capacity, revision = np.frombuffer(raw[:16], np.dtype([("n", "<u4"), ("c", "<u4"), ("r", "<u8")]))[0]
        return (int(count), int(capacity), int(revision)), np.frombuffer(raw[16:16 + 56 * int(count)],
                                                                         PM_EVENT_DTYPE).copy()

    def write_constraints(self, active):
        """Rewrite every constraint slot with the given active flags
        (pmCmdWriteRigidConstraints: removing or re-adding joints)."""
        return self._record(lambda: self._write_constraints(active))

    def copy_constraint_states(self):
        """Records pmCmdCopyConstraintStates of every slot; returns the
        (enabled, broken, appliedImpulse) records."""
        n = self.constraint_count
        if n == 0:
            return np.zeros(0, np.dtype([("enabled", "<u4"), ("broken", "<u4"), ("applied", "<f4")]))
        rc = self._record(lambda: check(self.api.pmCmdCopyConstraintStates(
            self.cb, self.sim, 0, n, ref(BufferRange(self.cstate_buf, 0, 12 * n))), "pmCmdCopyConstraintStates"))
        check(rc, "copy constraint states")
        raw = bytes((C.c_uint8 * (12 * n)).from_address(self.cstate_ptr))
        return np.frombuffer(raw, np.dtype([("enabled", "<u4"), ("broken", "<u4"), ("applied", "<f4")])).copy()

    def set_states(self, first, states):
        arr = (RigidState * len(states))(*[_state(s) for s in states])
        return self._record(lambda: check(self.api.pmCmdSetRigidStates(self.cb, self.sim, first, len(states), arr),
                                          "pmCmdSetRigidStates"))

    def step_statistics(self):
        """PmStepStatistics of the last step(statistics=True)."""
        out = StepStatistics()
        check(self.api.pmGetQueryPoolResults(self.dev, self.query_pools[QUERY_STEP_STATISTICS], 0, 1,
                                             C.sizeof(out), ref(out), C.sizeof(out), QUERY_RESULT_WAIT),
              "pmGetQueryPoolResults")
        return out

    def realtime_statistics(self):
        """PmRealtimeStepStatistics of the last step(statistics="realtime")."""
        out = RealtimeStepStatistics()
        check(self.api.pmGetQueryPoolResults(self.dev, self.query_pools[QUERY_REALTIME_STEP_STATISTICS], 0, 1,
                                             C.sizeof(out), ref(out), C.sizeof(out), QUERY_RESULT_WAIT),
              "pmGetQueryPoolResults")
        return out

    def states(self):
        buf = (C.c_uint8 * self.state_bytes).from_address(self.state_ptr)
        return np.frombuffer(bytes(buf), STATE_DTYPE).copy()

    def status(self):
        r = i32()
        rc = self.api.pmGetSimulationStatus(self.dev, self.sim, ref(r))
        return rc, r.value

    def close(self):
        if getattr(self, "dev", None) is None:
            return
        a = self.api
        a.pmDeviceWaitIdle(self.dev)
        a.pmDestroyFence(self.dev, self.fence)
        for qp in self.query_pools.values():
            a.pmDestroyQueryPool(self.dev, qp)
        a.pmDestroyCommandPool(self.dev, self.pool)
        a.pmDestroyPhysicsPipeline(self.dev, self.pipeline)
        a.pmDestroySimulation(self.dev, self.sim)
        for g in self.geometries:
            a.pmDestroyGeometry(self.dev, g)
        for b in self._buffers:
            a.pmDestroyBuffer(self.dev, b)
        for m in self._memories:
            a.pmFreeMemory(self.dev, m)
        a.pmDestroyDevice(self.dev)
        a.pmDestroyInstance(self.instance)
        self.dev = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _state(s):
    return RigidState((f32 * 3)(*[float(v) for v in s["x"]]), (f32 * 4)(*[float(v) for v in s["q"]]),
                      (f32 * 3)(*[float(v) for v in s["v"]]), (f32 * 3)(*[float(v) for v in s["w"]]))


def canonical_scene(scene: Scene) -> Scene:
    """The scene as a pm* application describes it: each dynamic body's
    inverse mass and inertia replaced by 1/(1/x) in float32 (the application
    passes mass and inertia; the driver inverts them), and every joint with at
    least one solver iteration (the API's valid range is 1..64). Oracle and
    API runs of the returned scene share every input bit."""
    b = scene.bodies.copy()
    dyn = b["motion"] == DYNAMIC
    one = np.float32(1.0)
    b["inv_mass"][dyn] = one / (one / b["inv_mass"][dyn])
    b["inv_inertia"][dyn] = one / (one / b["inv_inertia"][dyn])
    j = scene.joints.copy()
    if len(j):
        j["solver_iterations"] = np.maximum(j["solver_iterations"], 1)
    return dataclasses.replace(scene, bodies=b, joints=j)


__all__ = ["Api", "RigidSession", "driver", "canonical_scene", "PmError", "KINEMATIC"]

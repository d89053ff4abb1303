// SPDX-License-Identifier: MIT
// Simulations and the rigid-body commands of libpm_b200_driver.so.
//
// A simulation keeps the application's body and constraint slots on the host
// and one pmb_world (the CUDA rigid tick) carved from the persistent and
// scratch memory the application bound. Body or constraint writes mark the
// world stale; the next command that needs it rebuilds it in the same
// memory, carrying over the current state of every body that was not
// rewritten. Bodies take dense indices in slot order. Inputs and kinematic
// targets are merged per body on the host and handed to the device right
// before the tick that consumes them.
//
// Validation follows the reference command by command
// (src/api/resources.cpp:535-1292, src/simulation/runtime.cpp:344-456,
// src/simulation/runtime_rigid.cu.inc); the tick is the realtime v1 profile
// the reference's command path runs (production_realtime_backend.cu.inc:7811-7830).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>

#include "pm_objects.hpp"

using namespace pmd;

namespace {

constexpr float kEpsilon = 1.0e-6f;  // runtime.cpp:96

bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }
bool finite4(const float* v) { return finite3(v) && std::isfinite(v[3]); }
bool finite_state(const PmRigidState& s) {
    return finite3(s.position) && finite4(s.orientation) && finite3(s.linearVelocity) && finite3(s.angularVelocity);
}
bool nonzero_orientation(const float* q) {
    return q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3] > kEpsilon * kEpsilon;
}

// Exact 1/60 s within one ulp on either side (resources.cpp:51-57).
bool realtime_timestep(float value) {
    const float expected = 1.0f / 60.0f;
    return std::isfinite(value) && value >= std::nextafter(expected, 0.0f) &&
           value <= std::nextafter(expected, INFINITY);
}

// validate_body_options (runtime.cpp:344-384).
PmResult validate_body(const PmRigidBodyInfo& b) {
    if (!finite_state(b.state) || !nonzero_orientation(b.state.orientation)) return PM_ERROR_INVALID_ARGUMENT;
    if (b.motionType == PM_MOTION_DYNAMIC && (!std::isfinite(b.mass) || b.mass <= 0.0f))
        return PM_ERROR_INVALID_ARGUMENT;
    const float* i = b.inertiaDiagonal;
    const bool zero = i[0] == 0.0f && i[1] == 0.0f && i[2] == 0.0f;
    if (!finite3(i) || (!zero && (i[0] <= 0.0f || i[1] <= 0.0f || i[2] <= 0.0f))) return PM_ERROR_INVALID_ARGUMENT;
    if (!std::isfinite(b.friction) || b.friction < 0.0f || !std::isfinite(b.restitution) || b.restitution < 0.0f ||
        b.restitution > 1.0f || !std::isfinite(b.linearDamping) || b.linearDamping < 0.0f ||
        !std::isfinite(b.angularDamping) || b.angularDamping < 0.0f || !std::isfinite(b.maximumLinearSpeed) ||
        b.maximumLinearSpeed <= 0.0f || !std::isfinite(b.maximumAngularSpeed) || b.maximumAngularSpeed <= 0.0f ||
        !std::isfinite(b.collisionMargin) || b.collisionMargin <= 0.0f)
        return PM_ERROR_INVALID_ARGUMENT;
    return PM_SUCCESS;
}

// validate_constraint_options (runtime.cpp:390-456) on the converted record.
PmResult validate_constraint(const pmb_joint& j) {
    if (j.body_a == j.body_b) return PM_ERROR_INVALID_ARGUMENT;
    if (!finite3(j.anchor_a) || !finite3(j.anchor_b) || !finite4(j.frame_a) || !finite4(j.frame_b))
        return PM_ERROR_INVALID_ARGUMENT;
    if (!nonzero_orientation(j.frame_a) || !nonzero_orientation(j.frame_b)) return PM_ERROR_INVALID_ARGUMENT;
    const auto limits_ok = [](uint32_t axes, const float* lo, const float* hi) {
        if (!finite3(lo) || !finite3(hi)) return false;
        for (int a = 0; a < 3; ++a)
            if ((axes >> a & 1u) && lo[a] > hi[a]) return false;
        return true;
    };
    const auto springs_ok = [](uint32_t axes, const float* k, const float* c) {
        if (!finite3(k) || !finite3(c)) return false;
        for (int a = 0; a < 3; ++a)
            if ((axes >> a & 1u) && (k[a] < 0.0f || c[a] < 0.0f)) return false;
        return true;
    };
    if (!limits_ok(j.lin_limit_axes, j.lin_lower, j.lin_upper) || !limits_ok(j.ang_limit_axes, j.ang_lower, j.ang_upper))
        return PM_ERROR_INVALID_ARGUMENT;
    if (!springs_ok(j.lin_spring_axes, j.lin_stiffness, j.lin_damping) ||
        !springs_ok(j.ang_spring_axes, j.ang_stiffness, j.ang_damping))
        return PM_ERROR_INVALID_ARGUMENT;
    if (!std::isfinite(j.motor_linear_velocity) || !std::isfinite(j.motor_angular_velocity) ||
        !std::isfinite(j.motor_linear_max_impulse) || j.motor_linear_max_impulse < 0.0f ||
        !std::isfinite(j.motor_angular_max_impulse) || j.motor_angular_max_impulse < 0.0f)
        return PM_ERROR_INVALID_ARGUMENT;
    if (!std::isfinite(j.breaking_threshold) || j.breaking_threshold < 0.0f || j.solver_iterations == 0u ||
        j.solver_iterations > 64u)
        return PM_ERROR_INVALID_ARGUMENT;
    return PM_SUCCESS;
}

// make_parameters (runtime.cpp:459-486): a zero inertia diagonal takes the
// mesh's unit box inertia (runtime_deformables.cu.inc:268-279) times mass.
pmb_body body_parameters(const PmRigidBodyInfo& b, const PmGeometry_T& g) {
    float inertia[3] = {b.inertiaDiagonal[0], b.inertiaDiagonal[1], b.inertiaDiagonal[2]};
    if (inertia[0] == 0.0f && inertia[1] == 0.0f && inertia[2] == 0.0f) {
        float h[3];
        for (int k = 0; k < 3; ++k) h[k] = (g.hi[k] - g.lo[k]) * 0.5f;
        const float unit[3] = {std::fmax((h[1] * h[1] + h[2] * h[2]) / 3.0f, kEpsilon),
                               std::fmax((h[0] * h[0] + h[2] * h[2]) / 3.0f, kEpsilon),
                               std::fmax((h[0] * h[0] + h[1] * h[1]) / 3.0f, kEpsilon)};
        for (int k = 0; k < 3; ++k) inertia[k] = unit[k] * b.mass;
    }
    const bool dynamic = b.motionType == PM_MOTION_DYNAMIC;
    pmb_body p{};
    p.motion = uint32_t(b.motionType);
    p.inv_mass = dynamic ? 1.0f / b.mass : 0.0f;
    for (int k = 0; k < 3; ++k) p.inv_inertia[k] = dynamic ? 1.0f / inertia[k] : 0.0f;
    p.friction = b.friction;
    p.restitution = b.restitution;
    p.linear_damping = b.linearDamping;
    p.angular_damping = b.angularDamping;
    p.max_linear_speed = b.maximumLinearSpeed;
    p.max_angular_speed = b.maximumAngularSpeed;
    p.margin = b.collisionMargin;
    return p;
}

// The public constraint record as the runtime's options
// (resources.cpp:404-436, 1032-1057). Unknown types read as fixed there too.
pmb_joint joint_parameters(const PmRigidConstraintInfo& c) {
    pmb_joint j{};
    j.type = uint32_t(c.type) <= uint32_t(PM_CONSTRAINT_MOTOR) ? uint32_t(c.type) : 0u;
    j.body_a = c.bodyA;
    j.body_b = c.bodyB;
    std::memcpy(j.anchor_a, c.frameA.position, sizeof(j.anchor_a));
    std::memcpy(j.anchor_b, c.frameB.position, sizeof(j.anchor_b));
    std::memcpy(j.frame_a, c.frameA.orientation, sizeof(j.frame_a));
    std::memcpy(j.frame_b, c.frameB.orientation, sizeof(j.frame_b));
    for (uint32_t a = 0; a < 3; ++a) {
        if (c.linearLimits[a].enabled == PM_TRUE) j.lin_limit_axes |= 1u << a;
        j.lin_lower[a] = c.linearLimits[a].lower;
        j.lin_upper[a] = c.linearLimits[a].upper;
        if (c.angularLimits[a].enabled == PM_TRUE) j.ang_limit_axes |= 1u << a;
        j.ang_lower[a] = c.angularLimits[a].lower;
        j.ang_upper[a] = c.angularLimits[a].upper;
        if (c.linearSprings[a].enabled == PM_TRUE) j.lin_spring_axes |= 1u << a;
        j.lin_stiffness[a] = c.linearSprings[a].stiffness;
        j.lin_damping[a] = c.linearSprings[a].damping;
        if (c.angularSprings[a].enabled == PM_TRUE) j.ang_spring_axes |= 1u << a;
        j.ang_stiffness[a] = c.angularSprings[a].stiffness;
        j.ang_damping[a] = c.angularSprings[a].damping;
    }
    j.motor_linear = c.linearMotors[0].enabled == PM_TRUE ? 1u : 0u;
    j.motor_linear_velocity = c.linearMotors[0].targetVelocity;
    j.motor_linear_max_impulse = c.linearMotors[0].maximumForce;
    j.motor_angular = c.angularMotors[0].enabled == PM_TRUE ? 1u : 0u;
    j.motor_angular_velocity = c.angularMotors[0].targetVelocity;
    j.motor_angular_max_impulse = c.angularMotors[0].maximumForce;
    j.enabled = 1u;
    j.disable_collisions = c.collideConnected == PM_FALSE ? 1u : 0u;
    j.breaking_threshold = c.breakingImpulseThreshold;
    j.solver_iterations = c.solverIterations;
    return j;
}

pmb_state to_core(const PmRigidState& s) {
    pmb_state o;
    std::memcpy(&o, &s, sizeof(o));
    return o;
}

void release_world(PmSimulation_T* s) {
    if (s->world) pmb_world_destroy(s->world);
    s->world = nullptr;
    s->dirty = true;
}

// Rebuilds the device world from the slots when they changed.
PmResult ensure_world(PmSimulation_T* s) {
    if (!s->dirty) return PM_SUCCESS;
    if (!s->bound) return PM_ERROR_INVALID_STATE;
    PmDevice_T* device = s->device;
    std::vector<pmb_state> current;
    const std::vector<uint32_t> old_dense = s->dense_of_slot;
    if (s->world) {
        uint32_t n_old = 0;
        for (uint32_t d : old_dense) n_old += d != PM_INVALID_INDEX;
        current.resize(n_old);
        const int r = pmb_world_get_states(s->world, current.data());
        if (r != PMB_SUCCESS) return from_core(r);
        pmb_world_destroy(s->world);
        s->world = nullptr;
    }
    const uint32_t cap = uint32_t(s->bodies.size());
    s->dense_of_slot.assign(cap, PM_INVALID_INDEX);
    std::vector<pmb_body> bodies;
    std::vector<pmb_state> states;
    std::vector<const PmGeometry_T*> meshes;
    std::vector<uint32_t> vertex_offsets{0}, index_offsets{0}, indices;
    std::vector<float> vertices;
    for (uint32_t slot = 0; slot < cap; ++slot) {
        const auto& b = s->bodies[slot];
        if (!b.active) continue;
        const PmGeometry_T* g = b.info.geometry;
        auto found = std::find(meshes.begin(), meshes.end(), g);
        uint32_t mesh = uint32_t(found - meshes.begin());
        if (found == meshes.end()) {
            meshes.push_back(g);
            vertices.insert(vertices.end(), g->vertices.begin(), g->vertices.end());
            indices.insert(indices.end(), g->indices.begin(), g->indices.end());
            vertex_offsets.push_back(uint32_t(vertices.size() / 3));
            index_offsets.push_back(uint32_t(indices.size()));
        }
        pmb_body p = body_parameters(b.info, *g);
        p.mesh = mesh;
        s->dense_of_slot[slot] = uint32_t(bodies.size());
        bodies.push_back(p);
        const bool carry = !s->fresh[slot] && slot < old_dense.size() && old_dense[slot] != PM_INVALID_INDEX &&
                           old_dense[slot] < current.size();
        states.push_back(carry ? current[old_dense[slot]] : to_core(b.info.state));
    }
    std::fill(s->fresh.begin(), s->fresh.end(), 0);
    std::vector<pmb_joint> joints;
    s->joint_of_slot.assign(s->constraints.size(), PM_INVALID_INDEX);
    for (uint32_t slot = 0; slot < s->constraints.size(); ++slot) {
        const auto& c = s->constraints[slot];
        if (!c.active) continue;
        const uint32_t a = s->dense_of_slot[c.info.bodyA], b = s->dense_of_slot[c.info.bodyB];
        if (a == PM_INVALID_INDEX || b == PM_INVALID_INDEX) continue;  // a body of it was removed
        pmb_joint j = joint_parameters(c.info);
        j.body_a = a;
        j.body_b = b;
        s->joint_of_slot[slot] = uint32_t(joints.size());
        joints.push_back(j);
    }
    s->dirty = false;
    if (bodies.empty()) return PM_SUCCESS;
    if (meshes.size() > s->capacity.mesh_count || vertices.size() / 3 > s->capacity.mesh_vertex_count ||
        indices.size() / 3 > s->capacity.mesh_triangle_count)
        return PM_ERROR_CAPACITY_EXCEEDED;
    pmb_world_desc desc{};
    desc.body_count = uint32_t(bodies.size());
    desc.bodies = bodies.data();
    desc.states = states.data();
    desc.mesh_count = uint32_t(meshes.size());
    desc.vertex_offsets = vertex_offsets.data();
    desc.vertices = vertices.data();
    desc.index_offsets = index_offsets.data();
    desc.indices = indices.data();
    desc.joint_count = uint32_t(joints.size());
    desc.joints = joints.data();
    desc.candidate_capacity = s->capacity.candidate_capacity;
    desc.pair_capacity = s->capacity.pair_capacity;
    desc.contact_capacity = s->capacity.contact_capacity;
    desc.event_capacity = s->capacity.event_capacity;
    desc.device = device->ordinal;
    desc.persistent_memory = static_cast<char*>(s->binding.persistentMemory->ptr) + s->binding.persistentOffset;
    desc.persistent_bytes = s->requirements.persistent.size;
    desc.scratch_memory = static_cast<char*>(s->binding.scratchMemory->ptr) + s->binding.scratchOffset;
    desc.scratch_bytes = s->requirements.scratch.size;
    int r = pmb_world_create(&desc, &s->world);
    if (r == PMB_SUCCESS) r = pmb_world_set_stream(s->world, device->stream);
    if (r != PMB_SUCCESS) {
        if (s->world) pmb_world_destroy(s->world);
        s->world = nullptr;
        s->dirty = true;
        return from_core(r);
    }
    return PM_SUCCESS;
}

PmResult require_bound(PmSimulation_T* s) { return s->bound ? PM_SUCCESS : PM_ERROR_INVALID_STATE; }

PmResult status_result(uint32_t status) {
    if (status & PMB_STATUS_BARRIER_TIMEOUT) return PM_ERROR_DEVICE_LOST;
    if (status & (PMB_STATUS_CANDIDATE_OVERFLOW | PMB_STATUS_CONTACT_OVERFLOW | PMB_STATUS_PAIR_OVERFLOW |
                  PMB_STATUS_COLOR_OVERFLOW | PMB_STATUS_GRID_OVERFLOW))
        return PM_ERROR_CAPACITY_EXCEEDED;
    return PM_SUCCESS;
}

// ====================================================================
// simulations (reference src/api/resources.cpp:535-820)
// ====================================================================
PmResult PMAPI_CALL pmCreateSimulation(PmDevice device, const PmSimulationCreateInfo* info,
                                       PmSimulation* simulation) {
    if (!simulation) return PM_ERROR_INVALID_ARGUMENT;
    *simulation = nullptr;
    if (!device || !info || !valid_structure(info->sType, PM_STRUCTURE_TYPE_SIMULATION_CREATE_INFO, info->pNext) ||
        info->queueFamilyIndex != 0u || info->rigidBodyCapacity == 0u)
        return PM_ERROR_INVALID_ARGUMENT;
    // Domains this driver does not provide cannot have been enabled on the
    // device, which the reference reports as an invalid argument.
    if (info->fluidCount || info->clothCount || info->ropeCount || info->softBodyCount || info->smokeCount ||
        info->emitterCapacity || info->paintFieldCount || info->paintRuleCapacity || info->debugFrameCapacity)
        return PM_ERROR_INVALID_ARGUMENT;
    if (device->enabled.rigidBodies != PM_TRUE ||
        (info->constraintCapacity != 0u && device->enabled.rigidConstraints != PM_TRUE))
        return PM_ERROR_INVALID_ARGUMENT;
    auto* created = new (std::nothrow) PmSimulation_T;
    if (!created) return PM_ERROR_OUT_OF_HOST_MEMORY;
    created->device = device;
    created->info = *info;
    created->info.pNext = nullptr;
    const uint32_t n = info->rigidBodyCapacity;
    pmb_world_capacity& c = created->capacity;
    c.body_count = n;
    c.joint_count = info->constraintCapacity;
    c.mesh_count = std::max(16u, n);
    // The simulation holds a copy of every geometry its bodies use (the
    // reference keeps geometry in separate objects, so its create info names
    // no geometry budget). The budget allows a box mesh per body plus 64k
    // vertices and 128k triangles of authored meshes (gears, frames, scanned
    // props): a few MB of persistent memory.
    c.mesh_vertex_count = 65536u + 16u * n;
    c.mesh_triangle_count = 131072u + 32u * n;
    // Contact events kept per tick (resources.cpp:212, contact_capacity),
    // and at least as many contact points (with the triangle-pair work of
    // the mesh path, which is sized like the contact points): authored
    // meshes such as meshing gears make thousands of triangle pairs among a
    // handful of bodies, more than the per-body default allows.
    c.event_capacity = std::max(1u, info->contactCapacity);
    c.contact_capacity = std::max(64u * n + 4096u, info->contactCapacity);
    uint64_t persistent = 0, scratch = 0;
    if (pmb_world_memory_requirements(&c, &persistent, &scratch) != PMB_SUCCESS) {
        delete created;
        return PM_ERROR_INVALID_ARGUMENT;
    }
    const auto round = [](uint64_t v) { return (v + 255u) & ~uint64_t(255u); };
    created->requirements.persistent = {round(persistent), 256u, 0x3u, PM_FALSE};
    created->requirements.scratch = {round(scratch), 256u, 0x3u, PM_FALSE};
    created->bodies.resize(n);
    created->fresh.assign(n, 0);
    created->constraints.resize(info->constraintCapacity);
    created->dense_of_slot.assign(n, PM_INVALID_INDEX);
    *simulation = created;
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmDeviceWaitIdleRigid(PmDevice device) {
    device->worker.wait_idle();
    return from_core(pmb_stream_synchronize(device->ordinal, device->stream));
}

void PMAPI_CALL pmDestroySimulation(PmDevice device, PmSimulation simulation) {
    if (!device || !simulation || simulation->device != device) return;
    (void)pmDeviceWaitIdleRigid(device);
    if (simulation->world) pmb_world_destroy(simulation->world);
    delete simulation;
}

void PMAPI_CALL pmGetSimulationMemoryRequirements(PmDevice device, PmSimulation simulation,
                                                  PmSimulationMemoryRequirements* req) {
    if (!req) return;
    *req = {};
    if (!device || !simulation || simulation->device != device) return;
    *req = simulation->requirements;
}

PmResult PMAPI_CALL pmBindSimulationMemory(PmDevice device, PmSimulation simulation,
                                           const PmSimulationMemoryBinding* binding) {
    if (!device || !simulation || !binding || simulation->device != device || !binding->persistentMemory ||
        !binding->scratchMemory || binding->persistentMemory->device != device ||
        binding->scratchMemory->device != device || binding->persistentOffset % 256u ||
        binding->scratchOffset % 256u)
        return PM_ERROR_INVALID_ARGUMENT;
    const PmSimulationMemoryRequirements& r = simulation->requirements;
    if (!(r.persistent.memoryTypeBits & (1u << binding->persistentMemory->type)) ||
        !(r.scratch.memoryTypeBits & (1u << binding->scratchMemory->type)) ||
        !range_fits(binding->persistentOffset, r.persistent.size, binding->persistentMemory->size) ||
        !range_fits(binding->scratchOffset, r.scratch.size, binding->scratchMemory->size))
        return PM_ERROR_INVALID_ARGUMENT;
    if (binding->persistentMemory == binding->scratchMemory) {
        const PmDeviceSize pe = binding->persistentOffset + r.persistent.size;
        const PmDeviceSize se = binding->scratchOffset + r.scratch.size;
        if (binding->persistentOffset < se && binding->scratchOffset < pe) return PM_ERROR_INVALID_ARGUMENT;
    }
    if (simulation->bound) return PM_ERROR_INVALID_STATE;
    simulation->binding = *binding;
    simulation->bound = true;
    return PM_SUCCESS;
}

PmResult PMAPI_CALL pmGetSimulationStatus(PmDevice device, PmSimulation simulation, PmResult* execution) {
    if (!execution) return PM_ERROR_INVALID_ARGUMENT;
    *execution = PM_ERROR_FEATURE_NOT_PRESENT;
    if (!device || !simulation || simulation->device != device) return PM_ERROR_INVALID_ARGUMENT;
    if (simulation->pending.load() != 0u) return PM_NOT_READY;
    *execution = PmResult(simulation->execution_result.load());
    return PM_SUCCESS;
}

// ====================================================================
// rigid commands
// ====================================================================
PmResult PMAPI_CALL pmCmdResetSimulation(PmCommandBuffer buffer, PmSimulation simulation) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!simulation || simulation->device != buffer->device) return PM_ERROR_INVALID_ARGUMENT;
    return record_simulation(buffer, simulation, [simulation]() -> PmResult {
        const PmResult r = require_bound(simulation);
        if (r != PM_SUCCESS) return r;
        release_world(simulation);
        for (auto& b : simulation->bodies) b = {};
        for (auto& c : simulation->constraints) c = {};
        std::fill(simulation->fresh.begin(), simulation->fresh.end(), 0);
        simulation->inputs.clear();
        simulation->targets.clear();
        simulation->last = {};
        return PM_SUCCESS;
    });
}

PmResult PMAPI_CALL pmCmdWriteRigidBodies(PmCommandBuffer buffer, PmSimulation simulation, uint32_t first,
                                          uint32_t count, const PmRigidBodyInfo* bodies) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!simulation || simulation->device != buffer->device || count == 0u || !bodies ||
        first > simulation->bodies.size() || count > simulation->bodies.size() - first)
        return PM_ERROR_INVALID_ARGUMENT;
    std::vector<PmRigidBodyInfo> copied(bodies, bodies + count);
    for (const auto& b : copied)
        if (b.active != PM_FALSE && (!b.geometry || !finite_state(b.state) || uint32_t(b.motionType) > 2u))
            return PM_ERROR_INVALID_ARGUMENT;
    return record_simulation(buffer, simulation, [simulation, first, copied]() -> PmResult {
        PmResult r = require_bound(simulation);
        if (r != PM_SUCCESS) return r;
        for (uint32_t k = 0; k < copied.size(); ++k) {
            const uint32_t slot = first + k;
            auto& body = simulation->bodies[slot];
            body = {};
            simulation->fresh[slot] = 1;
            simulation->inputs.erase(slot);
            simulation->targets.erase(slot);
            simulation->dirty = true;
            const PmRigidBodyInfo& src = copied[k];
            if (src.active == PM_FALSE) continue;
            if (src.geometry->device != simulation->device) return PM_ERROR_INVALID_ARGUMENT;
            if (!src.geometry->built) return PM_ERROR_INVALID_STATE;
            r = validate_body(src);
            if (r != PM_SUCCESS) return r;
            body.active = true;
            body.info = src;
        }
        return PM_SUCCESS;
    });
}

PmResult PMAPI_CALL pmCmdApplyRigidInputs(PmCommandBuffer buffer, PmSimulation simulation, uint32_t count,
                                          const PmRigidInput* inputs) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!simulation || simulation->device != buffer->device || count == 0u || !inputs) return PM_ERROR_INVALID_ARGUMENT;
    std::vector<PmRigidInput> copied(inputs, inputs + count);
    for (const auto& in : copied)
        if (in.bodyIndex >= simulation->bodies.size()) return PM_ERROR_INVALID_ARGUMENT;
    return record_simulation(buffer, simulation, [simulation, copied]() -> PmResult {
        for (const auto& in : copied) {
            const auto& body = simulation->bodies[in.bodyIndex];
            if (!body.active) return PM_ERROR_INVALID_STATE;
            if (!finite3(in.force) || !finite3(in.torque) || !finite3(in.linearImpulse) || !finite3(in.angularImpulse))
                return PM_ERROR_INVALID_ARGUMENT;
            if (body.info.motionType != PM_MOTION_DYNAMIC) return PM_ERROR_INVALID_ARGUMENT;
            // Accumulate like runtime_rigid.cu.inc:288-292.
            auto it = simulation->inputs.find(in.bodyIndex);
            if (it == simulation->inputs.end())
                it = simulation->inputs.emplace(in.bodyIndex, std::array<float, 12>{}).first;
            const float* v[4] = {in.force, in.torque, in.linearImpulse, in.angularImpulse};
            for (int f = 0; f < 4; ++f)
                for (int a = 0; a < 3; ++a) it->second[3 * f + a] = it->second[3 * f + a] + v[f][a];
        }
        return PM_SUCCESS;
    });
}

PmResult PMAPI_CALL pmCmdSetRigidStates(PmCommandBuffer buffer, PmSimulation simulation, uint32_t first,
                                        uint32_t count, const PmRigidState* states) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!simulation || simulation->device != buffer->device || count == 0u || !states ||
        first > simulation->bodies.size() || count > simulation->bodies.size() - first)
        return PM_ERROR_INVALID_ARGUMENT;
    std::vector<PmRigidState> copied(states, states + count);
    return record_simulation(buffer, simulation, [simulation, first, copied]() -> PmResult {
        PmResult r = require_bound(simulation);
        if (r != PM_SUCCESS) return r;
        for (uint32_t k = 0; k < copied.size(); ++k) {
            if (!simulation->bodies[first + k].active) return PM_ERROR_INVALID_STATE;
            if (!finite_state(copied[k]) || !nonzero_orientation(copied[k].orientation))
                return PM_ERROR_INVALID_ARGUMENT;
        }
        r = ensure_world(simulation);
        if (r != PM_SUCCESS) return r;
        for (uint32_t k = 0; k < copied.size(); ++k) {
            const uint32_t slot = first + k;
            simulation->inputs.erase(slot);
            simulation->targets.erase(slot);
            const pmb_state s = to_core(copied[k]);
            const int rc = pmb_world_write_states(simulation->world, simulation->dense_of_slot[slot], 1u, &s);
            if (rc != PMB_SUCCESS) return from_core(rc);
        }
        return PM_SUCCESS;
    });
}

PmResult PMAPI_CALL pmCmdSetKinematicTargets(PmCommandBuffer buffer, PmSimulation simulation, uint32_t first,
                                             uint32_t count, const PmRigidState* targets) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!simulation || simulation->device != buffer->device || count == 0u || !targets ||
        first > simulation->bodies.size() || count > simulation->bodies.size() - first)
        return PM_ERROR_INVALID_ARGUMENT;
    std::vector<PmRigidState> copied(targets, targets + count);
    for (const auto& t : copied)
        if (!finite_state(t)) return PM_ERROR_INVALID_ARGUMENT;
    return record_simulation(buffer, simulation, [simulation, first, copied]() -> PmResult {
        for (uint32_t k = 0; k < copied.size(); ++k) {
            const auto& body = simulation->bodies[first + k];
            if (!body.active) return PM_ERROR_INVALID_STATE;
            if (body.info.motionType != PM_MOTION_KINEMATIC) return PM_ERROR_INVALID_ARGUMENT;
            if (!nonzero_orientation(copied[k].orientation)) return PM_ERROR_INVALID_ARGUMENT;
            simulation->targets[first + k] = copied[k];
        }
        return PM_SUCCESS;
    });
}

PmResult PMAPI_CALL pmCmdWriteRigidConstraints(PmCommandBuffer buffer, PmSimulation simulation, uint32_t first,
                                               uint32_t count, const PmRigidConstraintInfo* constraints) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!simulation || simulation->device != buffer->device || count == 0u || !constraints ||
        first > simulation->constraints.size() || count > simulation->constraints.size() - first)
        return PM_ERROR_INVALID_ARGUMENT;
    std::vector<PmRigidConstraintInfo> copied(constraints, constraints + count);
    return record_simulation(buffer, simulation, [simulation, first, copied]() -> PmResult {
        for (uint32_t k = 0; k < copied.size(); ++k) {
            auto& slot = simulation->constraints[first + k];
            slot = {};
            simulation->dirty = true;
            const auto& src = copied[k];
            if (src.active == PM_FALSE) continue;
            const size_t cap = simulation->bodies.size();
            if (src.bodyA >= cap || src.bodyB == PM_INVALID_INDEX || src.bodyB >= cap ||
                !simulation->bodies[src.bodyA].active || !simulation->bodies[src.bodyB].active)
                return PM_ERROR_INVALID_ARGUMENT;
            const PmResult r = validate_constraint(joint_parameters(src));
            if (r != PM_SUCCESS) return r;
            slot.active = true;
            slot.info = src;
        }
        return PM_SUCCESS;
    });
}

PmResult PMAPI_CALL pmCmdStepSimulation(PmCommandBuffer buffer, PmSimulation simulation, const PmStepInfo* step) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!simulation || !step || !(step->timestep > 0.0f) || step->substeps == 0u ||
        simulation->device != buffer->device || !buffer->bound_pipeline ||
        (step->flags & ~PmFlags(PM_STEP_COLLECT_CONTACT_EVENTS_BIT)) != 0u)
        return PM_ERROR_INVALID_ARGUMENT;
    if (!realtime_timestep(step->timestep) || step->substeps != 1u) return PM_ERROR_INVALID_ARGUMENT;
    if (buffer->statistics_open && buffer->statistics_pool->type == PM_QUERY_REALTIME_STEP_STATISTICS &&
        buffer->statistics_step_count != 0u)
        return PM_ERROR_INVALID_ARGUMENT;  // one step per realtime statistics query (resources.cpp:1243-1246)
    const PmStepInfo copied = *step;
    const uint32_t iterations = buffer->bound_pipeline->rigid.rigidIterations;
    const PmResult recorded = record_simulation(buffer, simulation, [simulation, copied, iterations]() -> PmResult {
        PmResult r = require_bound(simulation);
        if (r == PM_SUCCESS) r = ensure_world(simulation);
        if (r == PM_SUCCESS && simulation->world) {
            pmb_world* w = simulation->world;
            // Inputs and targets gathered since the last tick.
            if (!simulation->inputs.empty()) {
                std::vector<uint32_t> bodies;
                std::vector<float> values;
                for (const auto& kv : simulation->inputs) {
                    bodies.push_back(simulation->dense_of_slot[kv.first]);
                    values.insert(values.end(), kv.second.begin(), kv.second.end());
                }
                r = from_core(pmb_world_set_inputs(w, uint32_t(bodies.size()), bodies.data(), values.data()));
                simulation->inputs.clear();
            }
            if (r == PM_SUCCESS && !simulation->targets.empty()) {
                std::vector<uint32_t> bodies;
                std::vector<pmb_state> targets;
                for (const auto& kv : simulation->targets) {
                    bodies.push_back(simulation->dense_of_slot[kv.first]);
                    targets.push_back(to_core(kv.second));
                }
                r = from_core(pmb_world_set_targets(w, uint32_t(bodies.size()), bodies.data(), targets.data()));
                simulation->targets.clear();
            }
#if defined(PMB_TEST_FAILURE_DRIVER)
            // Test build only: a device upload that fails at execution
            // (reference src/device/cpu_device.cpp:151-153, reported through
            // the fence), and grid-barrier waits bounded to a given number of
            // polls so that they run out (a bounded wait, never a fault).
            if (r == PM_SUCCESS && std::getenv("PM_TEST_FAIL_UPLOAD") != nullptr) r = PM_ERROR_OUT_OF_DEVICE_MEMORY;
            if (r == PM_SUCCESS) {
                const char* spins = std::getenv("PM_TEST_BARRIER_SPINS");
                r = from_core(pmb_world_set_barrier_limit(w, spins ? uint32_t(std::strtoul(spins, nullptr, 10)) : 0u));
            }
#endif
            if (r == PM_SUCCESS) {
                pmb_step_desc sd{};
                sd.dt = copied.timestep;
                std::memcpy(sd.gravity, copied.gravity, sizeof(sd.gravity));
                sd.profile = 1u;  // realtime v1
                sd.requested_iterations = iterations;
                sd.base_iterations = iterations;
                sd.collect_events = (copied.flags & PM_STEP_COLLECT_CONTACT_EVENTS_BIT) ? 1u : 0u;
                pmb_step_stats stats{};
                r = from_core(pmb_world_step(w, &sd, &stats));
                if (r == PM_SUCCESS) {
                    simulation->last = stats;
                    r = status_result(stats.status);
                }
            }
        }
        simulation->execution_result.store(r);
        if (r == PM_SUCCESS) {
            ++simulation->submitted_steps;
            simulation->last_substeps = copied.substeps;
        }
        return r;
    });
    if (recorded == PM_SUCCESS && buffer->statistics_open) {
        buffer->statistics_simulation = simulation;
        ++buffer->statistics_step_count;
    }
    return recorded;
}

PmResult PMAPI_CALL pmCmdCopyRigidStates(PmCommandBuffer buffer, PmSimulation simulation, uint32_t first,
                                         uint32_t count, const PmBufferRange* destination) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!simulation || !destination || simulation->device != buffer->device || !destination->buffer ||
        destination->buffer->device != buffer->device || first > simulation->bodies.size() ||
        count > simulation->bodies.size() - first ||
        destination->size < PmDeviceSize(count) * sizeof(PmRigidState) ||
        !range_fits(destination->offset, destination->size, destination->buffer->size))
        return PM_ERROR_INVALID_ARGUMENT;
    const PmBufferRange copied = *destination;
    return record_simulation(buffer, simulation, [simulation, first, count, copied]() -> PmResult {
        if (!copied.buffer->ptr || copied.buffer->queue_family != 0u) return PM_ERROR_INVALID_STATE;
        PmResult r = require_bound(simulation);
        if (r == PM_SUCCESS) r = ensure_world(simulation);
        if (r != PM_SUCCESS) return r;
        char* target = copied.buffer->ptr + copied.offset;
        for (uint32_t k = 0; k < count;) {
            const uint32_t dense = simulation->dense_of_slot[first + k];
            if (dense == PM_INVALID_INDEX || !simulation->world) return PM_ERROR_INVALID_STATE;
            uint32_t run = 1;
            while (k + run < count && simulation->dense_of_slot[first + k + run] == dense + run) ++run;
            const int rc = pmb_world_copy_states_to_device(simulation->world, dense, run,
                                                           target + size_t(k) * sizeof(PmRigidState));
            if (rc != PMB_SUCCESS) return from_core(rc);
            k += run;
        }
        return PM_SUCCESS;
    });
}

// pmCmdCopyContactEvents (reference src/api/domains.cpp:1692-1746): a
// PmDomainOutputHeader {events, simulation contact capacity, steps taken}
// followed by the last tick's rigid-rigid events, bodies as application
// slots. Capacity-exceeded when the range cannot hold them all.
PmResult PMAPI_CALL pmCmdCopyContactEvents(PmCommandBuffer buffer, PmSimulation simulation,
                                           const PmBufferRange* destination) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    if (!destination || !destination->buffer || destination->buffer->device != buffer->device ||
        destination->size < sizeof(PmDomainOutputHeader) ||
        !range_fits(destination->offset, destination->size, destination->buffer->size) || !simulation ||
        simulation->device != buffer->device)
        return PM_ERROR_INVALID_ARGUMENT;
    const PmBufferRange copied = *destination;
    PmDevice_T* device = buffer->device;
    return record_simulation(buffer, simulation, [simulation, copied, device]() -> PmResult {
        if (!copied.buffer->ptr) return PM_ERROR_INVALID_STATE;
        std::vector<pmb_contact_event> events;
        if (simulation->world) {
            uint32_t n = 0;
            int rc = pmb_world_contact_events(simulation->world, nullptr, 0, &n);
            if (rc == PMB_SUCCESS && n) {
                events.resize(n);
                rc = pmb_world_contact_events(simulation->world, events.data(), n, &n);
            }
            if (rc != PMB_SUCCESS) return from_core(rc);
        }
        std::vector<uint32_t> slot_of_dense(simulation->dense_of_slot.size(), PM_INVALID_INDEX);
        for (uint32_t slot = 0; slot < simulation->dense_of_slot.size(); ++slot)
            if (simulation->dense_of_slot[slot] != PM_INVALID_INDEX)
                slot_of_dense[simulation->dense_of_slot[slot]] = slot;
        const auto slot = [&](uint32_t dense) {
            return dense < slot_of_dense.size() ? slot_of_dense[dense] : PM_INVALID_INDEX;
        };
        const PmDeviceSize required =
            sizeof(PmDomainOutputHeader) + PmDeviceSize(events.size()) * sizeof(PmContactEvent);
        if (required > copied.size) return PM_ERROR_CAPACITY_EXCEEDED;
        std::vector<char> staging(static_cast<size_t>(required));
        const PmDomainOutputHeader header{uint32_t(events.size()), simulation->capacity.event_capacity,
                                          simulation->submitted_steps};
        std::memcpy(staging.data(), &header, sizeof(header));
        for (size_t k = 0; k < events.size(); ++k) {
            const pmb_contact_event& e = events[k];
            PmContactEvent t{};
            t.type = PM_CONTACT_RIGID_RIGID;
            t.first = slot(e.body);
            t.second = slot(e.collider);
            t.position = {e.position[0], e.position[1], e.position[2]};
            t.normal = {e.normal[0], e.normal[1], e.normal[2]};
            t.penetration = e.penetration;
            t.normalImpulse = e.normal_impulse;
            t.frictionImpulse = {e.friction_impulse[0], e.friction_impulse[1], e.friction_impulse[2]};
            std::memcpy(staging.data() + sizeof(header) + k * sizeof(PmContactEvent), &t, sizeof(t));
        }
        int rc = pmb_copy_async(device->ordinal, copied.buffer->ptr + copied.offset, staging.data(),
                                uint64_t(required), device->stream);
        if (rc == PMB_SUCCESS) rc = pmb_stream_synchronize(device->ordinal, device->stream);
        return from_core(rc);
    });
}

PmResult PMAPI_CALL pmCmdCopyConstraintStates(PmCommandBuffer buffer, PmSimulation simulation, uint32_t first,
                                              uint32_t count, const PmBufferRange* destination) {
    const PmResult state = require_recording(buffer);
    if (state != PM_SUCCESS) return state;
    const PmDeviceSize bytes = PmDeviceSize(count) * sizeof(PmConstraintState);
    if (!destination || !destination->buffer || destination->buffer->device != buffer->device ||
        destination->size < bytes || !range_fits(destination->offset, destination->size, destination->buffer->size) ||
        !simulation || simulation->device != buffer->device || count == 0u || first > simulation->constraints.size() ||
        count > simulation->constraints.size() - first)
        return PM_ERROR_INVALID_ARGUMENT;
    const PmBufferRange copied = *destination;
    PmDevice_T* device = buffer->device;
    return record_simulation(buffer, simulation, [simulation, first, count, copied, device]() -> PmResult {
        if (!copied.buffer->ptr) return PM_ERROR_INVALID_STATE;
        PmResult r = require_bound(simulation);
        if (r == PM_SUCCESS) r = ensure_world(simulation);
        if (r != PM_SUCCESS) return r;
        const uint32_t nj = uint32_t(std::count_if(simulation->joint_of_slot.begin(), simulation->joint_of_slot.end(),
                                                   [](uint32_t j) { return j != PM_INVALID_INDEX; }));
        std::vector<uint32_t> flags(std::max(1u, nj));
        std::vector<float> applied(std::max(1u, nj));
        if (simulation->world && nj) {
            const int rc = pmb_world_joints(simulation->world, flags.data(), applied.data(), nullptr, nj);
            if (rc != PMB_SUCCESS) return from_core(rc);
        }
        std::vector<PmConstraintState> out(count);
        for (uint32_t k = 0; k < count; ++k) {
            const uint32_t j = simulation->joint_of_slot.empty() ? PM_INVALID_INDEX : simulation->joint_of_slot[first + k];
            if (j == PM_INVALID_INDEX || !simulation->world)
                out[k] = {PM_FALSE, PM_FALSE, 0.0f};
            else
                out[k] = {(flags[j] & 1u) ? PM_TRUE : PM_FALSE, (flags[j] & 2u) ? PM_TRUE : PM_FALSE, applied[j]};
        }
        int rc = pmb_copy_async(device->ordinal, copied.buffer->ptr + copied.offset, out.data(),
                                uint64_t(count) * sizeof(PmConstraintState), device->stream);
        if (rc == PMB_SUCCESS) rc = pmb_stream_synchronize(device->ordinal, device->stream);
        return from_core(rc);
    });
}

}  // namespace

namespace pmd {

void fill_statistics(PmSimulation_T* s, PmStepStatistics& out) {
    out = {};
    uint64_t bodies = 0;
    for (uint32_t d : s->dense_of_slot) bodies += d != PM_INVALID_INDEX;
    out.stepCount = s->submitted_steps;
    out.substepsExecuted = s->last_substeps;
    out.poseIterations = s->last.iterations;
    out.impactIterations = 0;  // the realtime profile has no velocity phase
    out.peakContactCount = s->last.contacts;
    out.peakActiveBodies = bodies;
    out.peakAwakeBodies = bodies;  // sleeping is not part of this tick
    out.scratchHighWaterBytes = s->world ? s->requirements.scratch.size : 0u;
    const uint32_t overflow = PMB_STATUS_CANDIDATE_OVERFLOW | PMB_STATUS_CONTACT_OVERFLOW | PMB_STATUS_PAIR_OVERFLOW |
                              PMB_STATUS_COLOR_OVERFLOW | PMB_STATUS_GRID_OVERFLOW;
    out.overflowCount = uint64_t(__builtin_popcount(s->last.status & overflow));
    out.executionResult = s->execution_result.load();
    out.earlyExitCount = 0;
}

// Realtime step statistics (reference src/api/queries.cpp:215-250): the
// latest tick's telemetry from the core library, in the reference's work
// phases. The tick issues one queue submission, reads nothing back and waits
// for nothing inside itself; one spatial index is built and published.
PmResult fill_realtime_statistics(PmSimulation_T* s, PmRealtimeStepStatistics& out) {
    out = {};
    out.schemaVersion = 1;
    out.profileVersion = 1;
    out.budgetVersion = 1;
    out.phaseCount = PM_REALTIME_WORK_PHASE_COUNT;
    out.tick = s->submitted_steps;
    if (!s->world) return PM_SUCCESS;
    pmb_tick_telemetry t{};
    const int rc = pmb_world_tick_telemetry(s->world, &t);
    if (rc != PMB_SUCCESS) return from_core(rc);
    for (int p = 0; p < PM_REALTIME_WORK_PHASE_COUNT; ++p) {
        PmRealtimeWorkStatistics& w = out.phases[p];
        w.dispatches = t.dispatches[p];
        w.workgroups = t.workgroups[p];
        w.bytesMoved = t.bytes_moved[p];
        w.barriers = t.barriers[p];
    }
    out.phases[PM_REALTIME_WORK_PHASE_INDEX].spatialIndexBuilds = t.spatial_builds;
    out.phases[PM_REALTIME_WORK_PHASE_INDEX].spatialIndexPublications = t.spatial_builds;
    out.phases[PM_REALTIME_WORK_PHASE_DOMAIN].numericalIterations = t.sweeps;
    out.phases[PM_REALTIME_WORK_PHASE_BOUNDARY].queueSubmissions = 1;
    for (const auto& w : out.phases) {
        out.total.dispatches += w.dispatches;
        out.total.workgroups += w.workgroups;
        out.total.bytesMoved += w.bytesMoved;
        out.total.spatialIndexBuilds += w.spatialIndexBuilds;
        out.total.spatialIndexRefits += w.spatialIndexRefits;
        out.total.spatialIndexPublications += w.spatialIndexPublications;
        out.total.numericalIterations += w.numericalIterations;
        out.total.barriers += w.barriers;
        out.total.queueSubmissions += w.queueSubmissions;
        out.total.intraTickHostReadbacks += w.intraTickHostReadbacks;
        out.total.intraTickHostWaits += w.intraTickHostWaits;
    }
    out.timeAdvances = s->execution_result.load() == PM_SUCCESS ? 1u : 0u;
    out.domainIterations[0] = t.sweeps;  // rigid contact and joint sweeps
    return PM_SUCCESS;
}

PFN_pmVoidFunction lookup_rigid(const char* name) {
#define PM_ENTRY(fn) \
    if (std::strcmp(name, #fn) == 0) return reinterpret_cast<PFN_pmVoidFunction>(&fn);
    PM_ENTRY(pmCreateSimulation)
    PM_ENTRY(pmDestroySimulation)
    PM_ENTRY(pmGetSimulationMemoryRequirements)
    PM_ENTRY(pmBindSimulationMemory)
    PM_ENTRY(pmGetSimulationStatus)
    PM_ENTRY(pmCmdResetSimulation)
    PM_ENTRY(pmCmdWriteRigidBodies)
    PM_ENTRY(pmCmdApplyRigidInputs)
    PM_ENTRY(pmCmdSetRigidStates)
    PM_ENTRY(pmCmdSetKinematicTargets)
    PM_ENTRY(pmCmdWriteRigidConstraints)
    PM_ENTRY(pmCmdStepSimulation)
    PM_ENTRY(pmCmdCopyRigidStates)
    PM_ENTRY(pmCmdCopyConstraintStates)
    PM_ENTRY(pmCmdCopyContactEvents)
#undef PM_ENTRY
    return nullptr;
}

}  // namespace pmd

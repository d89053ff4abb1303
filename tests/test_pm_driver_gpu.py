# SPDX-License-Identifier: MIT
"""The pm* driver on the GPU, through the command API an application uses.

- The reference's own command-API scenario (tests/api/command_api_tests.cpp:
  338-532): a static and a dynamic cube, a torque input, a step-statistics
  query, states copied to a mapped buffer; the same checks it makes.
- Parity: scenes stepped through pm* commands equal the CPU oracle stepped
  with the same inputs (realtime profile), tick by tick. Inputs, kinematic
  targets, state writes and joints travel through the commands.
- The API path and the core library's direct path produce identical bits.
- Synchronisation objects and error codes behave as the reference's.

Tolerance: poses and velocities within 1e-5 (the oracle and the kernels run
the same FP32 operation order without contraction, so agreement is in fact
bit-exact on these scenes; the bound leaves room for the oracle's host libm).
"""
import ctypes
import dataclasses

import numpy as np
import pytest

import oracle as O
from pmb200 import core, pm, scenes

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _err(a, b):
    return max(float(np.abs(a[k] - b[k]).max()) for k in ("x", "q", "v", "w"))


def test_reference_command_flow(gpu_available):
    scene = pm.canonical_scene(scenes.cube_pair())
    s = pm.RigidSession(scene, iterations=10)
    try:
        torque = [(1, (0, 0, 0), (0, 0, 0.5), (0, 0, 0), (0, 0, 0.25))]
        assert s.step(inputs=torque, statistics=True) == pm.SUCCESS
        st = s.states()
        assert st["x"][0][1] == -1.0
        assert st["x"][1][1] < 2.0
        assert st["w"][1][2] > 0.0
        rc, execution = s.status()
        assert rc == pm.SUCCESS and execution == pm.SUCCESS
        q = s.step_statistics()
        assert q.stepCount >= 1 and q.peakActiveBodies == 2 and q.executionResult == 0
        # The same tick on the oracle.
        o = O.OracleWorld(scene)
        o.set_inputs([1], np.array([[0, 0, 0, 0, 0, 0.5, 0, 0, 0, 0, 0, 0.25]], np.float32))
        o.step(profile=scenes.REALTIME)
        assert _err(st, o.states()) <= TOL
    finally:
        s.close()


def test_realtime_step_statistics(gpu_available):
    """PM_QUERY_REALTIME_STEP_STATISTICS brackets one step and reports its
    work ledger with the invariants the reference's realtime tests check
    (tests/api/native_realtime_runtime_tests.cpp:550-555): one time advance,
    one spatial index built and published, no host readback inside the tick;
    the total is the sum of the phases and the dispatch count is every kernel
    the tick launched (the first step also creates the world, whose set-up
    launches are not part of a tick)."""
    scene = pm.canonical_scene(scenes.pyramid(levels=5, seed=2, profile=scenes.REALTIME))
    s = pm.RigidSession(scene, iterations=8)
    try:
        assert s.step(states=False) == pm.SUCCESS
        for t in range(3):
            before = core.kernel_launches()
            assert s.step(statistics="realtime", states=False) == pm.SUCCESS
            launched = core.kernel_launches() - before
            r = s.realtime_statistics()
            assert (r.schemaVersion, r.profileVersion, r.budgetVersion, r.phaseCount) == (1, 1, 1, 7)
            assert r.tick == t + 2 and r.step.stepCount == 1 and r.step.executionResult == 0
            assert r.timeAdvances == 1
            assert r.total.spatialIndexBuilds == 1 and r.total.spatialIndexPublications == 1
            assert r.total.intraTickHostReadbacks == 0 and r.total.intraTickHostWaits == 0
            assert r.total.queueSubmissions == 1
            assert r.domainIterations[0] == r.phases[4].numericalIterations >= 8
            assert list(r.domainIterations)[1:] == [0] * 5 and r.couplingEdgeCount == 0
            for f, _ in pm.RealtimeWorkStatistics._fields_:
                assert getattr(r.total, f) == sum(getattr(p, f) for p in r.phases), f
            assert r.total.dispatches == launched
            by_phase = {name: r.phases[k] for k, name in enumerate(pm.REALTIME_PHASES)}
            for name in ("predict", "index", "candidates", "domain", "commit"):
                assert by_phase[name].dispatches > 0 and by_phase[name].workgroups > 0, name
                assert by_phase[name].bytesMoved > 0, name
            assert by_phase["coupling"].dispatches == 0
            assert by_phase["domain"].barriers > 0
        # A realtime query brackets exactly one step: a second step inside
        # the open query, or an end with no step, is rejected at recording.
        a, cb, qp = s.api, s.cb, s.query_pools[pm.QUERY_REALTIME_STEP_STATISTICS]
        step = pm.StepInfo(1.0 / 60.0, 1, (ctypes.c_float * 3)(0, -9.81, 0), 0)
        assert a.pmBeginCommandBuffer(cb, ctypes.byref(pm.CommandBufferBeginInfo(pm.ST_BEGIN, None, 0))) == 0
        assert a.pmCmdBindPhysicsPipeline(cb, s.pipeline) == 0
        assert a.pmCmdResetQueryPool(cb, qp, 0, 1) == 0
        assert a.pmCmdBeginStatisticsQuery(cb, qp, 0) == 0
        assert a.pmCmdEndStatisticsQuery(cb, qp, 0) == pm.ERROR_INVALID_ARGUMENT
        assert a.pmCmdStepSimulation(cb, s.sim, ctypes.byref(step)) == 0
        assert a.pmCmdStepSimulation(cb, s.sim, ctypes.byref(step)) == pm.ERROR_INVALID_ARGUMENT
        assert a.pmCmdEndStatisticsQuery(cb, qp, 0) == 0
        assert a.pmEndCommandBuffer(cb) == 0
        assert s.submit() == pm.SUCCESS
        assert s.realtime_statistics().tick == 5
    finally:
        s.close()


def _run_api_vs_oracle(scene, ticks, per_tick=None):
    scene = pm.canonical_scene(scene)
    s = pm.RigidSession(scene)
    o = O.OracleWorld(scene)
    worst = 0.0
    try:
        for t in range(ticks):
            inputs, targets = per_tick(t) if per_tick else (None, None)
            if inputs:
                o.set_inputs([b for b, *_ in inputs],
                             np.array([np.concatenate([f, tq, li, ai]) for _, f, tq, li, ai in inputs], np.float32))
            if targets:
                o.set_targets(list(targets), np.array(list(targets.values()), scenes.STATE_DTYPE))
            assert s.step(inputs=inputs, targets=targets) == pm.SUCCESS, t
            so = o.step(profile=scenes.REALTIME)
            assert so["status"] == 0
            e = _err(s.states(), o.states())
            worst = max(worst, e)
            assert e <= TOL, (t, e)
    finally:
        s.close()
    return worst


def test_api_pyramid_matches_oracle(gpu_available):
    worst = _run_api_vs_oracle(scenes.pyramid(levels=6, profile=scenes.REALTIME), 30)
    print("pyramid through pm* commands, worst |api - oracle| =", worst)


def test_api_small_pile_matches_oracle(gpu_available):
    scene = scenes.box_pile((4, 3, 4), seed=9, spacing=1.6, profile=scenes.REALTIME)
    worst = _run_api_vs_oracle(scene, 40)
    print("pile through pm* commands, worst =", worst)


def test_api_chains_match_oracle(gpu_available):
    scene = dataclasses.replace(scenes.chains(count=2, links=6), profile=scenes.REALTIME)
    worst = _run_api_vs_oracle(scene, 30)
    print("chains through pm* commands, worst =", worst)


def _kinematic_scene():
    b = scenes._Builder()
    ground = b.mesh(*scenes.box_mesh((6.0, 0.5, 6.0)))
    plate = b.mesh(*scenes.box_mesh((1.0, 0.1, 1.0)))
    cube = b.mesh(*scenes.box_mesh((0.25, 0.25, 0.25)))
    b.body(ground, scenes.STATIC, (0, -0.5, 0))
    b.body(plate, scenes.KINEMATIC, (0, 0.4, 0))
    b.body(cube, scenes.DYNAMIC, (0.1, 0.751, 0.0), mass=2.0, inertia=scenes.box_inertia(2.0, (0.25,) * 3))
    b.body(cube, scenes.DYNAMIC, (3.0, 0.251, 0.0), mass=1.0, inertia=scenes.box_inertia(1.0, (0.25,) * 3))
    return b.build("kinematic plate", 8, scenes.REALTIME)


def test_api_kinematic_targets_and_inputs_match_oracle(gpu_available):
    def per_tick(t):
        target = np.zeros((), scenes.STATE_DTYPE)
        target["x"] = (0.01 * (t + 1), 0.4, 0.0)
        ang = 0.005 * (t + 1)
        target["q"] = (0.0, np.sin(ang / 2), 0.0, np.cos(ang / 2))
        inputs = [(3, (4.0, 0.0, 0.0), (0.0, 0.3, 0.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))]
        if t == 5:
            inputs = [(3, (4.0, 0.0, 0.0), (0.0, 0.3, 0.0), (0.0, 2.0, 0.0), (0.1, 0.0, 0.0))]
        return inputs, {1: target}

    worst = _run_api_vs_oracle(_kinematic_scene(), 40, per_tick)
    print("kinematic plate + inputs through pm* commands, worst =", worst)


def test_api_set_states_matches_oracle(gpu_available):
    scene = pm.canonical_scene(scenes.pyramid(levels=4, profile=scenes.REALTIME))
    s = pm.RigidSession(scene)
    o = O.OracleWorld(scene)
    try:
        for t in range(20):
            if t == 8:
                new = s.states()[5:7].copy()
                new["x"][:, 1] += 0.3
                new["v"][:, 0] = 1.0
                new["q"] = (0.0, 0.0, 0.2, 1.0)  # normalised by the driver and the oracle alike
                assert s.set_states(5, new) == pm.SUCCESS
                o.write_states(5, new)
            assert s.step() == pm.SUCCESS
            o.step(profile=scenes.REALTIME)
            assert _err(s.states(), o.states()) <= TOL, t
    finally:
        s.close()


def test_api_equals_core_world_bits(gpu_available):
    scene = pm.canonical_scene(scenes.box_pile((4, 3, 4), seed=4, spacing=1.6, profile=scenes.REALTIME))
    s = pm.RigidSession(scene)
    w = core.World(scene)
    try:
        for _ in range(15):
            assert s.step() == pm.SUCCESS
            w.step(profile=scenes.REALTIME)
        assert np.array_equal(s.states().view(np.uint8), w.states().view(np.uint8))
    finally:
        s.close()
        w.close()


def test_sync_objects_and_queries(gpu_available):
    s = pm.RigidSession(pm.canonical_scene(scenes.cube_pair()))
    a, dev = s.api, s.dev
    try:
        sem = ctypes.c_void_p()
        assert a.pmCreateSemaphore(dev, ctypes.byref(pm.SemaphoreCreateInfo(pm.ST_SEMAPHORE, None, 5)),
                                   ctypes.byref(sem)) == 0
        ts = ctypes.c_void_p()
        assert a.pmCreateQueryPool(dev, ctypes.byref(pm.QueryPoolCreateInfo(pm.ST_QUERY_POOL, None,
                                                                             pm.QUERY_TIMESTAMP, 2)),
                                   ctypes.byref(ts)) == 0
        cb = s.cb
        assert a.pmBeginCommandBuffer(cb, ctypes.byref(pm.CommandBufferBeginInfo(pm.ST_BEGIN, None, 0))) == 0
        assert a.pmCmdWriteTimestamp(cb, pm.STAGE_ALL_COMMANDS, ts, 0) == 0
        assert a.pmCmdBindPhysicsPipeline(cb, s.pipeline) == 0
        step = pm.StepInfo(1.0 / 60.0, 1, (ctypes.c_float * 3)(0, -9.81, 0), 0)
        assert a.pmCmdStepSimulation(cb, s.sim, ctypes.byref(step)) == 0
        assert a.pmCmdWriteTimestamp(cb, pm.STAGE_ALL_COMMANDS, ts, 1) == 0
        assert a.pmEndCommandBuffer(cb) == 0
        sig = pm.SemaphoreSubmitInfo(sem, 9, pm.STAGE_ALL_COMMANDS)
        cbs = (ctypes.c_void_p * 1)(cb)
        si = pm.SubmitInfo(pm.ST_SUBMIT, None, 0, None, 1, ctypes.cast(cbs, ctypes.c_void_p), 1,
                           ctypes.cast(ctypes.pointer(sig), ctypes.c_void_p))
        assert a.pmQueueSubmit(s.queue, ctypes.byref(si), None) == 0
        assert a.pmWaitSemaphore(dev, sem, 9, pm.TIMEOUT_INFINITE) == 0
        v = ctypes.c_uint64()
        assert a.pmGetSemaphoreCounterValue(dev, sem, ctypes.byref(v)) == 0 and v.value == 9
        # A signal value not above the current one is rejected.
        bad = pm.SemaphoreSubmitInfo(sem, 9, pm.STAGE_ALL_COMMANDS)
        si2 = pm.SubmitInfo(pm.ST_SUBMIT, None, 0, None, 0, None, 1,
                            ctypes.cast(ctypes.pointer(bad), ctypes.c_void_p))
        assert a.pmQueueSubmit(s.queue, ctypes.byref(si2), None) == pm.ERROR_INVALID_ARGUMENT
        stamps = (ctypes.c_uint64 * 2)()
        assert a.pmGetQueryPoolResults(dev, ts, 0, 2, 16, stamps, 8, pm.QUERY_RESULT_WAIT) == 0
        assert stamps[1] >= stamps[0]
        budget = (ctypes.c_uint8 * 1024)()
        assert a.pmGetDeviceMemoryBudget(dev, budget) == 0
        a.pmDestroyQueryPool(dev, ts)
        a.pmDestroySemaphore(dev, sem)
    finally:
        s.close()


def test_error_codes(gpu_available):
    s = pm.RigidSession(pm.canonical_scene(scenes.cube_pair()))
    a, dev, cb = s.api, s.dev, s.cb
    try:
        assert a.pmBeginCommandBuffer(cb, ctypes.byref(pm.CommandBufferBeginInfo(pm.ST_BEGIN, None, 0))) == 0
        step = pm.StepInfo(1.0 / 60.0, 1, (ctypes.c_float * 3)(0, -9.81, 0), 0)
        # no pipeline bound yet
        assert a.pmCmdStepSimulation(cb, s.sim, ctypes.byref(step)) == pm.ERROR_INVALID_ARGUMENT
        assert a.pmCmdBindPhysicsPipeline(cb, s.pipeline) == 0
        slow = pm.StepInfo(1.0 / 30.0, 1, (ctypes.c_float * 3)(0, -9.81, 0), 0)
        assert a.pmCmdStepSimulation(cb, s.sim, ctypes.byref(slow)) == pm.ERROR_INVALID_ARGUMENT
        two = pm.StepInfo(1.0 / 60.0, 2, (ctypes.c_float * 3)(0, -9.81, 0), 0)
        assert a.pmCmdStepSimulation(cb, s.sim, ctypes.byref(two)) == pm.ERROR_INVALID_ARGUMENT
        events = pm.StepInfo(1.0 / 60.0, 1, (ctypes.c_float * 3)(0, -9.81, 0), 1)
        assert a.pmCmdStepSimulation(cb, s.sim, ctypes.byref(events)) == 0
        other = pm.StepInfo(1.0 / 60.0, 1, (ctypes.c_float * 3)(0, -9.81, 0), 2)
        assert a.pmCmdStepSimulation(cb, s.sim, ctypes.byref(other)) == pm.ERROR_INVALID_ARGUMENT
        assert a.pmCmdCopyContactEvents(cb, s.sim, None) == pm.ERROR_INVALID_ARGUMENT
        short = pm.BufferRange(s.event_buf, 0, 8)
        assert a.pmCmdCopyContactEvents(cb, s.sim, ctypes.byref(short)) == pm.ERROR_INVALID_ARGUMENT
        # an input on the static body fails when the submission executes
        bad = pm.RigidInput(0, (ctypes.c_float * 3)(1, 0, 0))
        assert a.pmCmdApplyRigidInputs(cb, s.sim, 1, ctypes.byref(bad)) == 0
        assert a.pmEndCommandBuffer(cb) == 0
        assert s.submit() == pm.ERROR_INVALID_ARGUMENT
        rc, execution = s.status()
        assert rc == 0 and execution == pm.ERROR_INVALID_ARGUMENT
        # other domains cannot be created on this device
        sci = pm.SimulationCreateInfo(pm.ST_SIMULATION, None, 0, 4, 0, 0, 1)
        sim = ctypes.c_void_p()
        assert a.pmCreateSimulation(dev, ctypes.byref(sci), ctypes.byref(sim)) == pm.ERROR_INVALID_ARGUMENT
        # an unknown query type
        mem = ctypes.c_void_p()
        assert a.pmCreateQueryPool(dev, ctypes.byref(pm.QueryPoolCreateInfo(pm.ST_QUERY_POOL, None, 3, 1)),
                                   ctypes.byref(mem)) == pm.ERROR_INVALID_ARGUMENT
    finally:
        s.close()


def test_contact_events_through_the_api_match_the_core_world(gpu_available):
    """pmCmdCopyContactEvents: header (events, contact capacity, steps taken)
    and one record per contact point, bodies as slots; the records carry the
    bits of the core world's events for the same ticks, and capacity bounds
    the count."""
    scene = pm.canonical_scene(scenes.pyramid(levels=5, seed=2, profile=scenes.REALTIME))
    s = pm.RigidSession(scene, contact_capacity=4096)
    w = core.World(scene, event_capacity=4096)
    try:
        for t in range(12):
            assert s.step(events=True) == 0
            st = w.step(collect_events=1)
            (count, capacity, revision), ev = s.contact_events()
            want = w.contact_events()
            assert capacity == 4096 and revision == t + 1
            assert count == len(want) == int(st["contacts"]) > 0
            assert (ev["type"] == 0).all()
            assert np.array_equal(ev["first"], want["body"]) and np.array_equal(ev["second"], want["collider"])
            for a, b in (("position", "position"), ("normal", "normal"), ("penetration", "penetration"),
                         ("normalImpulse", "normal_impulse"), ("frictionImpulse", "friction_impulse")):
                assert np.array_equal(ev[a].view(np.uint32), want[b].view(np.uint32)), (t, a)
        assert s.step(events=False, copy_events=True) == 0
        (count, _, revision), _ = s.contact_events()
        assert count == 0 and revision == 13
    finally:
        s.close()
        w.close()
    small = pm.RigidSession(scene, contact_capacity=5)
    try:
        for _ in range(3):
            assert small.step(events=True) == 0
        (count, capacity, _), ev = small.contact_events()
        assert count == 5 and capacity == 5
    finally:
        small.close()

# SPDX-License-Identifier: MIT
"""Failure detection without a GPU fault.

1. Bounded device waits that run out: a world whose grid-barrier wait is cut
   to one poll (pmb_world_set_barrier_limit) abandons the tick, latches
   PMB_STATUS_BARRIER_TIMEOUT, and returns; the same world steps normally once
   the default limit is back, and a new world on the same device still
   matches the CPU oracle bit for bit -- the context survived.
2. Host-side injection through the driver's test build
   (libpm_b200_driver_failtest.so), with the reference's hooks
   (tests/api/failure_lifecycle_tests.cpp:57-150): allocation, recording and
   submission failures are synchronous and leave nothing published or
   pending; an upload failure is deferred to the fence; a barrier wait that
   runs out is reported as PM_ERROR_DEVICE_LOST. Every failure is followed by
   a successful retry on the same objects.
"""
import ctypes as C
import os

import numpy as np
import pytest

from pmb200 import core, pm, scenes
import oracle as O

pytestmark = pytest.mark.gpu

BARRIER_TIMEOUT = 1 << 4
OUT_OF_HOST_MEMORY, OUT_OF_DEVICE_MEMORY, DEVICE_LOST = -3, -4, -8
FAILTEST = os.path.join(pm.PKG_DIR, "libpm_b200_driver_failtest.so")
HOOKS = ("PM_TEST_FAIL_ALLOCATION", "PM_TEST_FAIL_RECORDING", "PM_TEST_FAIL_SUBMISSION", "PM_TEST_FAIL_UPLOAD",
         "PM_TEST_BARRIER_SPINS")


def test_barrier_wait_runs_out_and_the_device_recovers(gpu_available):
    scene = scenes.box_pile((6, 4, 6), seed=7, spacing=1.6)
    w = core.World(scene)
    for _ in range(30):
        assert int(w.step()["status"]) == 0
    w.set_barrier_limit(1)
    st = w.step()
    assert int(st["status"]) & BARRIER_TIMEOUT, core.status_names(int(st["status"]))
    w.set_barrier_limit(0)
    for _ in range(5):
        st = w.step()
        assert int(st["status"]) == 0, core.status_names(int(st["status"]))
    assert np.isfinite(w.states()["x"]).all()
    w.close()
    # A new world on the same device: the context is intact, the tick exact.
    fresh = core.World(scene)
    cpu = O.OracleWorld(scene)
    for frame in range(8):
        assert int(fresh.step()["status"]) == 0
        cpu.step()
        assert np.array_equal(fresh.candidate_pairs(), cpu.candidate_pairs()), frame
        xg, xo = fresh.states(), cpu.states()
        err = max(float(np.abs(xg[k] - xo[k]).max()) for k in ("x", "q", "v", "w"))
        assert err <= 1e-5, (frame, err)
    fresh.close()


@pytest.fixture
def failtest_driver():
    assert os.path.exists(FAILTEST), "libpm_b200_driver_failtest.so is not built"
    pm.use_driver(FAILTEST)
    yield
    for k in HOOKS:
        os.environ.pop(k, None)
    pm.use_driver(None)


def _set(name, value="1"):
    if value is None:
        os.environ.pop(name, None)
    else:
        os.environ[name] = value


def test_driver_failure_lifecycle(gpu_available, failtest_driver):
    s = pm.RigidSession(scenes.pyramid(levels=4, profile=scenes.REALTIME))
    api = s.api
    assert s.step() == pm.SUCCESS

    # Device allocation failure publishes no handle; a retry succeeds.
    info = pm.MemoryAllocateInfo(pm.ST_MEMORY, None, 256, 1)
    mem = C.c_void_p()
    _set("PM_TEST_FAIL_ALLOCATION")
    assert api.pmAllocateMemory(s.dev, pm.ref(info), pm.ref(mem)) == OUT_OF_DEVICE_MEMORY
    assert not mem.value
    _set("PM_TEST_FAIL_ALLOCATION", None)
    assert api.pmAllocateMemory(s.dev, pm.ref(info), pm.ref(mem)) == pm.SUCCESS and mem.value
    api.pmFreeMemory(s.dev, mem)

    # Recording failure is synchronous and latched until the buffer is begun again.
    begin = pm.CommandBufferBeginInfo(pm.ST_BEGIN, None, 0)
    step = pm.StepInfo(1.0 / 60.0, 1, (C.c_float * 3)(0.0, -9.81, 0.0), 0)
    assert api.pmBeginCommandBuffer(s.cb, pm.ref(begin)) == pm.SUCCESS
    assert api.pmCmdBindPhysicsPipeline(s.cb, s.pipeline) == pm.SUCCESS
    _set("PM_TEST_FAIL_RECORDING")
    assert api.pmCmdStepSimulation(s.cb, s.sim, pm.ref(step)) == OUT_OF_HOST_MEMORY
    _set("PM_TEST_FAIL_RECORDING", None)
    assert api.pmEndCommandBuffer(s.cb) == OUT_OF_HOST_MEMORY
    # The buffer stays in the recording state with its error latched
    # (reference src/api/commands.cpp:132-140); a reset clears it.
    assert api.pmBeginCommandBuffer(s.cb, pm.ref(begin)) == pm.ERROR_INVALID_STATE
    assert api.pmResetCommandBuffer(s.cb) == pm.SUCCESS
    assert s.step() == pm.SUCCESS

    # Submission failure comes before acceptance: the fence does not become pending.
    assert api.pmBeginCommandBuffer(s.cb, pm.ref(begin)) == pm.SUCCESS
    assert api.pmCmdBindPhysicsPipeline(s.cb, s.pipeline) == pm.SUCCESS
    assert api.pmCmdStepSimulation(s.cb, s.sim, pm.ref(step)) == pm.SUCCESS
    assert api.pmEndCommandBuffer(s.cb) == pm.SUCCESS
    cbs = (C.c_void_p * 1)(s.cb)
    submit = pm.SubmitInfo(pm.ST_SUBMIT, None, 0, None, 1, C.cast(cbs, C.c_void_p), 0, None)
    assert api.pmResetFences(s.dev, 1, pm.ref(s.fence)) == pm.SUCCESS
    _set("PM_TEST_FAIL_SUBMISSION")
    assert api.pmQueueSubmit(s.queue, pm.ref(submit), s.fence) == OUT_OF_HOST_MEMORY
    _set("PM_TEST_FAIL_SUBMISSION", None)
    assert api.pmGetFenceStatus(s.dev, s.fence) == pm.NOT_READY
    assert api.pmQueueSubmit(s.queue, pm.ref(submit), s.fence) == pm.SUCCESS
    assert api.pmWaitForFences(s.dev, 1, pm.ref(s.fence), 1, pm.TIMEOUT_INFINITE) == pm.SUCCESS

    # An upload failure at execution is deferred to the fence.
    _set("PM_TEST_FAIL_UPLOAD")
    assert s.step() == OUT_OF_DEVICE_MEMORY
    _set("PM_TEST_FAIL_UPLOAD", None)
    assert s.step() == pm.SUCCESS

    # A grid-barrier wait that runs out: the tick is abandoned and reported
    # as a lost device; the next tick runs normally.
    _set("PM_TEST_BARRIER_SPINS", "1")
    assert s.step() == DEVICE_LOST
    _set("PM_TEST_BARRIER_SPINS", None)
    for _ in range(3):
        assert s.step() == pm.SUCCESS
    assert np.isfinite(s.states()["x"]).all()
    s.close()

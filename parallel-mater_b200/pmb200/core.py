# SPDX-License-Identifier: MIT
"""ctypes binding of libpmb200_core.so (include/pmb200_core.h).

There is no CPU path: constructing a ``World`` without the built library or
without a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from .scenes import STATE_DTYPE, STATS_DTYPE, Scene

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libpmb200_core.so")

ERRORS = {-1: "invalid argument", -4: "out of device memory", -5: "feature not present",
          -7: "capacity exceeded", -8: "device lost", -10: "no CUDA device"}

STATUS_BITS = {1: "candidate overflow", 2: "contact overflow", 4: "pair overflow",
               8: "invalid bounds", 16: "barrier timeout", 32: "colour overflow",
               64: "grid overflow"}


class PmbError(RuntimeError):
    pass


class WorldDesc(ctypes.Structure):
    _fields_ = [("body_count", ctypes.c_uint32), ("bodies", ctypes.c_void_p),
                ("states", ctypes.c_void_p), ("mesh_count", ctypes.c_uint32),
                ("vertex_offsets", ctypes.c_void_p), ("vertices", ctypes.c_void_p),
                ("index_offsets", ctypes.c_void_p), ("indices", ctypes.c_void_p),
                ("joint_count", ctypes.c_uint32), ("joints", ctypes.c_void_p),
                ("candidate_capacity", ctypes.c_uint32), ("pair_capacity", ctypes.c_uint32),
                ("contact_capacity", ctypes.c_uint32), ("device", ctypes.c_int32),
                ("persistent_memory", ctypes.c_void_p), ("persistent_bytes", ctypes.c_uint64),
                ("scratch_memory", ctypes.c_void_p), ("scratch_bytes", ctypes.c_uint64),
                ("scene_count", ctypes.c_uint32), ("body_scene", ctypes.c_void_p),
                ("scene_iterations", ctypes.c_void_p), ("event_capacity", ctypes.c_uint32)]


EVENT_DTYPE = np.dtype([("body", "<u4"), ("collider", "<u4"), ("position", "<f4", 3), ("normal", "<f4", 3),
                        ("penetration", "<f4"), ("normal_impulse", "<f4"), ("friction_impulse", "<f4", 3)])
assert EVENT_DTYPE.itemsize == 52


class WorldCapacity(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint32) for k in ("body_count", "joint_count", "mesh_count", "mesh_vertex_count",
                                                "mesh_triangle_count", "candidate_capacity", "pair_capacity",
                                                "contact_capacity", "event_capacity")]


_lib = None


def build():
    subprocess.run(["make", "-s", "-j8", "-C", PKG_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PmbError(f"{LIB_PATH} is not built (run `make -C {PKG_DIR}`)")
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int
        sig = {
            "pmb_world_create": [vp, vp], "pmb_world_destroy": [vp],
            "pmb_world_set_stream": [vp, vp], "pmb_world_step": [vp, vp, vp],
            "pmb_world_capture": [vp, vp, u32], "pmb_world_replay": [vp],
            "pmb_world_profile_step": [vp, vp, vp, u32],
            "pmb_world_solve_timer": [vp, i32, vp, vp], "pmb_kernel_launches": [vp],
            "pmb_prepare_mesh": [vp, u32, vp, u32, vp, vp, vp, vp],
            "pmb_mesh_bvh_build": [vp, u32, vp, u32, vp, vp, u32, vp, vp],
            "pmb_world_get_states": [vp, vp], "pmb_world_set_states": [vp, vp],
            "pmb_world_last_stats": [vp, vp], "pmb_world_apply_impulse": [vp, u32, vp, vp],
            "pmb_world_candidate_pairs": [vp, vp, u32, vp],
            "pmb_world_manifolds": [vp, vp, vp, vp, u32, vp],
            "pmb_world_graph": [vp, vp, vp], "pmb_world_residual_trace": [vp, vp, u32, vp],
            "pmb_world_snapshot": [vp], "pmb_world_restore": [vp],
            "pmb_math_eval": [u32, u32, vp, vp],
            "pmb_world_memory_requirements": [vp, vp, vp],
            "pmb_world_set_inputs": [vp, u32, vp, vp], "pmb_world_set_targets": [vp, u32, vp, vp],
            "pmb_world_write_states": [vp, u32, u32, vp],
            "pmb_world_copy_states_to_device": [vp, u32, u32, vp], "pmb_world_stream": [vp, vp],
            "pmb_world_joints": [vp, vp, vp, vp, u32],
            "pmb_world_scene_stats": [vp, vp, vp, vp, vp, u32],
            "pmb_world_set_launch_plan": [vp, u32, u32], "pmb_world_autotune": [vp, vp, u32, vp, vp, vp, u32],
            "pmb_world_set_barrier_limit": [vp, u32],
            "pmb_world_contact_duals": [vp, u32, vp, vp, u32, vp],
            "pmb_world_mlp_attach": [vp, vp, u32], "pmb_world_mlp_train": [vp, i32, ctypes.c_float, u32],
            "pmb_world_mlp_params": [vp, vp, vp, vp, vp], "pmb_world_mlp_apply_mode": [vp, u32], "pmb_world_mlp_rows": [vp, vp, vp, u32, vp],
            "pmb_mlp_forward_backward": [i32, u32, vp, vp, vp, vp, vp, vp, vp],
            "pmb_world_set_warm_table": [vp, u32, vp, vp, u32],
            "pmb_world_contact_events": [vp, vp, u32, vp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = None if name == "pmb_world_destroy" else i32
        _lib = L
    return _lib


def memory_requirements(body_count, joint_count=0, mesh_count=1, mesh_vertex_count=0, mesh_triangle_count=0,
                        candidate_capacity=0, pair_capacity=0, contact_capacity=0):
    """(persistent, scratch) bytes of caller-owned memory for a world within these bounds."""
    c = WorldCapacity(body_count, joint_count, mesh_count, mesh_vertex_count, mesh_triangle_count,
                      candidate_capacity, pair_capacity, contact_capacity)
    p, s = ctypes.c_uint64(), ctypes.c_uint64()
    _check(lib().pmb_world_memory_requirements(ctypes.byref(c), ctypes.byref(p), ctypes.byref(s)),
           "pmb_world_memory_requirements")
    return p.value, s.value


MLP_PARAMS = 7424


def mlp_forward_backward(features, targets, weights, params, device=0):
    """GPU forward + backward of the warm-start MLP over given rows:
    (outputs [n,2], gradient [7424], loss)."""
    f = np.ascontiguousarray(features, np.float32).reshape(-1, 8)
    n = len(f)
    y = np.ascontiguousarray(targets, np.float32).reshape(n, 2)
    w = np.ascontiguousarray(weights, np.float32).reshape(n)
    p = np.ascontiguousarray(params, np.float32).reshape(MLP_PARAMS)
    out = np.zeros((n, 2), np.float32)
    g = np.zeros(MLP_PARAMS, np.float32)
    loss = ctypes.c_float()
    _check(lib().pmb_mlp_forward_backward(device, n, _p(f), _p(y), _p(w), _p(p), _p(out), _p(g), ctypes.byref(loss)),
           "pmb_mlp_forward_backward")
    return out, g, loss.value


def _check(rc, what):
    if rc != 0:
        raise PmbError(f"{what}: {ERRORS.get(rc, rc)}")


def _p(a):
    return a.ctypes.data if a is not None and a.size else None


class World:
    """A rigid world resident on one GPU, stepped by the CUDA kernels."""

    def __init__(self, scene: Scene, device=0, candidate_capacity=0, pair_capacity=0,
                 contact_capacity=0, event_capacity=0):
        self.scene = scene
        L = lib()
        s = scene
        self._keep = [np.ascontiguousarray(x) for x in (s.bodies, s.states, s.mesh_vertex_offsets,
                                                         s.vertices, s.mesh_index_offsets, s.indices,
                                                         s.joints)]
        b, st, vo, v, io, i, j = self._keep
        d = WorldDesc(len(b), _p(b), _p(st), len(vo) - 1, _p(vo), _p(v), _p(io), _p(i), len(j), _p(j),
                      candidate_capacity, pair_capacity, contact_capacity, device)
        d.event_capacity = event_capacity
        if s.body_scene is not None:
            bs = np.ascontiguousarray(s.body_scene, np.uint32)
            si = np.ascontiguousarray(s.scene_iterations if s.scene_iterations is not None
                                      else np.zeros(int(bs.max()) + 1), np.uint32)
            self._keep += [bs, si]
            d.scene_count = len(si)
            d.body_scene = _p(bs)
            d.scene_iterations = _p(si)
        h = ctypes.c_void_p()
        _check(L.pmb_world_create(ctypes.byref(d), ctypes.byref(h)), "pmb_world_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pmb_world_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def step(self, desc=None, stats=True, **kw):
        d = np.ascontiguousarray(self.scene.step_desc(**kw) if desc is None else desc)
        out = np.zeros((), STATS_DTYPE) if stats else None
        _check(lib().pmb_world_step(self.h, d.ctypes.data, out.ctypes.data if stats else None),
               "pmb_world_step")
        return out

    def capture(self, steps=2, desc=None, **kw):
        d = np.ascontiguousarray(self.scene.step_desc(**kw) if desc is None else desc)
        _check(lib().pmb_world_capture(self.h, d.ctypes.data, steps), "pmb_world_capture")

    def profile_step(self, desc=None, **kw):
        d = np.ascontiguousarray(self.scene.step_desc(**kw) if desc is None else desc)
        buf = ctypes.create_string_buffer(8192)
        _check(lib().pmb_world_profile_step(self.h, d.ctypes.data, buf, 8192), "pmb_world_profile_step")
        return buf.value.decode()

    def solve_timer(self, enable=True):
        """(summed solve-kernel ms, launches) since the last call; sets enable."""
        ms = ctypes.c_float()
        n = ctypes.c_uint32()
        _check(lib().pmb_world_solve_timer(self.h, 1 if enable else 0, ctypes.byref(ms), ctypes.byref(n)),
               "pmb_world_solve_timer")
        return ms.value, n.value

    def replay(self):
        _check(lib().pmb_world_replay(self.h), "pmb_world_replay")

    def set_stream(self, stream_ptr):
        _check(lib().pmb_world_set_stream(self.h, stream_ptr), "pmb_world_set_stream")

    def stats(self):
        out = np.zeros((), STATS_DTYPE)
        _check(lib().pmb_world_last_stats(self.h, out.ctypes.data), "pmb_world_last_stats")
        return out

    def states(self, out=None):
        """All body states (STATE_DTYPE); `out`: a contiguous array of n
        records to fill instead of a new one (pinned memory makes the copy a
        DMA transfer)."""
        if out is None:
            out = np.empty(self.scene.n, STATE_DTYPE)
        assert out.dtype == STATE_DTYPE and out.size == self.scene.n and out.flags.c_contiguous
        _check(lib().pmb_world_get_states(self.h, out.ctypes.data), "pmb_world_get_states")
        return out

    def set_states(self, states):
        s = np.ascontiguousarray(states, STATE_DTYPE)
        _check(lib().pmb_world_set_states(self.h, s.ctypes.data), "pmb_world_set_states")

    def apply_impulse(self, body, linear, angular=(0, 0, 0)):
        lin = np.asarray(linear, np.float32)
        ang = np.asarray(angular, np.float32)
        _check(lib().pmb_world_apply_impulse(self.h, body, lin.ctypes.data, ang.ctypes.data),
               "pmb_world_apply_impulse")

    def candidate_pairs(self):
        n = ctypes.c_uint32()
        _check(lib().pmb_world_candidate_pairs(self.h, None, 0, ctypes.byref(n)), "candidate_pairs")
        out = np.zeros(max(n.value, 1), np.uint64)
        _check(lib().pmb_world_candidate_pairs(self.h, out.ctypes.data, n.value, ctypes.byref(n)),
               "candidate_pairs")
        return out[:n.value]

    def manifolds(self):
        n = ctypes.c_uint32()
        _check(lib().pmb_world_manifolds(self.h, None, None, None, 0, ctypes.byref(n)), "manifolds")
        k = max(n.value, 1)
        codes = np.zeros(k, np.uint64)
        counts = np.zeros(k, np.uint32)
        contacts = np.zeros((k, 8, 22), np.float32)
        _check(lib().pmb_world_manifolds(self.h, codes.ctypes.data, counts.ctypes.data,
                                         contacts.ctypes.data, k, ctypes.byref(n)), "manifolds")
        return codes[:n.value], counts[:n.value], contacts[:n.value]

    def graph(self):
        colors = np.zeros(self.scene.n, np.uint32)
        parents = np.zeros(self.scene.n, np.uint32)
        _check(lib().pmb_world_graph(self.h, colors.ctypes.data, parents.ctypes.data), "graph")
        return colors, parents

    def residual_trace(self):
        out = np.zeros(256, np.float32)
        n = ctypes.c_uint32()
        _check(lib().pmb_world_residual_trace(self.h, out.ctypes.data, 256, ctypes.byref(n)),
               "residual_trace")
        return out[:n.value]

    def contact_events(self):
        """The last tick's contact events (EVENT_DTYPE records), or an empty
        array when that tick did not collect them."""
        n = ctypes.c_uint32()
        _check(lib().pmb_world_contact_events(self.h, None, 0, ctypes.byref(n)), "pmb_world_contact_events")
        out = np.zeros(n.value, EVENT_DTYPE)
        if n.value:
            _check(lib().pmb_world_contact_events(self.h, out.ctypes.data, n.value, ctypes.byref(n)),
                   "pmb_world_contact_events")
        return out

    def snapshot(self):
        _check(lib().pmb_world_snapshot(self.h), "snapshot")

    def restore(self):
        _check(lib().pmb_world_restore(self.h), "restore")

    def joints(self):
        j = len(self.scene.joints)
        flags = np.zeros(max(j, 1), np.uint32)
        applied = np.zeros(max(j, 1), np.float32)
        counts = np.zeros(max(j, 1), np.uint32)
        _check(lib().pmb_world_joints(self.h, flags.ctypes.data, applied.ctypes.data, counts.ctypes.data,
                                      max(j, 1)), "pmb_world_joints")
        return flags[:j], applied[:j], counts[:j]

    def set_launch_plan(self, solve_variant=0, solve_policy=0):
        _check(lib().pmb_world_set_launch_plan(self.h, solve_variant, solve_policy), "pmb_world_set_launch_plan")

    def set_barrier_limit(self, spins=0):
        """Polls a block makes at a grid barrier before the tick is abandoned
        with PMB_STATUS_BARRIER_TIMEOUT (0: the default)."""
        _check(lib().pmb_world_set_barrier_limit(self.h, spins), "set_barrier_limit")

    def autotune(self, desc=None, ticks=3, **kw):
        """Time every launch plan over `ticks` ticks (state restored), keep
        the fastest; returns (solve_variant, solve_policy, report)."""
        d = np.ascontiguousarray(self.scene.step_desc(**kw) if desc is None else desc)
        v, p = ctypes.c_uint32(), ctypes.c_uint32()
        buf = ctypes.create_string_buffer(4096)
        _check(lib().pmb_world_autotune(self.h, d.ctypes.data, ticks, ctypes.byref(v), ctypes.byref(p), buf, 4096),
               "pmb_world_autotune")
        return v.value, p.value, buf.value.decode()

    def scene_stats(self):
        """Per scene of a batched world: (residual RMS, residual max, sweeps, contact points)."""
        ns = len(self.scene.scene_iterations)
        rms, mx = np.zeros(ns, np.float32), np.zeros(ns, np.float32)
        its, cts = np.zeros(ns, np.uint32), np.zeros(ns, np.uint32)
        _check(lib().pmb_world_scene_stats(self.h, _p(rms), _p(mx), _p(its), _p(cts), ns), "pmb_world_scene_stats")
        return rms, mx, its, cts

    def mlp_attach(self, params=None, seed=1):
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        _check(lib().pmb_world_mlp_attach(self.h, _p(p), seed), "pmb_world_mlp_attach")

    def mlp_apply_mode(self, mode):
        _check(lib().pmb_world_mlp_apply_mode(self.h, mode), "pmb_world_mlp_apply_mode")

    def mlp_train(self, enable=True, lr=1e-3, steps_per_tick=1):
        _check(lib().pmb_world_mlp_train(self.h, 1 if enable else 0, lr, steps_per_tick), "pmb_world_mlp_train")

    def mlp_params(self):
        """(master parameters, last training loss, plain warm start's loss on
        the same rows, gate)."""
        p = np.zeros(MLP_PARAMS, np.float32)
        loss, plain, gate = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        _check(lib().pmb_world_mlp_params(self.h, p.ctypes.data, ctypes.byref(loss), ctypes.byref(plain),
                                          ctypes.byref(gate)), "pmb_world_mlp_params")
        return p, loss.value, plain.value, gate.value

    def mlp_rows(self):
        """(features [n, 8], meta [n, 4]) of the last tick's contacts."""
        n = ctypes.c_uint32()
        _check(lib().pmb_world_mlp_rows(self.h, None, None, 0, ctypes.byref(n)), "mlp_rows")
        f = np.zeros((max(n.value, 1), 8), np.float32)
        m = np.zeros((max(n.value, 1), 4), np.float32)
        _check(lib().pmb_world_mlp_rows(self.h, f.ctypes.data, m.ctypes.data, n.value, ctypes.byref(n)), "mlp_rows")
        return f[:n.value], m[:n.value]

    def contact_duals(self, rows=1):
        """(lambda, penalty) of the first `rows` rows of every contact point
        after the last tick, shape [contacts, rows]."""
        n = ctypes.c_uint32()
        _check(lib().pmb_world_contact_duals(self.h, rows, None, None, 0, ctypes.byref(n)), "contact_duals")
        lam = np.zeros((max(n.value, 1), rows), np.float32)
        pen = np.zeros((max(n.value, 1), rows), np.float32)
        _check(lib().pmb_world_contact_duals(self.h, rows, lam.ctypes.data, pen.ctypes.data, n.value,
                                             ctypes.byref(n)), "contact_duals")
        return lam[:n.value], pen[:n.value]

    def set_warm_table(self, lam, pen):
        lam = np.ascontiguousarray(lam, np.float32)
        pen = np.ascontiguousarray(pen, np.float32)
        rows = 1 if lam.ndim == 1 else lam.shape[1]
        _check(lib().pmb_world_set_warm_table(self.h, rows, lam.ctypes.data, pen.ctypes.data, len(lam)),
               "set_warm_table")

    def set_inputs(self, bodies, values):
        """values: [k, 12] float32 (force, torque, linear, angular impulse)."""
        b = np.ascontiguousarray(bodies, np.uint32)
        v = np.ascontiguousarray(values, np.float32).reshape(len(b), 12)
        _check(lib().pmb_world_set_inputs(self.h, len(b), _p(b), _p(v)), "pmb_world_set_inputs")

    def set_targets(self, bodies, targets):
        b = np.ascontiguousarray(bodies, np.uint32)
        t = np.ascontiguousarray(targets, STATE_DTYPE)
        _check(lib().pmb_world_set_targets(self.h, len(b), _p(b), _p(t)), "pmb_world_set_targets")

    def write_states(self, first, states):
        t = np.ascontiguousarray(states, STATE_DTYPE)
        _check(lib().pmb_world_write_states(self.h, first, len(t), _p(t)), "pmb_world_write_states")



def prepare_mesh(vertices, indices):
    """Host mesh preparation of the library: (convex, indices, planes[T,4], bounds[10])."""
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
    i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    out_i = np.zeros_like(i)
    planes = np.zeros((len(i) // 3, 4), np.float32)
    bounds = np.zeros(10, np.float32)
    convex = ctypes.c_int()
    _check(lib().pmb_prepare_mesh(v.ctypes.data, len(v), i.ctypes.data, len(i), out_i.ctypes.data,
                                  planes.ctypes.data, bounds.ctypes.data, ctypes.byref(convex)),
           "pmb_prepare_mesh")
    return bool(convex.value), out_i, planes, bounds


def kernel_launches() -> int:
    """CUDA kernels enqueued by the library so far in this process."""
    n = ctypes.c_ulonglong()
    _check(lib().pmb_kernel_launches(ctypes.byref(n)), "pmb_kernel_launches")
    return n.value


_MATH_WIDTH = {0: (27, 7), 1: (7, 5), 2: (4, 6), 3: (42, 7), 4: (3, 2)}


def math_eval(kind: int, inputs: np.ndarray) -> np.ndarray:
    """Run the device AVBD math (0 block solve, 1 dual, 2 contact, 3 row, 4 trig)."""
    win, wout = _MATH_WIDTH[kind]
    x = np.ascontiguousarray(inputs, np.float32).reshape(-1, win)
    out = np.zeros((len(x), wout), np.float32)
    _check(lib().pmb_math_eval(kind, len(x), x.ctypes.data, out.ctypes.data), "pmb_math_eval")
    return out


def status_names(status: int):
    return [v for k, v in STATUS_BITS.items() if status & k]

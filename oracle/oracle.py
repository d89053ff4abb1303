# SPDX-License-Identifier: MIT
"""ORACLE — test infrastructure only.

ctypes binding of ``liboracle_avbd.so``, the serial CPU restatement of the
reference's rigid AVBD tick (see avbd_step.hpp for the file:line map). Only
tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline leg use it,
always as the checker, never as the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_avbd.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, f32, ip = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_float, ctypes.c_int
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [u32, vp, vp, u32, vp, vp, vp, vp, u32, vp, ip]
        L.oracle_clone.restype = vp
        L.oracle_clone.argtypes = [vp]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_step.argtypes = [vp, vp, vp]
        L.oracle_get_states.argtypes = [vp, vp]
        L.oracle_set_states.argtypes = [vp, vp]
        L.oracle_apply_impulse.argtypes = [vp, u32, vp, vp]
        L.oracle_set_inputs.argtypes = [vp, u32, vp, vp]
        L.oracle_set_targets.argtypes = [vp, u32, vp, vp]
        L.oracle_write_states.argtypes = [vp, u32, u32, vp]
        L.oracle_candidate_pairs.restype = u32
        L.oracle_candidate_pairs.argtypes = [vp, vp, u32]
        L.oracle_manifolds.restype = u32
        L.oracle_manifolds.argtypes = [vp, vp, vp, vp, u32]
        L.oracle_graph.argtypes = [vp, vp, vp]
        L.oracle_contact_events.restype = u32
        L.oracle_contact_events.argtypes = [vp, vp, u32]
        L.oracle_residual_trace.restype = u32
        L.oracle_residual_trace.argtypes = [vp, vp, u32]
        L.oracle_aabbs.argtypes = [vp, vp, vp]
        L.oracle_joints.argtypes = [vp, vp, vp, vp]
        L.oracle_prepare_mesh.restype = ip
        L.oracle_prepare_mesh.argtypes = [vp, u32, vp, u32, vp, vp, vp]
        L.oracle_block_solve.restype = ip
        L.oracle_block_solve.argtypes = [vp, vp, vp]
        L.oracle_warm_start.argtypes = [f32, f32, f32, vp]
        L.oracle_update_dual.argtypes = [f32, f32, f32, f32, f32, f32, f32, vp]
        L.oracle_project_contact.argtypes = [vp, f32, vp]
        L.oracle_row_eval.argtypes = [vp, vp]
        L.oracle_trig_eval.restype = None
        L.oracle_trig_eval.argtypes = [vp, vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data if a is not None and a.size else None


class OracleWorld:
    """One world stepped by the CPU restatement (FP32, or FP64 replay)."""

    def __init__(self, scene, fp64=False, _handle=None):
        self.scene = scene
        L = lib()
        if _handle is not None:
            self.h = _handle
            return
        s = scene
        self._keep = [np.ascontiguousarray(x) for x in (s.bodies, s.states, s.mesh_vertex_offsets,
                                                         s.vertices, s.mesh_index_offsets, s.indices,
                                                         s.joints)]
        b, st, vo, v, io, i, j = self._keep
        self.h = L.oracle_create(len(b), _p(b), _p(st), len(vo) - 1, _p(vo), _p(v), _p(io), _p(i),
                                 len(j), _p(j), 1 if fp64 else 0)
        if not self.h:
            raise MemoryError("oracle_create failed")

    def clone(self):
        return OracleWorld(self.scene, _handle=lib().oracle_clone(self.h))

    def __del__(self):
        h = getattr(self, "h", None)
        if h and _lib is not None:
            _lib.oracle_destroy(h)
            self.h = None

    def step(self, desc=None, **kw):
        from pmb200.scenes import STATS_DTYPE
        d = self.scene.step_desc(**kw) if desc is None else desc
        d = np.ascontiguousarray(d)
        stats = np.zeros((), STATS_DTYPE)
        lib().oracle_step(self.h, d.ctypes.data, stats.ctypes.data)
        return stats

    def states(self):
        from pmb200.scenes import STATE_DTYPE
        out = np.zeros(self.scene.n, STATE_DTYPE)
        lib().oracle_get_states(self.h, out.ctypes.data)
        return out

    def set_states(self, states):
        states = np.ascontiguousarray(states)
        lib().oracle_set_states(self.h, states.ctypes.data)

    def apply_impulse(self, body, linear, angular=(0, 0, 0)):
        lin = np.asarray(linear, np.float32)
        ang = np.asarray(angular, np.float32)
        lib().oracle_apply_impulse(self.h, body, lin.ctypes.data, ang.ctypes.data)

    def set_inputs(self, bodies, values):
        b = np.ascontiguousarray(bodies, np.uint32)
        v = np.ascontiguousarray(values, np.float32).reshape(len(b), 12)
        lib().oracle_set_inputs(self.h, len(b), b.ctypes.data, v.ctypes.data)

    def set_targets(self, bodies, targets):
        b = np.ascontiguousarray(bodies, np.uint32)
        t = np.ascontiguousarray(targets)
        lib().oracle_set_targets(self.h, len(b), b.ctypes.data, t.ctypes.data)

    def write_states(self, first, states):
        t = np.ascontiguousarray(states)
        lib().oracle_write_states(self.h, first, len(t), t.ctypes.data)

    def candidate_pairs(self):
        n = lib().oracle_candidate_pairs(self.h, None, 0)
        out = np.zeros(max(n, 1), np.uint64)
        lib().oracle_candidate_pairs(self.h, out.ctypes.data, n)
        return out[:n]

    def manifolds(self):
        """codes[P], counts[P], contacts[P, 8, 22] (see oracle_capi.cpp)."""
        n = lib().oracle_manifolds(self.h, None, None, None, 0)
        codes = np.zeros(max(n, 1), np.uint64)
        counts = np.zeros(max(n, 1), np.uint32)
        contacts = np.zeros((max(n, 1), 8, 22), np.float32)
        lib().oracle_manifolds(self.h, codes.ctypes.data, counts.ctypes.data, contacts.ctypes.data, n)
        return codes[:n], counts[:n], contacts[:n]

    def contact_events(self, capacity=1 << 20):
        """The latest tick's contact events as the reference reports them
        (records of pmb200.core.EVENT_DTYPE)."""
        from pmb200.core import EVENT_DTYPE
        out = np.zeros(capacity, EVENT_DTYPE)
        n = lib().oracle_contact_events(self.h, out.ctypes.data, capacity)
        return out[:n]

    def graph(self):
        colors = np.zeros(self.scene.n, np.uint32)
        parents = np.zeros(self.scene.n, np.uint32)
        lib().oracle_graph(self.h, colors.ctypes.data, parents.ctypes.data)
        return colors, parents

    def residual_trace(self):
        out = np.zeros(4096, np.float32)
        n = lib().oracle_residual_trace(self.h, out.ctypes.data, 4096)
        return out[:n]

    def aabbs(self):
        lo = np.zeros((self.scene.n, 3), np.float32)
        hi = np.zeros((self.scene.n, 3), np.float32)
        lib().oracle_aabbs(self.h, lo.ctypes.data, hi.ctypes.data)
        return lo, hi

    def joints(self):
        j = len(self.scene.joints)
        flags = np.zeros(max(j, 1), np.uint32)
        applied = np.zeros(max(j, 1), np.float32)
        counts = np.zeros(max(j, 1), np.uint32)
        lib().oracle_joints(self.h, flags.ctypes.data, applied.ctypes.data, counts.ctypes.data)
        return flags[:j], applied[:j], counts[:j]


def prepare_mesh(vertices, indices):
    v = np.ascontiguousarray(vertices, np.float32)
    i = np.ascontiguousarray(indices, np.uint32)
    out_i = np.zeros_like(i)
    planes = np.zeros((len(i) // 3, 4), np.float32)
    bounds = np.zeros(10, np.float32)
    convex = lib().oracle_prepare_mesh(v.ctypes.data, len(v), i.ctypes.data, len(i), out_i.ctypes.data,
                                       planes.ctypes.data, bounds.ctypes.data)
    return bool(convex), out_i, planes, bounds


def block_solve(h21, g6):
    h = np.ascontiguousarray(h21, np.float32)
    g = np.ascontiguousarray(g6, np.float32)
    out = np.zeros(6, np.float32)
    ok = lib().oracle_block_solve(h.ctypes.data, g.ctypes.data, out.ctypes.data)
    return bool(ok), out


def warm_start(lam, pen, stiffness):
    out = np.zeros(2, np.float32)
    lib().oracle_warm_start(lam, pen, stiffness, out.ctypes.data)
    return out


def update_dual(lam, pen, err, beta, lo, hi, stiffness):
    out = np.zeros(3, np.float32)
    lib().oracle_update_dual(lam, pen, err, beta, lo, hi, stiffness, out.ctypes.data)
    return out


def project_contact(trial3, friction):
    t = np.ascontiguousarray(trial3, np.float32)
    out = np.zeros(6, np.float32)
    lib().oracle_project_contact(t.ctypes.data, friction, out.ctypes.data)
    return out


def row_eval(values42):
    v = np.ascontiguousarray(values42, np.float32)
    out = np.zeros(7, np.float32)
    lib().oracle_row_eval(v.ctypes.data, out.ctypes.data)
    return out


def trig_eval(values3):
    """(atan2(y, x), t cos(t) / sin(t)) of one (y, x, t) record, as the
    oracle's FP32 tick evaluates them."""
    v = np.ascontiguousarray(values3, np.float32)
    out = np.zeros(2, np.float32)
    lib().oracle_trig_eval(v.ctypes.data, out.ctypes.data)
    return out

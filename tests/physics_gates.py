# SPDX-License-Identifier: MIT
"""Physical quality measures of a rigid trajectory, computed on the host from
the states a world returns, for the long-run gates the reference applies to
its realtime rigid stack (tests/solver/rigid_realtime_cuda_tests.cu:217-371):
largest penetration, settled drift, rotation drift, energy growth and
tunnelling events.

Penetration is geometric: the post-step overlap depth of two boxes, i.e. the
smallest overlap of their projections over the 15 separating axes of an
oriented-box pair (positive: the boxes interpenetrate by that much), for the
pairs the tick reports in contact. Capsule links are measured as the
segment-to-segment distance against the sum of their radii.
"""
from __future__ import annotations

import numpy as np

from pmb200 import scenes


def quat_matrix(q):
    """Rotation matrices (..., 3, 3) of unit quaternions (x, y, z, w)."""
    q = np.asarray(q, np.float64)
    x, y, z, w = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], -2)


def mesh_half_extents(scene) -> np.ndarray:
    """Per body: half extents of its mesh's local bounds (a box mesh's halves)."""
    out = np.zeros((scene.n, 3))
    for i, m in enumerate(scene.bodies["mesh"]):
        v = scene.vertices[scene.mesh_vertex_offsets[m]:scene.mesh_vertex_offsets[m + 1]]
        out[i] = np.abs(v).max(axis=0)
    return out


def is_box(scene) -> np.ndarray:
    """Per body: its mesh has 8 vertices (a box)."""
    counts = np.diff(scene.mesh_vertex_offsets)
    return counts[scene.bodies["mesh"]] == 8


def box_overlap(xa, qa, ha, xb, qb, hb):
    """Overlap depth of oriented boxes a and b (arrays over pairs): the
    smallest projection overlap over the 15 separating axes; > 0 means the
    boxes interpenetrate by that depth, <= 0 that an axis separates them."""
    Ra, Rb = quat_matrix(qa), quat_matrix(qb)           # columns: box axes in world
    A = np.swapaxes(Ra, -1, -2)                         # rows: a's axes
    B = np.swapaxes(Rb, -1, -2)
    axes = [A[:, k] for k in range(3)] + [B[:, k] for k in range(3)]
    for i in range(3):
        for j in range(3):
            axes.append(np.cross(A[:, i], B[:, j]))
    t = np.asarray(xb, np.float64) - np.asarray(xa, np.float64)
    depth = np.full(len(t), np.inf)
    for L in axes:
        n = np.linalg.norm(L, axis=1)
        ok = n > 1e-6
        Ln = np.where(ok[:, None], L / np.where(ok, n, 1.0)[:, None], 0.0)
        ra = np.sum(ha * np.abs(np.einsum("pkj,pj->pk", A, Ln)), axis=1)
        rb = np.sum(hb * np.abs(np.einsum("pkj,pj->pk", B, Ln)), axis=1)
        overlap = ra + rb - np.abs(np.einsum("pj,pj->p", t, Ln))
        depth = np.where(ok, np.minimum(depth, overlap), depth)
    return depth


def segment_distance(p0, p1, q0, q1):
    """Closest distance between segments p0-p1 and q0-q1 (arrays over pairs)."""
    d1, d2, r = p1 - p0, q1 - q0, p0 - q0
    a = np.einsum("pj,pj->p", d1, d1)
    e = np.einsum("pj,pj->p", d2, d2)
    f = np.einsum("pj,pj->p", d2, r)
    c = np.einsum("pj,pj->p", d1, r)
    b = np.einsum("pj,pj->p", d1, d2)
    den = a * e - b * b
    s = np.where(den > 1e-12, np.clip((b * f - c * e) / np.where(den > 1e-12, den, 1.0), 0, 1), 0.0)
    t = np.where(e > 1e-12, (b * s + f) / np.where(e > 1e-12, e, 1.0), 0.0)
    s = np.where(t < 0, np.clip(-c / np.where(a > 1e-12, a, 1.0), 0, 1), np.where(t > 1, np.clip((b - c) / np.where(a > 1e-12, a, 1.0), 0, 1), s))
    t = np.clip(t, 0, 1)
    return np.linalg.norm((p0 + d1 * s[:, None]) - (q0 + d2 * t[:, None]), axis=1)


def pair_penetration(scene, states, pairs, capsule=None):
    """Largest post-step penetration over the pairs (a, b) of box bodies, and
    of capsule bodies when `capsule` = (radius, half_length along local y)."""
    if len(pairs) == 0:
        return 0.0
    pairs = np.asarray(pairs, np.int64)
    a, b = pairs[:, 0], pairs[:, 1]
    x = states["x"].astype(np.float64)
    q = states["q"].astype(np.float64)
    half = mesh_half_extents(scene)
    box = is_box(scene)
    worst = 0.0
    both = box[a] & box[b]
    if both.any():
        d = box_overlap(x[a[both]], q[a[both]], half[a[both]], x[b[both]], q[b[both]], half[b[both]])
        worst = max(worst, float(np.max(d, initial=0.0)))
    if capsule is not None:
        radius, hl = capsule
        caps = ~box
        cc = caps[a] & caps[b]
        if cc.any():
            ax = quat_matrix(q)[:, :, 1]
            ia, ib = a[cc], b[cc]
            dist = segment_distance(x[ia] - hl * ax[ia], x[ia] + hl * ax[ia], x[ib] - hl * ax[ib], x[ib] + hl * ax[ib])
            worst = max(worst, float(np.max(2 * radius - dist, initial=0.0)))
    return worst


def contact_pairs(world, n):
    """(a, b) of the last tick's non-empty manifolds."""
    codes, _, _ = world.manifolds()
    codes = codes.astype(np.int64)
    return np.stack([codes // n, codes % n], axis=1)


def energy(scene, states, gravity=9.81):
    """Total mechanical energy of the dynamic bodies: translational and
    rotational kinetic energy plus potential energy above y = 0 (J)."""
    dyn = scene.bodies["motion"] == scenes.DYNAMIC
    inv_m = scene.bodies["inv_mass"][dyn].astype(np.float64)
    m = 1.0 / inv_m
    inv_i = scene.bodies["inv_inertia"][dyn].astype(np.float64)
    v = states["v"][dyn].astype(np.float64)
    w = states["w"][dyn].astype(np.float64)
    R = quat_matrix(states["q"][dyn])
    w_local = np.einsum("pji,pj->pi", R, w)            # R^T w
    rot = 0.5 * np.sum(w_local * w_local / inv_i, axis=1)
    kin = 0.5 * m * np.sum(v * v, axis=1)
    pot = m * gravity * states["x"][dyn, 1].astype(np.float64)
    return float(np.sum(kin + rot + pot))


def rotation_angle(q):
    """Rotation angle (rad) of unit quaternions from the identity."""
    q = np.asarray(q, np.float64)
    return 2.0 * np.arctan2(np.linalg.norm(q[..., :3], axis=-1), np.abs(q[..., 3]))

# SPDX-License-Identifier: MIT
"""Physical quality measures of a rigid trajectory, computed on the host from
the states a world returns, for the long-run gates the reference applies to
its realtime rigid stack (tests/solver/rigid_realtime_cuda_tests.cu:217-371):
largest penetration, settled drift, rotation drift, energy growth and
tunnelling events.

Penetration is geometric: the post-step overlap depth of two convex meshes,
i.e. the smallest overlap of their projections over the separating axes of
the pair (the 15 axes of an oriented-box pair; face normals and edge-edge
cross products of general convex meshes such as tessellated capsules),
positive when they interpenetrate, for the pairs the tick reports in
contact.
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


def mesh_axes(scene, m):
    """Local vertices, unique face normals and unique edge directions of
    convex mesh m."""
    v = scene.vertices[scene.mesh_vertex_offsets[m]:scene.mesh_vertex_offsets[m + 1]].astype(np.float64)
    t = scene.indices[scene.mesh_index_offsets[m]:scene.mesh_index_offsets[m + 1]].reshape(-1, 3)
    n = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    e = np.concatenate([v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 1]], v[t[:, 0]] - v[t[:, 2]]])
    e /= np.linalg.norm(e, axis=1, keepdims=True)

    def unique(d):
        d = np.where((d[:, :1] < 0) | ((d[:, :1] == 0) & (d[:, 1:2] < 0)), -d, d)   # one sign per direction
        return np.unique(np.round(d, 6), axis=0)

    return v, unique(n), unique(e)


def convex_overlap(scene, states, a, b):
    """Overlap depth of the convex meshes of bodies a and b (arrays over
    pairs that share one mesh pair): the smallest projection overlap over the
    separating axes of two convex polyhedra (face normals of both, cross
    products of their edge directions); > 0 means interpenetration."""
    ma, mb = int(scene.bodies["mesh"][a[0]]), int(scene.bodies["mesh"][b[0]])
    va, na, ea = mesh_axes(scene, ma)
    vb, nb, eb = mesh_axes(scene, mb)
    Ra, Rb = quat_matrix(states["q"][a]), quat_matrix(states["q"][b])
    xa, xb = states["x"][a].astype(np.float64), states["x"][b].astype(np.float64)
    wa = np.einsum("pij,vj->pvi", Ra, va) + xa[:, None]
    wb = np.einsum("pij,vj->pvi", Rb, vb) + xb[:, None]
    Na, Nb = np.einsum("pij,kj->pki", Ra, na), np.einsum("pij,kj->pki", Rb, nb)
    Ea, Eb = np.einsum("pij,kj->pki", Ra, ea), np.einsum("pij,kj->pki", Rb, eb)
    C = np.cross(Ea[:, :, None, :], Eb[:, None, :, :]).reshape(len(a), -1, 3)
    cn = np.linalg.norm(C, axis=2, keepdims=True)
    C = np.where(cn > 1e-6, C / np.where(cn > 1e-6, cn, 1.0), 0.0)
    axes = np.concatenate([Na, Nb, C], axis=1)
    pa = np.einsum("pkj,pvj->pkv", axes, wa)
    pb = np.einsum("pkj,pvj->pkv", axes, wb)
    # translation along the axis that separates the projections (the
    # penetration depth along it; negative when already separated)
    overlap = np.minimum(pa.max(2) - pb.min(2), pb.max(2) - pa.min(2))
    valid = np.linalg.norm(axes, axis=2) > 0.5
    return np.where(valid, overlap, np.inf).min(axis=1)


def pair_penetration(scene, states, pairs):
    """Largest post-step penetration over the pairs (a, b): oriented-box
    overlap for box pairs, convex-mesh overlap for every other pair (the
    meshes the tick collides, e.g. tessellated capsules)."""
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
    other = ~both
    if other.any():
        mesh = scene.bodies["mesh"]
        key = mesh[a[other]].astype(np.int64) * (1 << 32) + mesh[b[other]]
        for k in np.unique(key):
            sel = key == k
            d = convex_overlap(scene, states, a[other][sel], b[other][sel])
            worst = max(worst, float(np.max(d, initial=0.0)))
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

# SPDX-License-Identifier: MIT
"""Mesh BVH build on the GPU (`pmb_mesh_bvh_build`).

The tree must be the one the host preparation builds at mesh upload (the
reference's builder, src/simulation/runtime_deformables.cu.inc:136-210):
median split on the longest axis of the node's triangle bounds, triangles
ordered by centroid on that axis with ties by triangle index, leaves of at
most four triangles, nodes in pre-order. `restated_bvh` restates that
builder in numpy float32 arithmetic; the CPU test pins it to the library's
host builder (the triangle order `pmb_prepare_mesh` stores), the GPU test
requires the device builder's order and every node (bounds, range,
children) to equal it, bit for bit. The meshes put vertices on a coarse
grid so that many centroids tie.
"""
import ctypes

import numpy as np
import pytest

from pmb200 import core, scenes


def restated_bvh(vertices, indices):
    """(order, nodes): nodes as [lo(3), hi(3), first, count, left, right]."""
    v = np.asarray(vertices, np.float32).reshape(-1, 3)
    tris = np.asarray(indices, np.uint32).reshape(-1, 3)
    cen = ((v[tris[:, 0]] + v[tris[:, 1]]) + v[tris[:, 2]]) * np.float32(1.0 / 3.0)
    order = list(range(len(tris)))
    nodes = []

    def build(b, e):
        pts = v[tris[order[b:e]]].reshape(-1, 3)
        lo, hi = pts.min(0), pts.max(0)
        node = len(nodes)
        nodes.append([lo, hi, 0, 0, 0, 0])
        if e - b <= 4:
            nodes[node][2], nodes[node][3] = b, e - b
            return node
        ext = hi - lo
        axis = 0 if ext[0] >= ext[1] and ext[0] >= ext[2] else (1 if ext[1] >= ext[2] else 2)
        order[b:e] = sorted(order[b:e], key=lambda t: (float(cen[t, axis]), t))
        mid = b + (e - b) // 2
        left = build(b, mid)
        right = build(mid, e)
        nodes[node][4], nodes[node][5] = left, right
        return node

    build(0, len(tris))
    return np.array(order, np.uint32), nodes


def _grid_soup(triangles, seed, cells=12):
    rng = np.random.Generator(np.random.Philox(seed))
    v = (rng.integers(0, cells, size=(3 * triangles, 3)) * 0.25 - 1.0).astype(np.float32)
    v[rng.random(len(v)) < 0.05] *= np.float32(-1.0)  # signed zeros and mirrored points
    return v, np.arange(3 * triangles, dtype=np.uint32)


MESHES = [
    ("one triangle", *_grid_soup(1, 1)),
    ("four", *_grid_soup(4, 2)),
    ("five", *_grid_soup(5, 3)),
    ("capsule 32", *scenes.capsule_mesh(0.2, 0.8, segments=32)),
    ("soup 1000", *_grid_soup(1000, 4)),
    ("soup 20000", *_grid_soup(20000, 5, cells=40)),
]


@pytest.mark.parametrize("name,vertices,indices", MESHES, ids=[m[0] for m in MESHES])
def test_restated_builder_matches_the_host_builder(name, vertices, indices):
    order, _ = restated_bvh(vertices, indices)
    _, stored, _, _ = core.prepare_mesh(vertices, indices)
    tris = np.asarray(indices, np.uint32).reshape(-1, 3)
    assert np.array_equal(stored.reshape(-1, 3), tris[order])


@pytest.mark.gpu
@pytest.mark.parametrize("name,vertices,indices", MESHES, ids=[m[0] for m in MESHES])
def test_device_builder_equals_the_host_tree(gpu_available, name, vertices, indices):
    import torch
    dev = torch.device("cuda", 0)
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1)
    i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    want_order, want_nodes = restated_bvh(vertices, indices)
    d_v = torch.from_numpy(v).to(dev)
    d_i = torch.from_numpy(i.view(np.int32)).to(dev)
    n = len(i) // 3
    d_order = torch.zeros(n, dtype=torch.int32, device=dev)
    d_nodes = torch.zeros(10 * 2 * n, dtype=torch.int32, device=dev)
    count = ctypes.c_uint32()
    stream = torch.cuda.current_stream().cuda_stream
    rc = core.lib().pmb_mesh_bvh_build(d_v.data_ptr(), len(v) // 3, d_i.data_ptr(), len(i), d_order.data_ptr(),
                                       d_nodes.data_ptr(), 2 * n, ctypes.byref(count), stream)
    assert rc == 0
    assert count.value == len(want_nodes)
    assert np.array_equal(d_order.cpu().numpy().view(np.uint32), want_order)
    got = d_nodes.cpu().numpy()[:10 * count.value].reshape(-1, 10)
    bounds = got[:, :6].copy().view(np.float32)
    links = got[:, 6:].view(np.uint32)
    for k, (lo, hi, first, cnt, left, right) in enumerate(want_nodes):
        assert np.array_equal(bounds[k, :3], lo) and np.array_equal(bounds[k, 3:], hi), k
        assert list(links[k]) == [first, cnt, left, right], k
    # A capacity below the node count is refused, with the count reported.
    rc = core.lib().pmb_mesh_bvh_build(d_v.data_ptr(), len(v) // 3, d_i.data_ptr(), len(i), d_order.data_ptr(),
                                       d_nodes.data_ptr(), count.value - 1 if count.value > 1 else 0,
                                       ctypes.byref(count), stream)
    assert rc == -7


@pytest.mark.gpu
def test_device_builder_rejects_out_of_range_indices(gpu_available):
    import torch
    dev = torch.device("cuda", 0)
    v, i = _grid_soup(8, 7)
    i = i.copy()
    i[5] = len(v)  # one past the last vertex
    d_v = torch.from_numpy(v.reshape(-1)).to(dev)
    d_i = torch.from_numpy(i.view(np.int32)).to(dev)
    d_order = torch.zeros(8, dtype=torch.int32, device=dev)
    d_nodes = torch.zeros(160, dtype=torch.int32, device=dev)
    count = ctypes.c_uint32()
    rc = core.lib().pmb_mesh_bvh_build(d_v.data_ptr(), len(v), d_i.data_ptr(), len(i), d_order.data_ptr(),
                                       d_nodes.data_ptr(), 16, ctypes.byref(count),
                                       torch.cuda.current_stream().cuda_stream)
    assert rc == -1

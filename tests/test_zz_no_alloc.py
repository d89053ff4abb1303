# SPDX-License-Identifier: MIT
"""pmb_graph_color_noalloc: the colouring entry point for callers that cannot
allocate device memory (a driver confined to application-bound memory, or a
real-time thread). Its colours for a tick's contact graph must equal the ones
the tick itself computed (pmb_world_step, read back with pmb_world_graph),
exactly, on two calls in a row. Collected last so a stop-at-first-failure
run has already run every other test."""
import ctypes

import numpy as np
import pytest

from pmb200 import core, scenes

pytestmark = pytest.mark.gpu


def _contact_graph(scene, world):
    codes, counts, _ = world.manifolds()
    n = scene.n
    a = (codes // n).astype(np.int64)
    b = (codes % n).astype(np.int64)
    src = np.concatenate([a, b])
    dst = np.concatenate([b, a])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    offsets = np.zeros(n + 1, np.uint32)
    np.add.at(offsets, src + 1, 1)
    offsets = np.cumsum(offsets).astype(np.uint32)
    dynamic = (scene.bodies["motion"] == scenes.DYNAMIC).astype(np.uint32)
    return offsets, dst.astype(np.uint32), dynamic


def test_noalloc_colouring_matches_tick(gpu_available):
    import torch
    scene = scenes.box_pile((6, 4, 6), seed=9, spacing=1.6)
    world = core.World(scene)
    for _ in range(45):
        world.step(stats=False)
    st = world.step()
    assert st["status"] == 0 and st["colors"] > 1
    tick_colors, _ = world.graph()
    offsets, neighbors, dynamic = _contact_graph(scene, world)
    dev = torch.device("cuda", 0)
    d_off = torch.from_numpy(offsets.view(np.int32)).to(dev)
    d_nbr = torch.from_numpy(neighbors.view(np.int32)).to(dev)
    d_dyn = torch.from_numpy(dynamic.view(np.int32)).to(dev)
    lib = core.lib()
    f = lib.pmb_graph_color_noalloc
    f.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]
    f.restype = ctypes.c_int
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for _ in range(2):
        d_col = torch.full((scene.n,), -7, dtype=torch.int32, device=dev)
        rc = f(d_off.data_ptr(), d_nbr.data_ptr(), d_dyn.data_ptr(), scene.n, d_col.data_ptr(), 0, stream)
        assert rc == 0
        results.append(d_col.cpu().numpy().view(np.uint32))
    assert np.array_equal(results[0], tick_colors)
    assert np.array_equal(results[1], tick_colors)
    # Sizes beyond the fixed working memory are rejected up front.
    assert f(d_off.data_ptr(), d_nbr.data_ptr(), d_dyn.data_ptr(), (1 << 20) + 1, d_col.data_ptr(), 0,
             stream) == -7

# SPDX-License-Identifier: MIT
"""Scene sharding for batched stepping on several GPUs, checked on the CPU.

Batched scenes are independent, so a multi-GPU run bin-packs them over the
ranks (no exchange inside a tick) and gathers per-scene metrics at the end.
These tests cover the packing, the subset builder and the gather, the last
with two `gloo` ranks whose per-scene numbers come from the CPU oracle.
"""
import os
import socket

import numpy as np
import pytest

from pmb200 import scenes, shard


def test_shard_scenes_is_a_balanced_partition():
    sizes, kinds = scenes.batched_plan(1024, seed=5)
    for ranks in (1, 2, 3, 8):
        parts = scenes.shard_scenes(sizes, ranks)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(1024))
        loads = [int(sizes[p].sum()) for p in parts]
        # greedy LPT: the spread is at most the largest single scene
        assert max(loads) - min(loads) <= int(sizes.max())
        assert all(p == sorted(p) for p in parts)
    assert scenes.shard_scenes([5, 1, 4], 2) == [[0], [1, 2]]


def test_subset_matches_full_batch_slices():
    count = 24
    full = scenes.batched_scenes(count, seed=5, smallest=16, largest=64)
    ids = [3, 7, 8, 20]
    sub = scenes.batched_scenes(count, seed=5, smallest=16, largest=64, subset=ids)
    starts = np.concatenate([[0], np.cumsum(np.bincount(full.body_scene, minlength=count))])
    pieces = [full.states[starts[k]:starts[k + 1]] for k in ids]
    assert np.array_equal(np.concatenate(pieces).view(np.uint8), sub.states.view(np.uint8))
    assert list(sub.scene_iterations) == [int(full.scene_iterations[k]) for k in ids]


def test_gather_by_scene_single_rank_checks_coverage():
    out = shard.gather_by_scene([2, 0, 1], np.array([[2.0], [0.0], [1.0]]), 3)
    assert out[:, 0].tolist() == [0.0, 1.0, 2.0]
    with pytest.raises(ValueError):
        shard.gather_by_scene([0, 0], np.zeros(2), 3)


COUNT, SEED, SMALL, LARGE = 6, 5, 16, 40


def _scene_metrics(ids):
    """Contact points per scene after 3 oracle ticks from the spawn."""
    import oracle as O
    sizes, kinds = scenes.batched_plan(COUNT, SEED, SMALL, LARGE)
    out = []
    for k in ids:
        p = scenes.batched_part(k, sizes[k], kinds[k], SEED)
        w = O.OracleWorld(p)
        st = None
        for _ in range(3):
            st = w.step(p.step_desc())
        out.append([float(st["contacts"]), float(p.n)])
    return np.array(out, np.float64).reshape(len(ids), 2)


def _rank_main(rank, world_size, port, result_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        sizes, _ = scenes.batched_plan(COUNT, SEED, SMALL, LARGE)
        mine = scenes.shard_scenes(sizes, world_size)[rank]
        got = shard.gather_by_scene(mine, _scene_metrics(mine), COUNT, world_size)
        if rank == 0:
            np.save(result_path, got)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gather_equals_one_process(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "gathered.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    want = _scene_metrics(range(COUNT))
    assert np.array_equal(got, want)

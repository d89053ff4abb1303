# SPDX-License-Identifier: MIT
"""Scene sharding across GPUs for batched stepping.

Independent scenes need no exchange inside a tick, so each rank steps its
own shard (``scenes.shard_scenes``) as one batched world. The only
cross-rank step is the end-of-run gather of per-scene metrics, done here on
the host through ``torch.distributed`` (``all_gather_object``; any backend).
"""
import numpy as np


def gather_by_scene(ids, values, total, world_size=1):
    """Per-scene values of every rank in global scene order.

    ``ids``: this rank's scene indices; ``values``: an array whose first axis
    runs over those scenes. Returns an array of ``total`` rows on every rank.
    Raises if a scene is missing or reported twice."""
    ids = np.asarray(ids, np.int64)
    values = np.asarray(values)
    if len(ids) != len(values):
        raise ValueError("one value row per scene id")
    parts = [(ids, values)]
    if world_size > 1:
        import torch.distributed as dist
        parts = [None] * world_size
        dist.all_gather_object(parts, (ids, values))
    out = np.zeros((total,) + values.shape[1:], values.dtype)
    seen = np.zeros(total, np.int64)
    for i, v in parts:
        out[i] = v
        np.add.at(seen, i, 1)
    if not np.all(seen == 1):
        raise ValueError("scenes missing or reported twice: %s" % np.flatnonzero(seen != 1)[:8].tolist())
    return out

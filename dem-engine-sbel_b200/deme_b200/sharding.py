"""Packed multi-scene runs over several GPUs: independent scenes shard with no exchange while they step.

* partition_scenes: scenes to ranks, balanced by sphere count (longest first to the least-loaded rank);
* gather_scene_rows: per-scene results (losses, gradients) of every rank assembled on every rank with one
  collective (an all-reduce of a zero-filled table, each scene's row written by the one rank that ran it).

Each rank packs its own scenes with workloads.batched_settling and runs them on its GPU; the only collective of a
run is the final gather of a few kilobytes.
"""
from __future__ import annotations

import numpy as np


def partition_scenes(sizes, world: int) -> list:
    """Scene indices per rank.  Scenes are taken by decreasing sphere count and given to the rank with the fewest
    spheres so far (ties to the lower rank); each rank's list is returned in ascending scene order."""
    sizes = np.asarray(sizes, np.int64)
    load = np.zeros(world, np.int64)
    parts = [[] for _ in range(world)]
    for i in np.argsort(-sizes, kind="stable"):
        r = int(np.argmin(load))
        parts[r].append(int(i))
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def gather_scene_rows(local: dict, n_scenes: int, width: int, dist=None, device="cpu") -> np.ndarray:
    """(n_scenes, width) float64 table of every rank's rows: ``local`` maps scene index -> row.  With ``dist`` (an
    initialised torch.distributed) the tables of all ranks are summed; every scene belongs to one rank."""
    table = np.zeros((n_scenes, width), np.float64)
    for i, row in local.items():
        table[i] = np.asarray(row, np.float64).reshape(width)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return table
    import torch
    t = torch.from_numpy(table).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()

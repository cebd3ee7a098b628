"""Packed multi-scene runs sharded over ranks (deme_b200.sharding), on the CPU: two gloo ranks each pack and run
their share of the scenes with the C oracle, and one all-reduce assembles the per-scene results.

* partition_scenes covers every scene once and balances the sphere counts;
* the gathered per-scene kinetic energies after a few steps equal those of a single process running every scene
  (each in a packed run of its own shard, on the same voxel grid as the scene run alone).
"""
import os
import socket

import numpy as np
import pytest

from _util import oracle, workloads
from deme_b200 import sharding
from deme_b200 import statistics as stats

torch = pytest.importorskip("torch")

N_SCENES, STEPS = 6, 5


def specs():
    sp = workloads.batch_scene_specs(N_SCENES, seed=13, n_range=(150, 600), r_range=(3e-3, 5e-3),
                                     side_range=(0.04, 0.07))
    for s in sp:
        s.update(pitch=2.05, lift=1.0)
    return sp


def shard_results(sp, shard):
    """Per-scene kinetic energy (translational and rotational) after STEPS steps of the packed run of ``shard``
    (oracle)."""
    built = workloads.batched_settling([sp[i] for i in shard])
    o = oracle(built, threads=2)
    o.step(STEPS)
    st = o.state()
    out = {}
    for local, i in enumerate(shard):
        first, n = built.info["scenes"][local]
        sub = {k: v[first:first + n] for k, v in st.items()}
        a = built.arrays
        m = np.asarray(a["mass"], np.float64)[first:first + n]
        v2 = sum(sub[k].astype(np.float64) ** 2 for k in ("vX", "vY", "vZ"))
        rot = sum(np.asarray(a[I], np.float64)[first:first + n] * sub[w].astype(np.float64) ** 2
                  for I, w in (("mmiXX", "omgX"), ("mmiYY", "omgY"), ("mmiZZ", "omgZ")))
        out[i] = [0.5 * float(np.sum(m * v2)) + 0.5 * float(np.sum(rot))]
    return out


def test_partition_is_complete_and_balanced():
    sizes = np.array([sp["n"] for sp in workloads.batch_scene_specs(512)])
    for world in (1, 2, 3, 8):
        parts = sharding.partition_scenes(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [int(sizes[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= int(sizes.max())


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sp = specs()
        shard = sharding.partition_scenes([s["n"] for s in sp], world)[rank]
        local = shard_results(sp, shard)
        table = sharding.gather_scene_rows(local, N_SCENES, 1, dist=dist)
        if rank == 0:
            np.save(out_path, table)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gather_the_single_process_results(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "table.npy")
    mp.spawn(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
    table = np.load(out)
    sp = specs()
    parts = sharding.partition_scenes([s["n"] for s in sp], 2)
    expect = np.zeros((N_SCENES, 1))
    for shard in parts:
        for i, row in shard_results(sp, shard).items():
            expect[i] = row
    np.testing.assert_array_equal(table, expect)
    assert np.all(table > 0)


def test_kinetic_energy_helper_matches_the_per_scene_sum():
    sp = specs()
    built = workloads.batched_settling(sp)
    o = oracle(built, threads=2)
    o.step(STEPS)
    st = o.state()
    per_scene = shard_results(sp, list(range(N_SCENES)))
    total = sum(v[0] for v in per_scene.values())
    assert abs(stats.kinetic_energy(built, st) - total) <= 1e-6 * total

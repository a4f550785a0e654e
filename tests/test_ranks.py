"""Multi-rank host logic on CPU: the world shards of the batched benchmark and
the max-over-ranks timing, run as two gloo ranks (the GPU runs use the same
functions over NCCL, one process per GPU)."""
import multiprocessing
import socket

import numpy as np
import pytest

import velox_b200
from velox_b200.ranks import max_over_ranks, shard_specs, world_range

BATCHED = 4  # the independent-worlds workload


@pytest.mark.parametrize("nworlds", [1, 7, 64, 4096])
@pytest.mark.parametrize("ranks", [1, 2, 3, 8])
def test_world_ranges_cover_every_world_once(nworlds, ranks):
    ranges = [world_range(nworlds, r, ranks) for r in range(ranks)]
    assert ranges[0][0] == 0 and ranges[-1][1] == nworlds
    for (lo, hi), (lo2, _) in zip(ranges, ranges[1:]):
        assert hi == lo2
    sizes = [hi - lo for lo, hi in ranges]
    assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        world_range(nworlds, ranks, ranks)


def _fields_equal(a, b):
    return all(np.array_equal(a[name], b[name]) for name in velox_b200.BODY.names)


def test_shard_bodies_are_the_batch_bodies_of_those_worlds():
    specs, pool = velox_b200.generate_scene(BATCHED, seed=BATCHED, size=16)
    whole, _, _ = velox_b200.bodies_from_specs(specs, pool)
    seen = 0
    for rank in range(3):
        mine, lo, hi = shard_specs(specs, 16, rank, 3)
        assert mine["world"].min() == 0 and mine["world"].max() == hi - lo - 1
        bodies, _, _ = velox_b200.bodies_from_specs(mine, pool)
        mask = (specs["world"] >= lo) & (specs["world"] < hi)
        assert _fields_equal(whole[mask], bodies)
        seen += len(bodies)
    assert seen == len(whole)


def _rank_main(rank, ranks, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ranks)
    try:
        specs, pool = velox_b200.generate_scene(BATCHED, seed=BATCHED, size=16)
        mine, lo, hi = shard_specs(specs, 16, rank, ranks)
        bodies, _, _ = velox_b200.bodies_from_specs(mine, pool)
        # the job's time is the slowest rank's; every rank takes the same collectives
        slowest = max_over_ranks(10.0 + rank, dist)
        total = max_over_ranks(0.0, dist)  # a second collective in the same order on every rank
        dist.barrier()
        out.put((rank, lo, hi, len(bodies), slowest, total))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_the_batch_and_agree_on_the_slowest_time():
    ranks = 2
    ctx = multiprocessing.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ranks, port, out)) for r in range(ranks)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in range(ranks))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    specs, _ = velox_b200.generate_scene(BATCHED, seed=BATCHED, size=16)
    assert [(lo, hi) for _, lo, hi, _, _, _ in results] == [(0, 8), (8, 16)]
    assert sum(n for _, _, _, n, _, _ in results) == len(specs)
    assert all(slowest == 11.0 and total == 0.0 for _, _, _, _, slowest, total in results)
    assert max_over_ranks(3.5) == 3.5  # no process group: the value itself

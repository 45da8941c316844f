"""Scene partitioning of the batched form across ranks (host logic, CPU).

The batched form shards without communication: each rank runs the scenes
``partition_scenes`` gives it and only the timing is reduced (max over
ranks).  Checked here with two gloo ranks on the CPU.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from peel_mpm_b200 import partition_scenes, scenes


def test_partition_covers_every_scene_once_and_balances():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 4, 8):
        sizes = rng.integers(4096, 262144, size=64)
        parts = partition_scenes(sizes, world)
        assert len(parts) == world
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(64))
        loads = [int(sum(sizes[k] for k in p)) for p in parts]
        # greedy largest-first: the spread is at most the largest scene
        assert max(loads) - min(loads) <= int(sizes.max())
        assert all(p == sorted(p) for p in parts)


def test_partition_edge_cases():
    assert partition_scenes([], 2) == [[], []]
    assert partition_scenes([5], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        partition_scenes([1, 2], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [sc.n for sc in scenes.batch_scenes(seed=0)]
        mine = partition_scenes(sizes, world)[rank]
        load = torch.tensor([float(sum(sizes[k] for k in mine))], dtype=torch.float64)
        gathered = [torch.zeros(64, dtype=torch.int64) for _ in range(world)]
        mask = torch.zeros(64, dtype=torch.int64)
        mask[mine] = 1
        dist.all_gather(gathered, mask)
        mx = load.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)   # the bench's max-over-ranks timing reduction
        if rank == 0:
            out.put((torch.stack(gathered).sum(0).tolist(), float(mx), sum(sizes)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_the_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    cover, max_load, total = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert cover == [1] * 64                  # every scene on exactly one rank
    assert total / 2 <= max_load <= total / 2 + 262144

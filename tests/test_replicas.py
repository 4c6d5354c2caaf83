"""Several GPUs run replicas: each rank filters its own frames and the job's time is the
slowest rank's.  The host side of that runs here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from imagestack_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        env = replicas.rank_env()
        seeds = replicas.frame_seeds(rank, 4, base_seed=2)
        mine = replicas.shard(10, rank, world)
        slowest = replicas.max_over_ranks(1.5 + rank)     # rank r "took" 1.5 + r seconds
        out.put((rank, env, seeds, mine, slowest))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_frames_and_agree_on_the_slowest_time():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.start_processes(_rank_main, args=(world, _free_port(), q), nprocs=world, join=True,
                       start_method="spawn")
    got = sorted(q.get(timeout=30) for _ in range(world))
    assert [g[1] for g in got] == [(2, 0, 0), (2, 1, 1)]
    seeds = [s for g in got for s in g[2]]
    assert len(set(seeds)) == len(seeds)                 # no frame filtered twice
    shards = [g[3] for g in got]
    assert sorted(i for sh in shards for i in sh) == list(range(10))
    assert all(g[4] == 2.5 for g in got)                 # every rank sees the max


def test_single_process_needs_no_group():
    assert replicas.max_over_ranks(3.25) == 3.25
    assert replicas.shard(5, 0, 1) == [0, 1, 2, 3, 4]
    with pytest.raises(ValueError):
        replicas.shard(5, 2, 2)
    with pytest.raises(ValueError):
        replicas.frame_seeds(0, 40, 2)

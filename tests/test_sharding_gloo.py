"""Multi-process (gloo, world size 2) checks of the clip-sharding path.

The GPU path shards clips across ranks with no data-path collective; what the
ranks do exchange -- the elapsed-time max and, here, the shard bookkeeping --
is exercised on CPU with two gloo ranks.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from metalmom_b200.shard import balanced_shards, frames_of, max_over_ranks


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, lengths, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        shards = balanced_shards(lengths, world)
        mine = shards[rank]
        frames = sum(frames_of(lengths[i]) for i in mine)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t_max = max_over_ranks(1.0 + rank, dist)
        q.put((rank, mine, frames, gathered, t_max))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_partitions_clips():
    rng = np.random.default_rng(0)
    lengths = [int(x) for x in rng.integers(22050, 120 * 22050, 37)]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, lengths, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    all_idx = sorted(i for r in results for i in r[1])
    assert all_idx == list(range(len(lengths)))          # every clip exactly once
    assert results[0][3] == results[1][3]                 # both ranks agree on the split
    f0, f1 = results[0][2], results[1][2]
    assert abs(f0 - f1) <= max(frames_of(L) for L in lengths)  # balanced within one clip
    assert all(r[4] == 2.0 for r in results)              # elapsed time: max over ranks


def test_single_rank_and_degenerate():
    assert balanced_shards([100, 200], 1) == [[0, 1]]
    assert balanced_shards([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        balanced_shards([1], 0)
    assert max_over_ranks(3.5) == 3.5

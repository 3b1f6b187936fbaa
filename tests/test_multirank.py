"""The multi-GPU host logic on CPU ranks (gloo, world size 2): the replica
reduction of bench.py (max of the ranks' times, sum of their work) and the
footprint split of batched jobs over GPUs (every rank computes the same
split; the shards partition the jobs and balance the footprints)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "icarat-contact_b200", "python"))
    import bench
    import icarat_b200 as icb
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms, units = bench.reduce_over_ranks(10.0 + 5.0 * rank, 100.0 * (rank + 1), dist, "cpu")
    fp = [int(v) for v in np.random.default_rng(1).integers(1 << 20, 1 << 30, 37)]
    mine = icb.shard_by_footprint(fp, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    dist.destroy_process_group()
    q.put((rank, ms, units, got, fp))


@pytest.mark.timeout(120)
def test_replica_reduction_and_footprint_shards():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=100) for _ in range(world)]
    for p in procs:
        p.join(30)
        assert p.exitcode == 0
    for rank, ms, units, got, fp in res:
        assert ms == 15.0 and units == 300.0  # max time, summed work
        flat = sorted(i for s in got for i in s)
        assert flat == list(range(len(fp)))    # a partition of the jobs
        loads = [sum(fp[i] for i in s) for s in got]
        assert max(loads) - min(loads) <= max(fp)  # greedy balance bound
    assert res[0][3] == res[1][3]                # both ranks computed the same split

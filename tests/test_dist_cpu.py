"""The multi-rank bench path (replicas, weak scaling) on CPU with gloo, world size 2."""

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = bench.rank_inputs(5, world, rank)
    t_local = 1.0 + rank  # a slower rank sets the job time
    t_max = bench.max_over_ranks(dist, t_local)
    total = bench.sum_over_ranks(dist, float(len(mine)))
    q.put((rank, list(mine), t_max, total))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_shard_inputs_and_aggregate_over_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    sys.path.insert(0, ROOT)
    import bench

    allj = bench.j2_stream(5 * world)
    got = np.concatenate([np.array(o[1]) for o in out])
    assert sorted(got.tolist()) == sorted(allj.tolist())  # every input once, no overlap
    assert all(o[2] == 2.0 for o in out)  # max over ranks
    assert all(o[3] == 10.0 for o in out)  # value = all units of all ranks / max time

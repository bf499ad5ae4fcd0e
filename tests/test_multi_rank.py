"""The multi-GPU form is replicas: every rank generates its own request set (seeds
offset by rank) and the only collective is the final reduction of the timings
(max over ranks) and star counts (sum).  Checked here with two gloo ranks on CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from galfast_b200 import workloads as W
    tmax, tsum = bench.reduce_max_sum(dist, 10.0 + rank, 1000.0 * (rank + 1))
    reqs = W.config4_requests(4, seed=1234567 + bench.C4_NREQ * rank)
    out.put((rank, tmax, tsum, [r["seed48"] for r in reqs]))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_reduction_and_request_sharding_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, tmax, tsum, seeds in res:
        assert tmax == 11.0                 # the slowest rank's time
        assert tsum == 3000.0               # all ranks' stars
    assert not set(res[0][3]) & set(res[1][3])   # different requests on each rank

"""Multi-rank host logic of bench.py on CPU: two gloo ranks, each an
independent replica with its own timing; the job value is the sum of the
ranks' attempted moves over the slowest rank's time, and only rank 0 would
run the reference arm."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import bench
    ranks = bench.Ranks(backend="gloo")
    ranks.barrier()
    attempts = 1000
    dev_s = 1.0 + rank            # rank 1 is the slower replica
    e2e_s = 2.0 + rank
    value, e2e, total = bench.aggregate(ranks, attempts, dev_s, e2e_s)
    out[rank] = (value, e2e, total, ranks.rank, ranks.world)
    ranks.close()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_aggregate_weak_scaling():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        value, e2e, total, rank, w = out[r]
        assert w == world and rank == r
        assert total == 2000
        assert value == pytest.approx(2000 / 2.0)   # slowest device time: 2.0 s
        assert e2e == pytest.approx(2000 / 3.0)     # slowest end-to-end time: 3.0 s

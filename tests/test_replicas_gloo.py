"""The multi-GPU path of bench.py is replicas only (the scoring path has no exchange step):
each rank scores the whole workload on its own GPU and the job time is the max over ranks.
This checks that host-side plumbing -- barrier and max-reduction over gloo -- with two
CPU ranks, no GPU involved."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench

    g = bench.Group(world)
    g.barrier()
    # rank r reports device times [10, 20 * (r + 1)] ms for 2 steps of 1e12 cells each
    gcups, max_ms = bench.aggregate(g, world, 1e12, 2, [10.0, 20.0 * (rank + 1)])
    g.barrier()
    g.close()
    q.put((rank, gcups, max_ms))


@pytest.mark.timeout(120)
def test_two_replicas_aggregate_with_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    # slowest rank: 10 + 40 = 50 ms; 2 replicas x 2 steps x 1e12 cells / 0.05 s
    for _, gcups, max_ms in out:
        assert max_ms == pytest.approx(50.0)
        assert gcups == pytest.approx(2 * 1e12 * 2 / 0.05 / 1e9)


def test_single_process_group_is_a_noop():
    import bench

    g = bench.Group(1)
    g.barrier()
    assert g.max(3.5) == 3.5
    assert bench.aggregate(g, 1, 1e9, 1, [1000.0]) == (pytest.approx(1.0), 1000.0)

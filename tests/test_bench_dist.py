"""The multi-GPU plumbing of bench.py on CPU: two gloo ranks.  Each rank
converts its own seeded volume (weak scaling, no collective on the data path)
and the reported time is the slowest rank's."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    slowest = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
    q.put((rank, slowest, bench.volume_seed(rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_distinct_volumes_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [15.0, 15.0]
    assert res[0][2] != res[1][2]


def test_max_over_ranks_single_process_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5

"""One volume's blocked construction split by z-tiles over two gloo ranks on
CPU (libapr_b200.distributed with the oracle as the tile backend): each rank
reads only its tiles' planes and ghosts, the ranks' particle-cell pyramids are
combined by one MAX all-reduce, and the structure both ranks build equals the
single-process blocked converter's (APRConverterBatch), bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from libapr_b200 import distributed as D

SHAPE, BLOBS, SEED = (40, 48, 56), 40, 12
CASES = [(9, 3), (5, 2), (16, 0), (10, 4)]  # (z_block, ghost): 4 to 8 tiles, in-bounds tilings


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, zblock, ghost, q):
    import datetime

    import torch.distributed as dist
    from oracle import bind as B
    from tests.helpers import oracle_params, volume
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    img = volume(SHAPE, BLOBS, SEED)
    lo, hi = D.rank_slab(SHAPE[0], zblock, ghost, rank, world)
    slab = np.ascontiguousarray(img[lo:hi])  # this rank's planes only
    acc = D.get_apr_by_block_distributed(B.OracleTileBackend(oracle_params()), SHAPE, slab, lo, zblock, ghost)
    q.put((rank, acc.xz_end.tobytes(), acc.y_vec.tobytes(), (lo, hi)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("zblock,ghost", CASES)
def test_two_gloo_ranks_equal_single_process_blocked_converter(zblock, ghost):
    from oracle import bind as B
    from tests.helpers import oracle_params, volume
    if not B.block_tiling_in_bounds(SHAPE, zblock, ghost):
        pytest.skip("tiling where the reference writes outside a coarse level")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, zblock, ghost, q)) for r in range(2)]
    for p in procs:
        p.start()
    # read the results before joining: a rank exits only once its queue is drained
    res = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    img = volume(SHAPE, BLOBS, SEED)
    e, ref = B.orc_get_apr_by_block(img, oracle_params(), 1, zblock, ghost)
    assert e == 0
    for rank, xe, yv, (lo, hi) in res:
        assert np.array_equal(np.frombuffer(xe, np.uint64), ref.xz_end), rank
        assert np.array_equal(np.frombuffer(yv, np.uint16), ref.y_vec), rank
    # the ranks read different planes (their tiles and ghosts), not the whole volume
    assert res[0][3] != res[1][3] and (res[0][3][1] - res[0][3][0]) < SHAPE[0]


def test_tile_partition_covers_every_tile_once():
    for nt in range(1, 12):
        for world in range(1, 6):
            got = []
            for r in range(world):
                f, c = D.rank_tiles(nt, r, world)
                got += list(range(f, f + c))
            assert got == list(range(nt))


def test_one_process_oracle_backend_matches_blocked_converter():
    """world size 1 (no process group): the same function is the blocked converter"""
    from oracle import bind as B
    from tests.helpers import oracle_params, volume
    img = volume(SHAPE, BLOBS, SEED)
    acc = D.get_apr_by_block_distributed(B.OracleTileBackend(oracle_params()), SHAPE, img, 0, 12, 3)
    e, ref = B.orc_get_apr_by_block(img, oracle_params(), 1, 12, 3)
    assert e == 0 and np.array_equal(acc.y_vec, ref.y_vec) and np.array_equal(acc.xz_end, ref.xz_end)

"""GPU parity of the blocked converter (APRConverterBatch) and of blocked
sampling against the CPU oracle, bit-exact, through the C ABI; and the batch
entry point against per-volume calls."""
import numpy as np
import pytest

import libapr_b200 as A
from oracle import bind as B
from tests.helpers import lib_params, oracle_params, volume

pytestmark = pytest.mark.gpu

CASES = [((100, 40, 48), 32, 8, 1), ((96, 30, 40), 20, 8, 0), ((65, 37, 29), 16, 4, 1), ((200, 32, 32), 128, 16, 0),
         ((80, 24, 70), 16, 16, 1), ((64, 40, 30), 128, 32, 1), ((70, 33, 50), 16, 4, 1), ((9, 20, 30), 4, 2, 1)]


@pytest.mark.parametrize("shape,zb,ghost,image_type", CASES)
def test_get_apr_by_block_bit_exact(shape, zb, ghost, image_type):
    img = volume(shape, 30, 3)
    e, acc = B.orc_get_apr_by_block(img, oracle_params(), image_type, zb, ghost)
    assert e == 0
    conv = A.APRConverterBatch("uint16" if image_type == 1 else "float", z_block_size=zb, ghost_z=ghost)
    conv.par = lib_params()
    apr = A.APR()
    assert conv.get_apr(apr, img)
    lx, xe, yv = apr.linear_access()
    assert np.array_equal(lx, acc.level_xz)
    assert np.array_equal(xe, acc.xz_end)
    assert np.array_equal(yv, acc.y_vec)
    parts = A.ParticleData().sample_parts_from_img_blocked(apr, img, zb, ghost).data
    assert np.array_equal(parts, B.orc_sample_by_block(acc, img, zb, ghost))


def test_get_apr_by_block_overflow_raises_like_reference():
    img = np.zeros((40, 20, 24), np.uint16)
    img[10:30, 5:15, 6:18] = 65535
    conv = A.APRConverterBatch("uint16", z_block_size=16, ghost_z=4)
    conv.par = lib_params()
    with pytest.raises(ValueError):
        conv.get_apr(A.APR(), img)


def test_batch_matches_per_volume_calls():
    import torch
    rng = np.random.default_rng(5)
    shapes = [(int(rng.choice([16, 24, 40])), int(rng.choice([16, 32, 48])), int(rng.choice([20, 64]))) for _ in range(6)]
    imgs = [volume(s, 8, 100 + i) for i, s in enumerate(shapes)]
    conv = A.APRConverterBatch("uint16", z_block_size=16, ghost_z=4)
    conv.par = lib_params()
    dev = [torch.from_numpy(im.view(np.int16)).cuda() for im in imgs]
    aprs = conv.get_apr_batch(dev)
    for im, apr in zip(imgs, aprs):
        one = A.APR()
        assert conv.get_apr(one, im)
        for a, b in zip(apr.linear_access(), one.linear_access()):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("shape,zb,ghost,image_type,world",
                         [((100, 40, 48), 32, 8, 1, 2), ((200, 32, 32), 32, 16, 0, 3), ((84, 33, 50), 16, 4, 1, 4),
                          ((96, 30, 40), 20, 8, 0, 2)])
def test_split_by_tiles_equals_blocked_converter(shape, zb, ghost, image_type, world):
    """The multi-GPU split on one GPU: each of `world` emulated ranks fills
    its own pyramid from its own slab (its tiles and ghosts only), the
    pyramids are combined by element-wise maximum (what the MAX all-reduce
    computes) and the structure built from the result equals the blocked
    converter's and the oracle's."""
    import torch
    from libapr_b200 import distributed as D
    if not B.block_tiling_in_bounds(shape, zb, ghost):
        pytest.skip("tiling where the reference writes outside a coarse level")
    img = volume(shape, 30, 3)
    it = "uint16" if image_type == 1 else "float"
    be = D.TileBackend(it, lib_params())
    total = None
    for r in range(world):
        lo, hi = D.rank_slab(shape[0], zb, ghost, r, world)
        first, count = D.rank_tiles(D.tile_count(shape[0], zb), r, world)
        pyr = be.pyramid(shape)
        if count:
            slab = torch.from_numpy(np.ascontiguousarray(img[lo:hi]).view(np.int16)).cuda()
            be.fill(pyr, shape, zb, ghost, first, count, slab, lo)
        total = pyr if total is None else torch.maximum(total, pyr)
    apr = be.finish(total, shape)
    conv = A.APRConverterBatch(it, z_block_size=zb, ghost_z=ghost)
    conv.par = lib_params()
    one = A.APR()
    assert conv.get_apr(one, img)
    for a, b in zip(apr.linear_access(), one.linear_access()):
        assert np.array_equal(a, b)
    e, acc = B.orc_get_apr_by_block(img, oracle_params(), image_type, zb, ghost)
    assert e == 0 and np.array_equal(apr.linear_access()[2], acc.y_vec)

"""One volume's blocked construction split over the ranks of a process group
(one GPU per rank, torch.distributed over NCCL).

APRConverterBatch (src/algorithm/APRConverterBatch.hpp:114-175) runs the pixel
pipeline per z-tile of ``z_block_size`` planes with ``ghost_z`` planes of
overlap, lets every tile fill one global particle-cell tree
(fill_global_particle_cell_tree :282-314, PullingScheme::fill_patch
PullingScheme.hpp:175-247) and solves that tree once.  A tile only ever sets
cells to SEED, so the tree of all tiles is the element-wise maximum of the
trees of any partition of the tiles.  Here each rank converts a contiguous
range of the tiles from its own z-slab of the volume (the tiles' planes plus
their ghosts: no rank needs the whole volume), the ranks' pyramids are
combined by one MAX all-reduce of a single uint8 buffer (about N / 7 bytes
for N voxels), and every rank runs the pulling scheme and the linear
structure on the combined tree, so that each holds the volume's whole APR.
The structure is the one the single-process blocked converter builds, bit for
bit.

The tile work goes through a backend with three calls: ``pyramid(shape)``
(a zeroed buffer on the backend's device), ``fill(pyr, shape, z_block, ghost,
first, count, slab, slab_z0)`` and ``finish(pyr, shape)``.  ``TileBackend``
is the GPU one (the library's C ABI); the CPU checker drives the same
function with a backend over the oracle on gloo ranks.
"""
import ctypes as C

from ._lib import check, lib


def tile_count(z_num, z_block_size):
    """Number of z-tiles of APRConverterBatch (APRConverterBatch.hpp:125)."""
    return max(z_num // z_block_size, 1)


def tile_planes(z_num, z_block_size, ghost_z, b):
    """(first plane, end plane) of tile b with its ghosts
    (APRConverterBatch.hpp:137-160)."""
    nb = tile_count(z_num, z_block_size)
    z0 = b * z_block_size
    zf = z_num if b == nb - 1 else (b + 1) * z_block_size
    return z0 - min(z0, ghost_z), zf + min(z_num - zf, ghost_z)


def rank_tiles(n_tiles, rank, world):
    """Contiguous tile range (first, count) of a rank: the first n_tiles %
    world ranks take one tile more."""
    base, extra = divmod(n_tiles, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def rank_slab(z_num, z_block_size, ghost_z, rank, world):
    """Planes [lo, hi) of the volume a rank reads: its tiles and their ghosts
    (empty when the rank has no tile)."""
    first, count = rank_tiles(tile_count(z_num, z_block_size), rank, world)
    if count == 0:
        return 0, 0
    return (tile_planes(z_num, z_block_size, ghost_z, first)[0],
            tile_planes(z_num, z_block_size, ghost_z, first + count - 1)[1])


class TileBackend:
    """The GPU side: a library converter (ImageType ``image_type``) and
    parameters; slabs and pyramids are CUDA tensors."""

    def __init__(self, image_type, par, stream=None):
        from . import APRConverter
        self.conv = APRConverter(image_type)
        self.par = par
        self.stream = stream

    def _s(self):
        return None if self.stream is None else C.c_void_p(self.stream.cuda_stream)

    def pyramid(self, shape):
        import torch
        z, x, y = shape
        n = C.c_uint64()
        check(lib().aprb_pyramid_bytes(y, x, z, C.byref(n)))
        return torch.zeros(int(n.value), dtype=torch.uint8, device="cuda")

    def fill(self, pyr, shape, z_block_size, ghost_z, first, count, slab, slab_z0):
        z, x, y = shape
        p = self.par.c()
        check(lib().aprb_pyramid_fill_tiles_device(self.conv._h, C.byref(p), C.c_void_p(pyr.data_ptr()), y, x, z,
                                                   z_block_size, ghost_z, first, count,
                                                   C.c_void_p(slab.data_ptr()), slab_z0, slab.shape[0], self._s()))

    def finish(self, pyr, shape):
        from . import APR
        z, x, y = shape
        p = self.par.c()
        h = C.c_void_p()
        check(lib().aprb_get_apr_from_pyramid_device(self.conv._h, C.byref(p), C.c_void_p(pyr.data_ptr()), y, x, z,
                                                     self._s(), C.byref(h)))
        apr = APR()
        apr._set(h)
        return apr


def get_apr_by_block_distributed(backend, shape, slab, slab_z0, z_block_size=128, ghost_z=16, group=None):
    """The blocked converter over the ranks of ``group`` (the default group
    when None, one process when torch.distributed is not initialised).
    ``shape`` is the whole volume's (z, x, y); ``slab`` holds planes
    [slab_z0, slab_z0 + len(slab)) and must contain this rank's tiles and
    ghosts (``rank_slab``).  Every rank takes part in the one all-reduce and
    returns the volume's APR."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    z = shape[0]
    first, count = rank_tiles(tile_count(z, z_block_size), rank, world)
    pyr = backend.pyramid(shape)
    if count:
        backend.fill(pyr, shape, z_block_size, ghost_z, first, count, slab, slab_z0)
    if world > 1:
        dist.all_reduce(pyr, op=dist.ReduceOp.MAX, group=group)
    return backend.finish(pyr, shape)


__all__ = ["TileBackend", "get_apr_by_block_distributed", "rank_slab", "rank_tiles", "tile_count", "tile_planes"]

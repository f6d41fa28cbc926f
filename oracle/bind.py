"""TEST INFRASTRUCTURE ONLY -- ctypes bindings for the CPU checkers.

* ``liboracle.so``: the plain-C restatement of LibAPR's path (apr_oracle.c).
* ``_ref/libaprref.so``: LibAPR's own CPU code compiled from its headers
  (strict IEEE flags); ``_ref/libaprref_fast.so`` the same at the reference's
  Release flags (-O3 -ffast-math), used only for timing.
* ``libblobs.so``: the CPU twin of the library's synthetic-volume generator
  (the same bytes as ``aprb_synth_blobs_u16`` / ``_f32``, without a GPU).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Images are numpy arrays of shape (z, x, y) in C order, i.e. the
reference's PixelData memory order (y fastest).
"""
import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAXL = 32


class OrcParams(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("dx", "dy", "dz", "psfx", "psfy", "psfz", "Ip_th", "lambda_",
                                         "rel_error", "sigma_th", "sigma_th_max", "grad_th")] + \
               [(n, C.c_int) for n in ("reflect_bc_lis", "neighborhood_optimization", "constant_intensity_scale")]


class OrcAccess(C.Structure):
    _fields_ = [("l_min", C.c_int), ("l_max", C.c_int), ("org", C.c_int * 3),
                ("y_num", C.c_int * MAXL), ("x_num", C.c_int * MAXL), ("z_num", C.c_int * MAXL),
                ("level_xz", C.c_uint64 * (MAXL + 2)), ("n_xz", C.c_uint64),
                ("xz_end", C.POINTER(C.c_uint64)), ("P", C.c_uint64), ("y_vec", C.POINTER(C.c_uint16))]


def make_params(lambda_=3.0, rel_error=0.1, Ip_th=0.0, sigma_th=0.0, sigma_th_max=0.0, grad_th=0.0,
                dx=1.0, dy=1.0, dz=1.0, psfx=2.0, psfy=2.0, psfz=2.0, reflect_bc_lis=1,
                neighborhood_optimization=1, constant_intensity_scale=0):
    return OrcParams(dx, dy, dz, psfx, psfy, psfz, Ip_th, lambda_, rel_error, sigma_th, sigma_th_max,
                     grad_th, reflect_bc_lis, neighborhood_optimization, constant_intensity_scale)


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


_lib = None
_ref = {}
_blobs = None


def blobs_lib():
    global _blobs
    if _blobs is None:
        L = C.CDLL(os.path.join(HERE, "libblobs.so"))
        for n, t in (("blobs_render_u16", C.c_uint16), ("blobs_render_f32", C.c_float)):
            f = getattr(L, n)
            f.argtypes = [C.POINTER(t), C.c_int, C.c_int, C.c_int, C.c_int] + [C.c_float] * 5 + [C.c_uint64]
            f.restype = C.c_int
        _blobs = L
    return _blobs


def blob_volume_cpu(shape_zxy, n_blobs, sigma, amp, background, seed, noise=True, out=None):
    """The benchmark generator's volume on the host cores: (z, x, y) uint16
    with Poisson noise, or float32 noise-free intensities; bit-identical to
    the device generator for the same arguments."""
    z, x, y = (int(v) for v in shape_zxy)
    dt = np.uint16 if noise else np.float32
    if out is None:
        out = np.empty((z, x, y), dt)
    assert out.dtype == dt and out.shape == (z, x, y) and out.flags.c_contiguous
    f = blobs_lib().blobs_render_u16 if noise else blobs_lib().blobs_render_f32
    e = f(_ptr(out, C.c_uint16 if noise else C.c_float), y, x, z, int(n_blobs), float(sigma[0]), float(sigma[1]),
          float(amp[0]), float(amp[1]), float(background), int(seed))
    if e != 0:
        raise MemoryError("blob generator could not allocate its brick lists")
    return out


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(os.path.join(HERE, "liboracle.so"))
        L.orc_get_apr.argtypes = [C.POINTER(C.c_uint16), C.c_int, C.c_int, C.c_int, C.POINTER(OrcParams),
                                  C.c_int, C.POINTER(C.c_void_p)]
        L.orc_get_apr_custom.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int,
                                         C.POINTER(OrcParams), C.POINTER(C.c_void_p)]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_get_access.argtypes = [C.c_void_p]
        L.orc_get_access.restype = C.POINTER(OrcAccess)
        L.orc_copy_intermediate.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.c_size_t]
        L.orc_bspline_offset.argtypes = [C.c_void_p]
        L.orc_bspline_offset.restype = C.c_float
        L.orc_sample_image.argtypes = [C.POINTER(OrcAccess), C.POINTER(C.c_uint16), C.POINTER(C.c_uint16)]
        L.orc_tree_init.argtypes = [C.POINTER(OrcAccess), C.POINTER(OrcAccess)]
        L.orc_access_free.argtypes = [C.POINTER(OrcAccess)]
        L.orc_fill_tree_mean.argtypes = [C.POINTER(OrcAccess), C.POINTER(OrcAccess), C.POINTER(C.c_float),
                                         C.POINTER(C.c_float)]
        L.orc_downsampled_stencils.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int,
                                               C.POINTER(C.c_float), C.POINTER(C.c_int)]
        L.orc_convolve.argtypes = [C.POINTER(OrcAccess), C.POINTER(OrcAccess), C.POINTER(C.c_float),
                                   C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                   C.c_int, C.POINTER(C.c_uint64)]
        L.orc_richardson_lucy.argtypes = [C.POINTER(OrcAccess), C.POINTER(OrcAccess), C.POINTER(C.c_uint16),
                                          C.c_void_p, C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.c_int]
        L.orc_bspline_axis.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int]
        L.orc_bspline_axis.restype = C.c_uint64
        L.orc_get_apr_by_block.argtypes = [C.POINTER(C.c_uint16), C.c_int, C.c_int, C.c_int, C.POINTER(OrcParams),
                                           C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.orc_sample_image_by_block.argtypes = [C.POINTER(OrcAccess), C.POINTER(C.c_uint16), C.c_int, C.c_int,
                                                C.POINTER(C.c_uint16)]
        L.orc_pyramid_bytes.argtypes = [C.c_int, C.c_int, C.c_int]
        L.orc_pyramid_bytes.restype = C.c_size_t
        L.orc_pyramid_fill_tiles.argtypes = [C.POINTER(C.c_uint16), C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.POINTER(OrcParams), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.POINTER(C.c_uint8)]
        L.orc_apr_from_pyramid.argtypes = [C.POINTER(C.c_uint8), C.c_int, C.c_int, C.c_int, C.POINTER(OrcParams),
                                           C.POINTER(C.c_void_p)]
        L.orc_threshold_li.argtypes = [C.POINTER(C.c_float), C.c_size_t, C.c_int, C.c_int]
        L.orc_threshold_li.restype = C.c_float
        L.orc_auto_parameters.argtypes = [C.POINTER(C.c_float)] * 3 + [C.c_size_t, C.c_float, C.c_int, C.c_int] + \
            [C.POINTER(C.c_float)] * 4 + [C.POINTER(C.c_size_t)]
        _lib = L
    return _lib


_bind = None


def bind_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libaprbind.so"))


def bind_lib():
    """_ref/libaprbind.so: include/aprb200_libapr.hpp driven with LibAPR's own
    objects (see ref_bind.cu)."""
    global _bind
    if _bind is None:
        L = C.CDLL(os.path.join(HERE, "_ref", "libaprbind.so"))
        vp, u16p = C.c_void_p, C.POINTER(C.c_uint16)
        L.bind_get_apr.argtypes = [u16p, C.c_int, C.c_int, C.c_int, C.POINTER(OrcParams), C.c_int,
                                   C.POINTER(vp), C.POINTER(C.c_uint64), C.POINTER(C.c_float)]
        L.bind_free.argtypes = [vp]
        L.bind_free.restype = None
        L.bind_particles.argtypes = [vp, u16p, u16p, u16p, u16p]
        L.bind_sample.argtypes = [vp, u16p, u16p]
        L.bind_convolve.argtypes = [vp, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                    C.c_int, C.c_int, C.c_int, C.c_int]
        L.bind_rl.argtypes = [vp, u16p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int]
        L.bind_get_apr_by_block.argtypes = [u16p, C.c_int, C.c_int, C.c_int, C.POINTER(OrcParams), C.c_int, C.c_int,
                                            C.c_int, C.POINTER(vp), C.POINTER(C.c_uint64)]
        L.bind_sample_blocked.argtypes = [vp, u16p, C.c_int, C.c_int, u16p]
        _bind = L
    return _bind


def ref_available(fast=False):
    return os.path.exists(os.path.join(HERE, "_ref", "libaprref_fast.so" if fast else "libaprref.so"))


def ref(fast=False):
    if fast not in _ref:
        R = C.CDLL(os.path.join(HERE, "_ref", "libaprref_fast.so" if fast else "libaprref.so"))
        vp = C.c_void_p
        R.ref_get_apr.argtypes = [C.POINTER(C.c_uint16), C.c_int, C.c_int, C.c_int, C.POINTER(OrcParams), C.c_int,
                                  C.POINTER(vp)]
        R.ref_get_apr_plain.argtypes = R.ref_get_apr.argtypes
        R.ref_gradient.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.c_int,
                                   C.POINTER(C.c_float)]
        R.ref_get_apr_custom.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int,
                                         C.POINTER(OrcParams), C.POINTER(vp)]
        R.ref_free.argtypes = [vp]
        R.ref_apr_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_float)]
        R.ref_apr_copy.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint16)]
        R.ref_copy_intermediate.argtypes = [vp, C.c_int, C.POINTER(C.c_float), C.c_size_t]
        R.ref_apr_from_arrays.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64), C.c_uint64,
                                          C.POINTER(C.c_uint64), C.c_uint64, C.POINTER(C.c_uint16), C.c_uint64]
        R.ref_apr_from_arrays.restype = vp
        R.ref_sample_image.argtypes = [vp, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16)]
        R.ref_tree_info.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        R.ref_tree_copy.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint16)]
        R.ref_fill_tree_mean.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        R.ref_convolve_pencil.argtypes = [vp, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float),
                                          C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int]
        R.ref_richardson_lucy.argtypes = [vp, C.POINTER(C.c_uint16), vp, C.POINTER(C.c_float), C.c_int, C.c_int,
                                          C.c_int, C.c_int, C.c_int, C.c_int]
        R.ref_get_apr_by_block.argtypes = [C.POINTER(C.c_uint16), C.c_int, C.c_int, C.c_int, C.POINTER(OrcParams),
                                           C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        R.ref_sample_image_by_block.argtypes = [vp, C.POINTER(C.c_uint16), C.c_int, C.c_int, C.POINTER(C.c_uint16)]
        R.ref_smooth.argtypes = [C.POINTER(C.c_uint16), C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_float,
                                 C.POINTER(C.c_float)]
        R.ref_threshold_li.argtypes = [C.POINTER(C.c_float), C.c_size_t, C.c_int, C.c_int]
        R.ref_threshold_li.restype = C.c_float
        R.ref_auto_parameters.argtypes = [C.POINTER(C.c_float)] * 3 + [C.c_int] * 4 + [C.c_float, C.c_float, C.c_int,
                                                                           C.POINTER(C.c_float), C.POINTER(C.c_float)]
        R.ref_get_apr_auto.argtypes = [C.POINTER(C.c_uint16), C.c_int, C.c_int, C.c_int, C.POINTER(OrcParams),
                                       C.c_int, C.c_int, C.POINTER(vp), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        R.ref_get_apr_by_block_auto.argtypes = [C.POINTER(C.c_uint16), C.c_int, C.c_int, C.c_int,
                                                C.POINTER(OrcParams), C.c_int, C.c_int, C.c_int, C.c_int,
                                                C.POINTER(vp), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        _ref[fast] = R
    return _ref[fast]


class Access:
    """A linear access structure held as numpy arrays (LinearAccess.hpp:33-35)."""

    def __init__(self, org, l_min, l_max, y_num, x_num, z_num, level_xz, xz_end, y_vec):
        self.org = tuple(int(v) for v in org)
        self.l_min, self.l_max = int(l_min), int(l_max)
        self.y_num, self.x_num, self.z_num = list(y_num), list(x_num), list(z_num)
        self.level_xz = np.ascontiguousarray(level_xz, dtype=np.uint64)
        self.xz_end = np.ascontiguousarray(xz_end, dtype=np.uint64)
        self.y_vec = np.ascontiguousarray(y_vec, dtype=np.uint16)

    @property
    def P(self):
        return int(self.xz_end[-1]) if len(self.xz_end) else 0

    def c(self):
        s = OrcAccess()
        s.l_min, s.l_max = self.l_min, self.l_max
        for i in range(3):
            s.org[i] = self.org[i]
        for l in range(MAXL):
            s.y_num[l] = self.y_num[l] if l < len(self.y_num) else 0
            s.x_num[l] = self.x_num[l] if l < len(self.x_num) else 0
            s.z_num[l] = self.z_num[l] if l < len(self.z_num) else 0
        for i in range(min(len(self.level_xz), MAXL + 2)):
            s.level_xz[i] = int(self.level_xz[i])
        s.n_xz = len(self.xz_end)
        s.xz_end = _ptr(self.xz_end, C.c_uint64)
        s.P = self.P
        s.y_vec = _ptr(self.y_vec, C.c_uint16) if len(self.y_vec) else _ptr(np.zeros(1, np.uint16), C.c_uint16)
        s._keep = (self.xz_end, self.y_vec)
        return s

    @staticmethod
    def from_c(s):
        L = s.l_max
        return Access([s.org[i] for i in range(3)], s.l_min, L, [s.y_num[i] for i in range(MAXL)],
                      [s.x_num[i] for i in range(MAXL)], [s.z_num[i] for i in range(MAXL)],
                      np.array([s.level_xz[i] for i in range(L + 2)], dtype=np.uint64),
                      np.ctypeslib.as_array(s.xz_end, shape=(s.n_xz,)).copy(),
                      np.ctypeslib.as_array(s.y_vec, shape=(max(s.P, 1),))[: s.P].copy())

    def rows(self, level):
        """(z, x, begin, end) for every row of a level."""
        base = int(self.level_xz[level])
        xn, zn = self.x_num[level], self.z_num[level]
        e = self.xz_end[base: base + xn * zn]
        b = self.xz_end[base - 1: base - 1 + xn * zn]
        return b.astype(np.int64), e.astype(np.int64)

    def particle_coords(self):
        """Per particle (level, z, x, y) arrays in linear order."""
        lev = np.zeros(self.P, np.int32)
        zz = np.zeros(self.P, np.int32)
        xx = np.zeros(self.P, np.int32)
        for l in range(self.l_min, self.l_max + 1):
            b, e = self.rows(l)
            xn = self.x_num[l]
            cnt = e - b
            idx = np.repeat(np.arange(len(cnt)), cnt)
            sl = slice(int(b[0]) if len(b) else 0, int(e[-1]) if len(e) else 0)
            lev[sl] = l
            zz[sl] = idx // xn
            xx[sl] = idx % xn
        return lev, zz, xx, self.y_vec.astype(np.int32)


def orc_get_apr(img, params, image_type=1, keep=True):
    """Returns (Access, offset, intermediates dict) from the C restatement."""
    L = lib()
    img = np.ascontiguousarray(img, dtype=np.uint16)
    z, x, y = img.shape
    h = C.c_void_p()
    e = L.orc_get_apr(_ptr(img, C.c_uint16), y, x, z, C.byref(params), image_type, C.byref(h))
    if e != 0:
        return e, None, None
    acc = Access.from_c(L.orc_get_access(h).contents)
    off = L.orc_bspline_offset(h)
    inter = {}
    if keep:
        yd, xd, zd = (y + 1) // 2, (x + 1) // 2, (z + 1) // 2
        for w in range(7):
            shp = (z, x, y) if w == 0 else (zd, xd, yd)
            a = np.zeros(shp, np.float32)
            if L.orc_copy_intermediate(h, w, _ptr(a, C.c_float), a.size) == 0:
                inter[w] = a
    L.orc_free(h)
    return 0, acc, (off, inter)


def orc_get_apr_custom(grad, lis, shape_zxy, params):
    L = lib()
    z, x, y = shape_zxy
    g = np.ascontiguousarray(grad, dtype=np.float32)
    s = np.ascontiguousarray(lis, dtype=np.float32)
    h = C.c_void_p()
    e = L.orc_get_apr_custom(_ptr(g, C.c_float), _ptr(s, C.c_float), y, x, z, C.byref(params), C.byref(h))
    assert e == 0
    acc = Access.from_c(L.orc_get_access(h).contents)
    L.orc_free(h)
    return acc


def orc_get_apr_by_block(img, params, image_type, z_block, ghost):
    """Blocked construction (APRConverterBatch) from the C restatement."""
    L = lib()
    img = np.ascontiguousarray(img, dtype=np.uint16)
    z, x, y = img.shape
    h = C.c_void_p()
    e = L.orc_get_apr_by_block(_ptr(img, C.c_uint16), y, x, z, C.byref(params), image_type, z_block, ghost,
                               C.byref(h))
    if e != 0:
        return e, None
    acc = Access.from_c(L.orc_get_access(h).contents)
    L.orc_free(h)
    return 0, acc


class OracleTileBackend:
    """The CPU checker behind libapr_b200.distributed.get_apr_by_block_distributed:
    the oracle's tile fill and pyramid solve on CPU torch tensors (gloo ranks)."""

    def __init__(self, params, image_type=1):
        self.p, self.it = params, image_type

    def pyramid(self, shape):
        import torch
        z, x, y = shape
        return torch.zeros(int(lib().orc_pyramid_bytes(y, x, z)), dtype=torch.uint8)

    def fill(self, pyr, shape, z_block, ghost, first, count, slab, slab_z0):
        z, x, y = shape
        a = np.ascontiguousarray(slab.numpy() if hasattr(slab, "numpy") else slab, dtype=np.uint16)
        pv = pyr.numpy()
        assert lib().orc_pyramid_fill_tiles(_ptr(a, C.c_uint16), slab_z0, y, x, z, C.byref(self.p), self.it,
                                            z_block, ghost, first, count, _ptr(pv, C.c_uint8)) == 0

    def finish(self, pyr, shape):
        z, x, y = shape
        h = C.c_void_p()
        pv = pyr.numpy()
        assert lib().orc_apr_from_pyramid(_ptr(pv, C.c_uint8), y, x, z, C.byref(self.p), C.byref(h)) == 0
        acc = Access.from_c(lib().orc_get_access(h).contents)
        lib().orc_free(h)
        return acc


def orc_sample_by_block(acc, img, z_block, ghost):
    out = np.zeros(max(acc.P, 1), np.uint16)
    img = np.ascontiguousarray(img, dtype=np.uint16)
    assert lib().orc_sample_image_by_block(C.byref(acc.c()), _ptr(img, C.c_uint16), z_block, ghost,
                                           _ptr(out, C.c_uint16)) == 0
    return out[:acc.P]


def orc_sample(acc, img):
    out = np.zeros(acc.P, np.uint16)
    img = np.ascontiguousarray(img, dtype=np.uint16)
    lib().orc_sample_image(C.byref(acc.c()), _ptr(img, C.c_uint16), _ptr(out, C.c_uint16))
    return out


def orc_reconstruct(acc, parts=None):
    """APRReconstruction::reconstruct_constant (parts given) or
    reconstruct_level (src/numerics/APRReconstruction.hpp:80-123, 132-170)
    restated in numpy: every full-resolution pixel takes the value (or the
    level) of the particle whose cell covers it; a particle of level l covers
    2^(l_max - l) samples per axis, clipped at the image edge.  Returns a
    (z, x, y) array: the parts' dtype, or uint8 levels."""
    L = acc.l_max
    Y, X, Z = acc.y_num[L], acc.x_num[L], acc.z_num[L]
    lev, zz, xx, yy = acc.particle_coords()
    vals = lev.astype(np.uint8) if parts is None else np.asarray(parts)
    out = np.empty((Z, X, Y), vals.dtype)
    for l in range(acc.l_min, L + 1):
        m = np.nonzero(lev == l)[0]
        if not len(m):
            continue
        st = 1 << (L - l)
        if st <= 8:
            for dz in range(st):
                for dx in range(st):
                    for dy in range(st):
                        z, x, y = zz[m] * st + dz, xx[m] * st + dx, yy[m] * st + dy
                        ok = (z < Z) & (x < X) & (y < Y)
                        out[z[ok], x[ok], y[ok]] = vals[m[ok]]
        else:
            for i in m:
                out[zz[i] * st:(zz[i] + 1) * st, xx[i] * st:(xx[i] + 1) * st, yy[i] * st:(yy[i] + 1) * st] = vals[i]
    return out


def orc_tree(acc):
    L = lib()
    t = OrcAccess()
    ca = acc.c()
    assert L.orc_tree_init(C.byref(ca), C.byref(t)) == 0
    tr = Access.from_c(t)
    L.orc_access_free(C.byref(t))
    return tr


def orc_tree_mean(acc, tree, parts):
    out = np.zeros(max(tree.P, 1), np.float32)
    p = np.ascontiguousarray(parts, dtype=np.float32)
    lib().orc_fill_tree_mean(C.byref(acc.c()), C.byref(tree.c()), _ptr(p, C.c_float), _ptr(out, C.c_float))
    return out[: tree.P]


def orc_stencils(stencil, nlevels, normalize):
    st = np.ascontiguousarray(stencil, dtype=np.float32).ravel()
    ks = int(round(st.size ** (1 / 3)))
    out = np.zeros(ks ** 3 * (nlevels + 1) + 64, np.float32)
    sides = np.zeros(MAXL, np.int32)
    n = lib().orc_downsampled_stencils(_ptr(st, C.c_float), ks, nlevels, int(normalize), _ptr(out, C.c_float),
                                       _ptr(sides, C.c_int))
    return out[:n].copy(), sides[: max(nlevels, 1)].copy()


def orc_convolve(acc, tree, stencil, parts, reflect=True, use_stencil_ds=True, normalize=False):
    nlev = max(acc.l_max - acc.l_min, 1) if use_stencil_ds else 1
    st, sides = orc_stencils(stencil, nlev, normalize)
    p = np.ascontiguousarray(parts, dtype=np.float32)
    out = np.zeros(acc.P, np.float32)
    stale = C.c_uint64()
    lib().orc_convolve(C.byref(acc.c()), C.byref(tree.c()), _ptr(st, C.c_float), _ptr(sides, C.c_int), len(sides),
                       _ptr(p, C.c_float), _ptr(out, C.c_float), int(reflect), C.byref(stale))
    return out, int(stale.value)


def gradient_stencils(dim, sobel, delta, ndims, nlev):
    """Per-level 3x3x3 stencils (flattened, z-major, y fastest) of
    APRNumerics::gradient_cfd / gradient_sobel (APRNumerics.hpp:165-215):
    the central difference {-1/(2 delta), 0, 1/(2 delta)} along dim, for Sobel
    times {0.25, 0.5, 0.25} along the other axes (APRStencil.hpp:254-299),
    each divided by 2^d for level delta d (rescale_stencil, :135-142).  The
    3x1x1 / 3x3x1 shapes of the reference sit in the middle of the cube with
    zeros around them: zero taps add nothing to the tap sums."""
    f32 = np.float32
    two_d = f32(2) * f32(delta)
    diff = [f32(-1.0) / two_d, f32(0.0), f32(1.0) / two_d]
    smooth = [f32(0.25), f32(0.5), f32(0.25)]
    base = np.zeros((3, 3, 3), np.float32)  # [z][x][y]
    if sobel and ndims == 3:
        bank = [diff if dim == k else smooth for k in range(3)]
        for i in range(3):
            for j in range(3):
                for k in range(3):
                    base[k, j, i] = f32(f32(bank[0][i] * bank[1][j]) * bank[2][k])
    elif sobel and ndims == 2 and dim != 2:
        bank = [diff if dim == k else smooth for k in range(2)]
        for j in range(3):
            for i in range(3):
                base[1, j, i] = f32(bank[0][i] * bank[1][j])
    else:
        for t in range(3):
            idx = [1, 1, 1]
            idx[2 - dim] = t
            base[idx[0], idx[1], idx[2]] = diff[t]
    nlev = max(nlev, 1)
    st = np.concatenate([(base / f32(2.0 ** d)).astype(np.float32).ravel() for d in range(nlev)])
    return st, np.full(nlev, 3, np.int32)


def orc_convolve_stencils(acc, tree, st, sides, parts, reflect=True):
    """orc_convolve with explicit per-level stencils (flattened) and sides."""
    p = np.ascontiguousarray(parts, dtype=np.float32)
    out = np.zeros(acc.P, np.float32)
    stale = C.c_uint64()
    st = np.ascontiguousarray(st, np.float32)
    sides = np.ascontiguousarray(sides, np.int32)
    lib().orc_convolve(C.byref(acc.c()), C.byref(tree.c()), _ptr(st, C.c_float), _ptr(sides, C.c_int), len(sides),
                       _ptr(p, C.c_float), _ptr(out, C.c_float), int(reflect), C.byref(stale))
    return out, int(stale.value)


def orc_gradient(acc, tree, parts, dim=-1, sobel=False, deltas=(1.0, 1.0, 1.0)):
    """gradient_cfd / _sobel of dimension dim, or the gradient magnitude
    (dim < 0: y^2, then + x^2 and + z^2 for axes longer than 1, then sqrtf,
    APRNumerics.hpp:218-287), from the oracle's convolution."""
    nd = sum(1 for v in acc.org if v > 1)
    nlev = acc.l_max - acc.l_min

    def grad(d):
        st, sides = gradient_stencils(d, sobel, deltas[d], nd, nlev)
        return orc_convolve_stencils(acc, tree, st, sides, parts)[0]

    if dim >= 0:
        return grad(dim)
    out = grad(0)
    out = (out * out).astype(np.float32)
    for d in (1, 2):
        if acc.org[d] > 1:
            g = grad(d)
            out = (out + (g * g).astype(np.float32)).astype(np.float32)
    return np.sqrt(out).astype(np.float32)


def orc_richardson_lucy(acc, tree, parts_u16, psf, niter, use_stencil_ds=True, normalize=False, use_double=False,
                        init=None):
    p = np.ascontiguousarray(parts_u16, dtype=np.uint16)
    st = np.ascontiguousarray(psf, dtype=np.float32).ravel()
    ks = int(round(st.size ** (1 / 3)))
    dt = np.float64 if use_double else np.float32
    out = np.ones(acc.P, dt) if init is None else np.ascontiguousarray(init, dtype=dt).copy()
    lib().orc_richardson_lucy(C.byref(acc.c()), C.byref(tree.c()), _ptr(p, C.c_uint16), out.ctypes.data_as(C.c_void_p),
                              _ptr(st, C.c_float), ks, niter, int(use_stencil_ds), int(normalize),
                              int(init is not None), int(use_double))
    return out


# ----------------------------------------------------------------------------- reference (oracle/_ref)

def _ref_access(R, h):
    lmin, lmax = C.c_int(), C.c_int()
    nl, nx, P = C.c_uint64(), C.c_uint64(), C.c_uint64()
    off = C.c_float()
    R.ref_apr_info(h, C.byref(lmin), C.byref(lmax), C.byref(nl), C.byref(nx), C.byref(P), C.byref(off))
    lx = np.zeros(nl.value, np.uint64)
    xe = np.zeros(nx.value, np.uint64)
    yv = np.zeros(max(P.value, 1), np.uint16)
    R.ref_apr_copy(h, _ptr(lx, C.c_uint64), _ptr(xe, C.c_uint64), _ptr(yv, C.c_uint16))
    return lmin.value, lmax.value, lx, xe, yv[: P.value], off.value


class RefAPR:
    """Handle on an APR held by the reference library."""

    def __init__(self, h, shape_zxy, fast=False):
        self.h, self.shape, self.fast = h, shape_zxy, fast
        self.R = ref(fast)

    def __del__(self):
        try:
            self.R.ref_free(self.h)
        except Exception:
            pass

    def access(self):
        lmin, lmax, lx, xe, yv, _ = _ref_access(self.R, self.h)
        z, x, y = self.shape
        a = Access((y, x, z), lmin, lmax, [0] * MAXL, [0] * MAXL, [0] * MAXL, lx, xe, yv)
        ref_geom(a)
        return a

    def offset(self):
        return _ref_access(self.R, self.h)[5]

    def intermediate(self, which):
        z, x, y = self.shape
        a = np.zeros(((z + 1) // 2, (x + 1) // 2, (y + 1) // 2), np.float32)
        assert self.R.ref_copy_intermediate(self.h, which, _ptr(a, C.c_float), a.size) == 0
        return a

    def sample(self, img):
        out = np.zeros(max(self.access().P, 1), np.uint16)
        img = np.ascontiguousarray(img, dtype=np.uint16)
        self.R.ref_sample_image(self.h, _ptr(img, C.c_uint16), _ptr(out, C.c_uint16))
        return out

    def sample_by_block(self, img, z_block, ghost):
        out = np.zeros(max(self.access().P, 1), np.uint16)
        img = np.ascontiguousarray(img, dtype=np.uint16)
        self.R.ref_sample_image_by_block(self.h, _ptr(img, C.c_uint16), z_block, ghost, _ptr(out, C.c_uint16))
        return out

    def tree(self):
        nl, nx, P = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.R.ref_tree_info(self.h, C.byref(nl), C.byref(nx), C.byref(P))
        lx = np.zeros(nl.value, np.uint64)
        xe = np.zeros(nx.value, np.uint64)
        yv = np.zeros(max(P.value, 1), np.uint16)
        self.R.ref_tree_copy(self.h, _ptr(lx, C.c_uint64), _ptr(xe, C.c_uint64), _ptr(yv, C.c_uint16))
        z, x, y = self.shape
        t = Access((y, x, z), 0, len(lx) - 2, [0] * MAXL, [0] * MAXL, [0] * MAXL, lx, xe, yv[: P.value])
        ref_geom(t, tree=True)
        return t

    def tree_mean(self, parts):
        t = self.tree()
        out = np.zeros(max(t.P, 1), np.float32)
        p = np.ascontiguousarray(parts, dtype=np.float32)
        self.R.ref_fill_tree_mean(self.h, _ptr(p, C.c_float), _ptr(out, C.c_float))
        return out[: t.P]

    def convolve(self, stencil, parts, reflect=True, use_stencil_ds=True, normalize=False):
        st = np.ascontiguousarray(stencil, dtype=np.float32).ravel()
        ks = int(round(st.size ** (1 / 3)))
        p = np.ascontiguousarray(parts, dtype=np.float32)
        out = np.zeros(len(p), np.float32)
        self.R.ref_convolve_pencil(self.h, _ptr(st, C.c_float), ks, _ptr(p, C.c_float), _ptr(out, C.c_float),
                                   int(reflect), int(use_stencil_ds), int(normalize))
        return out

    def gradient(self, parts, dim=-1, sobel=False, deltas=(1.0, 1.0, 1.0)):
        """APRNumerics::gradient_cfd / _sobel of dimension dim, or the
        gradient magnitude (dim < 0), computed by the reference itself."""
        p = np.ascontiguousarray(parts, dtype=np.float32)
        out = np.zeros(p.size, np.float32)
        dl = np.ascontiguousarray(deltas, dtype=np.float32)
        self.R.ref_gradient(self.h, _ptr(p, C.c_float), _ptr(out, C.c_float), int(dim), int(sobel),
                            _ptr(dl, C.c_float))
        return out

    def richardson_lucy(self, parts_u16, psf, niter, use_stencil_ds=True, normalize=False, use_double=False,
                        init=None):
        p = np.ascontiguousarray(parts_u16, dtype=np.uint16)
        st = np.ascontiguousarray(psf, dtype=np.float32).ravel()
        ks = int(round(st.size ** (1 / 3)))
        dt = np.float64 if use_double else np.float32
        out = np.ones(len(p), dt) if init is None else np.ascontiguousarray(init, dtype=dt).copy()
        self.R.ref_richardson_lucy(self.h, _ptr(p, C.c_uint16), out.ctypes.data_as(C.c_void_p), _ptr(st, C.c_float),
                                   ks, niter, int(use_stencil_ds), int(normalize), int(init is not None),
                                   int(use_double))
        return out


def ref_geom(a, tree=False):
    """Fills y/x/z_num of an Access from its org dims (GenInfo.hpp:33-98)."""
    import math
    y, x, z = a.org
    md = max(x, y, z)
    lm = math.ceil(math.log2(md))
    if not tree:
        lm = max(1, lm)
        for l in range(1, lm + 1):
            cell = round(2.0 ** (lm - l))
            a.y_num[l], a.x_num[l], a.z_num[l] = (math.ceil(y / cell), math.ceil(x / cell), math.ceil(z / cell))
    else:
        tl = max(lm - 1, 0)
        for l in range(0, tl + 1):
            cell = round(2.0 ** (tl - l + 1))
            a.y_num[l], a.x_num[l], a.z_num[l] = (math.ceil(y / cell), math.ceil(x / cell), math.ceil(z / cell))


def ref_get_apr(img, params, image_type=1, staged=True, fast=False):
    R = ref(fast)
    img = np.ascontiguousarray(img, dtype=np.uint16)
    z, x, y = img.shape
    h = C.c_void_p()
    fn = R.ref_get_apr if staged else R.ref_get_apr_plain
    e = fn(_ptr(img, C.c_uint16), y, x, z, C.byref(params), image_type, C.byref(h))
    if e != 0:
        return e, None
    return 0, RefAPR(h.value, img.shape, fast)


def orc_threshold_li(values, integer_values, fp32_sums):
    """threshold_li restated: float sums in index order (fp32_sums, the
    reference at one OpenMP thread) or double sums (the GPU's)."""
    v = np.ascontiguousarray(values, dtype=np.float32)
    return float(lib().orc_threshold_li(_ptr(v, C.c_float), v.size, int(integer_values), int(fp32_sums)))


def orc_auto_parameters(image, lis, grad, threshold, grad_integer, fp32_sums):
    """autoParametersLiEntropy restated: (grad_th, sigma_th, sub_grad, sub_lis)."""
    im, ls, g = (np.ascontiguousarray(a, dtype=np.float32).ravel() for a in (image, lis, grad))
    n = im.size
    sg, sl = np.zeros(max(n, 1), np.float32), np.zeros(max(n, 1), np.float32)
    gt, st, m = C.c_float(), C.c_float(), C.c_size_t()
    assert lib().orc_auto_parameters(_ptr(im, C.c_float), _ptr(ls, C.c_float), _ptr(g, C.c_float), n, threshold,
                                     int(grad_integer), int(fp32_sums), C.byref(gt), C.byref(st),
                                     _ptr(sg, C.c_float), _ptr(sl, C.c_float), C.byref(m)) == 0
    return gt.value, st.value, sg[: m.value], sl[: m.value]


def ref_threshold_li(values, integer_values, nthreads=1):
    """The reference's threshold_li at nthreads OpenMP threads."""
    v = np.ascontiguousarray(values, dtype=np.float32)
    return float(ref().ref_threshold_li(_ptr(v, C.c_float), v.size, int(integer_values), nthreads))


def ref_auto_parameters(image, lis, grad, Ip_th, bspline_offset, grad_u16, nthreads=1):
    """The reference's autoParametersLiEntropy on ds arrays (z, x, y):
    (grad_th, sigma_th)."""
    im, ls, g = (np.ascontiguousarray(a, dtype=np.float32) for a in (image, lis, grad))
    z, x, y = im.shape
    gt, st = C.c_float(), C.c_float()
    ref().ref_auto_parameters(_ptr(im, C.c_float), _ptr(ls, C.c_float), _ptr(g, C.c_float), y, x, z, int(grad_u16),
                              Ip_th, bspline_offset, nthreads, C.byref(gt), C.byref(st))
    return gt.value, st.value


def ref_get_apr_auto(img, params, image_type=1, nthreads=1):
    """The reference's get_apr with auto_parameters on: (status, RefAPR,
    grad_th, sigma_th)."""
    R = ref()
    img = np.ascontiguousarray(img, dtype=np.uint16)
    z, x, y = img.shape
    h = C.c_void_p()
    gt, st = C.c_float(), C.c_float()
    e = R.ref_get_apr_auto(_ptr(img, C.c_uint16), y, x, z, C.byref(params), image_type, nthreads, C.byref(h),
                           C.byref(gt), C.byref(st))
    if e != 0:
        return e, None, None, None
    return 0, RefAPR(h.value, img.shape), gt.value, st.value


def ref_get_apr_by_block_auto(img, params, image_type, z_block, ghost, nthreads=1):
    """The reference's blocked converter with auto_parameters on: (status,
    RefAPR, grad_th, sigma_th) of the last tile."""
    R = ref()
    img = np.ascontiguousarray(img, dtype=np.uint16)
    z, x, y = img.shape
    h = C.c_void_p()
    gt, st = C.c_float(), C.c_float()
    e = R.ref_get_apr_by_block_auto(_ptr(img, C.c_uint16), y, x, z, C.byref(params), image_type, z_block, ghost,
                                    nthreads, C.byref(h), C.byref(gt), C.byref(st))
    if e != 0:
        return e, None, None, None
    return 0, RefAPR(h.value, img.shape), gt.value, st.value


def ref_get_apr_by_block(img, params, image_type, z_block, ghost, fast=False):
    R = ref(fast)
    img = np.ascontiguousarray(img, dtype=np.uint16)
    z, x, y = img.shape
    h = C.c_void_p()
    e = R.ref_get_apr_by_block(_ptr(img, C.c_uint16), y, x, z, C.byref(params), image_type, z_block, ghost,
                               C.byref(h))
    if e != 0:
        return e, None
    return 0, RefAPR(h.value, img.shape, fast)


def ref_get_apr_custom(grad, lis, shape_zxy, params):
    R = ref()
    z, x, y = shape_zxy
    g = np.ascontiguousarray(grad, dtype=np.float32)
    s = np.ascontiguousarray(lis, dtype=np.float32)
    h = C.c_void_p()
    R.ref_get_apr_custom(_ptr(g, C.c_float), _ptr(s, C.c_float), y, x, z, C.byref(params), C.byref(h))
    return RefAPR(h.value, shape_zxy)


def ref_from_access(acc, shape_zxy):
    R = ref()
    z, x, y = shape_zxy
    h = R.ref_apr_from_arrays(y, x, z, _ptr(acc.level_xz, C.c_uint64), len(acc.level_xz),
                              _ptr(acc.xz_end, C.c_uint64), len(acc.xz_end),
                              _ptr(acc.y_vec if len(acc.y_vec) else np.zeros(1, np.uint16), C.c_uint16), acc.P)
    return RefAPR(h, shape_zxy)


def ref_smooth(img, lambda_, image_type, offset):
    R = ref()
    img = np.ascontiguousarray(img, dtype=np.uint16)
    z, x, y = img.shape
    out = np.zeros(img.shape, np.float32)
    e = R.ref_smooth(_ptr(img, C.c_uint16), y, x, z, lambda_, image_type, offset, _ptr(out, C.c_float))
    return e, out


def block_tiling_in_bounds(shape_zxy, z_block, ghost):
    """True when every z-tile of the blocked converter writes inside every
    level of the particle-cell pyramid and of the APR.  At coarse levels the
    reference maps a tile's planes by integer division of the ghost width, so
    the last tile can reach one plane past the level's end; the reference then
    writes (and its blocked sampling reads) outside the level's arrays."""
    z, x, y = shape_zxy
    L = max(int(math.ceil(math.log2(max(z, x, y)))), 0)
    nb = max(z // z_block, 1)
    for b in range(nb):
        z0 = b * z_block
        zf = z if b == nb - 1 else (b + 1) * z_block
        gl, gr = min(z0, ghost), min(z - zf, ghost)
        pz = zf + gr - (z0 - gl)
        for lf_exp in range(0, L + 1):
            lf = 2 ** lf_exp
            nzp = -(-pz // lf)
            hi = z0 // lf - gl // lf + nzp - gr // lf
            if hi > -(-z // lf):
                return False
    return True

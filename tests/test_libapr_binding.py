"""include/aprb200_libapr.hpp -- the B200 path as a LibAPR build includes it --
compiled against LibAPR's own headers (oracle/_ref/libaprbind.so) and driven
with LibAPR's own objects: get_apr fills the reference's APR, which LibAPR's
LinearIterator then walks; sample_image, convolve_pencil and richardson_lucy
fill the reference's ParticleData; the GPU forms (isotropic_convolve_333/555,
APRNumericsGPU::richardson_lucy) take the APR's own GPUAccessHelper objects.
Everything is compared with the oracle, bit for bit."""
import ctypes as C

import numpy as np
import pytest

from oracle import bind as B
from tests.helpers import gaussian_psf, oracle_params, random_stencil, volume

needs_bind = pytest.mark.skipif(not B.bind_available(), reason="oracle/_ref/libaprbind.so not built")

SYMBOLS = ["bind_get_apr", "bind_free", "bind_particles", "bind_sample", "bind_convolve", "bind_rl",
           "bind_get_apr_by_block", "bind_sample_blocked"]


@needs_bind
def test_binding_library_loads_and_exports_its_entry_points():
    L = B.bind_lib()
    for s in SYMBOLS:
        assert hasattr(L, s)


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Bound:
    def __init__(self, img, image_type, **kw):
        L = B.bind_lib()
        z, x, y = img.shape
        self.h, P, off = C.c_void_p(), C.c_uint64(), C.c_float()
        self.status = L.bind_get_apr(_ptr(img, C.c_uint16), y, x, z, C.byref(oracle_params(**kw)), image_type,
                                     C.byref(self.h), C.byref(P), C.byref(off))
        self.P, self.offset = int(P.value), off.value

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            B.bind_lib().bind_free(self.h)

    def particles(self):
        a = [np.zeros(max(self.P, 1), np.uint16) for _ in range(4)]
        assert B.bind_lib().bind_particles(self.h, *(_ptr(v, C.c_uint16) for v in a)) == 0
        return [v[: self.P].astype(np.int32) for v in a]

    def sample(self, img):
        out = np.zeros(max(self.P, 1), np.uint16)
        assert B.bind_lib().bind_sample(self.h, _ptr(img, C.c_uint16), _ptr(out, C.c_uint16)) == 0
        return out[: self.P]

    def convolve(self, st, parts, gpu_form, reflect=1, ds=1, normalize=0):
        out = np.zeros(max(self.P, 1), np.float32)
        ks = int(round(st.size ** (1 / 3)))
        assert B.bind_lib().bind_convolve(self.h, _ptr(st, C.c_float), ks, _ptr(parts, C.c_float),
                                          _ptr(out, C.c_float), reflect, ds, normalize, gpu_form) == 0
        return out[: self.P]

    def rl(self, raw, psf, niter, gpu_form):
        out = np.zeros(max(self.P, 1), np.float32)
        assert B.bind_lib().bind_rl(self.h, _ptr(raw, C.c_uint16), _ptr(out, C.c_float), _ptr(psf, C.c_float), 5,
                                    niter, gpu_form) == 0
        return out[: self.P]


CASES = [((40, 48, 56), 30, 1, 1), ((33, 65, 31), 20, 6, 0), ((64, 64, 64), 60, 8, 1), ((128, 256, 256), 400, 1, 0)]


@pytest.mark.gpu
@needs_bind
@pytest.mark.parametrize("shape,blobs,seed,image_type", CASES)
def test_get_apr_fills_the_reference_apr(shape, blobs, seed, image_type):
    img = volume(shape, blobs, seed)
    b = Bound(img, image_type)
    assert b.status == 0
    e, acc, (off, _) = B.orc_get_apr(img, oracle_params(), image_type, keep=False)
    assert e == 0 and b.P == acc.P and b.offset == off
    lev, zz, xx, yy = b.particles()  # LibAPR's LinearIterator over the filled APR
    ol, oz, ox, oy = acc.particle_coords()
    assert np.array_equal(lev, ol) and np.array_equal(zz, oz) and np.array_equal(xx, ox) and np.array_equal(yy, oy)
    parts = b.sample(img)
    assert np.array_equal(parts, B.orc_sample(acc, img))
    tree = B.orc_tree(acc)
    pf = parts.astype(np.float32)
    for ks in (3, 5):
        st = random_stencil(ks, 40 + ks)
        ref, stale = B.orc_convolve(acc, tree, st, pf)
        assert stale == 0
        for gpu_form in (0, 1):
            assert np.array_equal(b.convolve(st, pf, gpu_form).view(np.uint32), ref.view(np.uint32)), (ks, gpu_form)
    psf = gaussian_psf()
    ref = B.orc_richardson_lucy(acc, tree, parts, psf, 3)
    for gpu_form in (0, 1):
        assert np.array_equal(b.rl(parts, psf.ravel(), 3, gpu_form).view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
@needs_bind
def test_get_apr_overflow_throws_invalid_argument_like_the_reference():
    img = volume((20, 24, 28), 5, 7)
    img[10, 12, 14] = 65535 - 100
    img[0, 0, 0] = 0
    assert Bound(img, 1).status == 2


@pytest.mark.gpu
@needs_bind
@pytest.mark.parametrize("shape,zb,ghost,image_type", [((100, 40, 48), 32, 8, 1), ((96, 30, 40), 20, 8, 0),
                                                        ((200, 32, 32), 128, 16, 0)])
def test_blocked_converter_and_sampling_fill_the_reference_objects(shape, zb, ghost, image_type):
    """APRConverterBatch::get_apr and ParticleData::sample_parts_from_img_blocked
    through the binding on LibAPR's own objects, against the oracle's blocked
    converter and blocked sampling"""
    L = B.bind_lib()
    img = volume(shape, 30, 3)
    z, x, y = shape
    h, P = C.c_void_p(), C.c_uint64()
    assert L.bind_get_apr_by_block(_ptr(img, C.c_uint16), y, x, z, C.byref(oracle_params()), image_type, zb, ghost,
                                   C.byref(h), C.byref(P)) == 0
    try:
        e, acc = B.orc_get_apr_by_block(img, oracle_params(), image_type, zb, ghost)
        assert e == 0 and int(P.value) == acc.P
        a = [np.zeros(max(acc.P, 1), np.uint16) for _ in range(4)]
        assert L.bind_particles(h, *(_ptr(v, C.c_uint16) for v in a)) == 0
        ol, oz, ox, oy = acc.particle_coords()
        assert all(np.array_equal(v[: acc.P].astype(np.int32), o) for v, o in zip(a, (ol, oz, ox, oy)))
        parts = np.zeros(max(acc.P, 1), np.uint16)
        assert L.bind_sample_blocked(h, _ptr(img, C.c_uint16), zb, ghost, _ptr(parts, C.c_uint16)) == 0
        assert np.array_equal(parts[: acc.P], B.orc_sample_by_block(acc, img, zb, ghost))
    finally:
        L.bind_free(h)

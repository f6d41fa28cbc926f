"""GPU parity of the APR tree, tree means, isotropic 3x3x3 / 5x5x5
convolution and Richardson-Lucy against the CPU oracle, bit-exact."""
import numpy as np
import pytest

import libapr_b200 as A
from oracle import bind as B
from tests.helpers import bits_equal, gaussian_psf, lib_params, oracle_params, random_stencil, volume

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[((40, 48, 56), 30, 1), ((33, 65, 31), 20, 6), ((64, 64, 64), 60, 8)])
def pair(request):
    shape, blobs, seed = request.param
    img = volume(shape, blobs, seed)
    e, acc, _ = B.orc_get_apr(img, oracle_params(), 1)
    conv = A.APRConverter("uint16")
    conv.par = lib_params()
    apr = A.APR()
    assert conv.get_apr(apr, img)
    tr = B.orc_tree(acc)
    parts = B.orc_sample(acc, img)
    return img, acc, tr, apr, parts


def test_tree_structure(pair):
    img, acc, tr, apr, parts = pair
    lx, xe, yv = apr.tree_access()
    assert np.array_equal(lx, tr.level_xz) and np.array_equal(xe, tr.xz_end) and np.array_equal(yv, tr.y_vec)


def test_fill_tree_mean(pair):
    img, acc, tr, apr, parts = pair
    pf = parts.astype(np.float32)
    assert bits_equal(A.APRTreeNumerics.fill_tree_mean(apr, pf), B.orc_tree_mean(acc, tr, pf))


@pytest.mark.parametrize("ks", [3, 5])
@pytest.mark.parametrize("reflect", [True, False])
@pytest.mark.parametrize("ds,normalize", [(True, False), (False, False), (True, True)])
def test_convolve(pair, ks, reflect, ds, normalize):
    img, acc, tr, apr, parts = pair
    st = random_stencil(ks, 100 + ks)
    pf = parts.astype(np.float32)
    ref, stale = B.orc_convolve(acc, tr, st, pf, reflect=reflect, use_stencil_ds=ds, normalize=normalize)
    assert stale == 0
    out = A.APRFilter.convolve_pencil(apr, st, pf, reflect_boundary=reflect, use_stencil_downsample=ds,
                                      normalize=normalize)
    assert bits_equal(out, ref)


def test_richardson_lucy(pair):
    img, acc, tr, apr, parts = pair
    psf = gaussian_psf()
    ref = B.orc_richardson_lucy(acc, tr, parts, psf, 4)
    out = A.APRNumerics.richardson_lucy(apr, parts, None, psf, 4)
    assert bits_equal(out, ref)
    # resume continues from the current estimate (APRNumerics.hpp:559-562)
    po = A.ParticleData(out.copy())
    out2 = A.APRNumerics.richardson_lucy(apr, parts, po, psf, 2, resume=True)
    ref2 = B.orc_richardson_lucy(acc, tr, parts, psf, 2, init=ref)
    assert bits_equal(out2, ref2)


def test_unsupported_psf_size(pair):
    img, acc, tr, apr, parts = pair
    with pytest.raises(RuntimeError):
        A.APRNumerics.richardson_lucy(apr, parts, None, np.ones(49, np.float32) / 49, 1)


def test_richardson_lucy_fp64_bit_exact(pair):
    """The reference's double instantiation on the GPU against the FP64 oracle."""
    img, acc, tr, apr, parts = pair
    psf = gaussian_psf()
    ref = B.orc_richardson_lucy(acc, tr, parts, psf, 3, normalize=True, use_double=True)
    out = A.APRNumerics.richardson_lucy(apr, parts, None, psf, 3, normalize=True, dtype=np.float64)
    assert out.dtype == np.float64
    assert np.array_equal(out.view(np.uint64), ref.view(np.uint64))
    po = A.ParticleData(out.copy())
    out2 = A.APRNumerics.richardson_lucy(apr, parts, po, psf, 2, normalize=True, resume=True)
    ref2 = B.orc_richardson_lucy(acc, tr, parts, psf, 2, normalize=True, use_double=True, init=ref)
    assert np.array_equal(out2.view(np.uint64), ref2.view(np.uint64))


@pytest.mark.parametrize("shape", [(40, 48, 56), (1, 63, 64), (17, 33, 70)])
def test_gradients_match_reference_build(shape):
    """APR gradients (APRNumerics::gradient_cfd / gradient_sobel and the two
    magnitudes, APRNumerics.hpp:165-287) equal the reference's own results
    bit for bit (oracle/_ref, the reference compiled from its headers)."""
    if not B.ref_available():
        pytest.skip("oracle/_ref not built")
    img = volume(shape, 12, 5)
    conv = A.APRConverter("uint16")
    conv.par = lib_params()
    apr = A.APR()
    assert conv.get_apr(apr, img)
    _, r = B.ref_get_apr(img, oracle_params(), 1)
    parts = A.ParticleData().sample_image(apr, img).data.astype(np.float32)
    deltas = (1.0, 0.5, 2.0)
    for dim in (0, 1, 2):
        assert bits_equal(A.APRNumerics.gradient_cfd(apr, parts, dim, deltas[dim]), r.gradient(parts, dim, False, deltas))
        assert bits_equal(A.APRNumerics.gradient_sobel(apr, parts, dim, deltas[dim]), r.gradient(parts, dim, True, deltas))
    assert bits_equal(A.APRNumerics.gradient_magnitude_cfd(apr, parts, deltas), r.gradient(parts, -1, False, deltas))
    assert bits_equal(A.APRNumerics.gradient_magnitude_sobel(apr, parts, deltas), r.gradient(parts, -1, True, deltas))


@pytest.mark.parametrize("ks", [3, 5])
def test_convolve_device_in_place_and_out_of_place(pair, ks):
    """aprb_convolve_device out of place runs the z-streaming kernel; in place
    (input buffer = output buffer) each level's neighbourhood image is built
    before its outputs are written.  Both equal the oracle bit for bit."""
    import ctypes as C

    import torch

    from libapr_b200._lib import check, lib

    img, acc, tr, apr, parts = pair
    st = np.ascontiguousarray(random_stencil(ks, 200 + ks).ravel())
    pf = parts.astype(np.float32)
    ref, stale = B.orc_convolve(acc, tr, st, pf, reflect=True, use_stencil_ds=True, normalize=False)
    assert stale == 0
    d = torch.from_numpy(pf).cuda()
    o = torch.empty_like(d)

    def run(src, dst):
        check(lib().aprb_convolve_device(apr._h, st.ctypes.data_as(C.c_void_p), ks, C.c_void_p(src.data_ptr()),
                                         C.c_void_p(dst.data_ptr()), 1, 1, 0, None))
        torch.cuda.synchronize()

    run(d, o)
    assert bits_equal(o.cpu().numpy(), ref)
    run(d, d)
    assert bits_equal(d.cpu().numpy(), ref)

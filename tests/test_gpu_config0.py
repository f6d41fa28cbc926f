"""The plain get_apr configuration (128x256x256 uint16 volume: background 100,
400 Gaussian blobs sigma U[2,6] px, amplitude U[800,4000], Poisson noise;
lambda=3, E=0.1, Ip_th=0, sigma_th=50, grad_th=10), both ImageTypes, through
the C ABI against the reference's own CPU code (oracle/_ref/libaprref.so,
strict IEEE build) on the same bytes: every intermediate, the linear access
structure, the uint16 intensities, the level decisions and their margins,
the tree means, 3x3x3 and 5x5x5 convolution and Richardson-Lucy on that APR.
The volume comes from the benchmark generator's CPU twin, which the device
generator matches bit for bit (test_gpu_synth.py)."""
import numpy as np
import pytest

import libapr_b200 as A
from oracle import bind as B
from tests.helpers import bits_equal, gaussian_psf, lib_params, oracle_params, random_stencil

pytestmark = pytest.mark.gpu

SHAPE, BLOBS, SIGMA, AMP, BG, SEED = (128, 256, 256), 400, (2.0, 6.0), (800.0, 4000.0), 100.0, 1
REL = 1e-5  # relative margin of a level decision


def level_margins_numpy(grad_applied, scale_applied, l_max, rel, dx=1.0, dy=1.0, dz=1.0, E=0.1):
    """Cells whose computeLevels argument (LocalParticleCellSet.hpp:129-171)
    lies within rel of a power of two 2^k, k >= 1, and cells with argument >= 1."""
    mn = np.float32(min(min(dz, dx), dy))
    mult = np.float32(np.float32(2.0 ** l_max * float(mn)) / np.float32(E))
    q = (grad_applied.astype(np.float32) / scale_applied.astype(np.float32)).astype(np.float32)
    v = (q * mult).astype(np.float32).astype(np.float64)
    act = v >= 1.0
    m, e = np.frexp(v[act])
    lo, hi = np.ldexp(1.0, e - 1), np.ldexp(1.0, e)
    near = ((e - 1 >= 1) & (v[act] - lo <= rel * lo)) | (hi - v[act] <= rel * hi)
    return int(near.sum()), int(act.sum())


@pytest.fixture(scope="module")
def img():
    return B.blob_volume_cpu(SHAPE, BLOBS, SIGMA, AMP, BG, SEED)


@pytest.fixture(scope="module", params=[1, 0], ids=["uint16", "float"])
def pair(request, img):
    it = request.param
    e, ref = B.ref_get_apr(img, oracle_params(), it, staged=True)
    conv = A.APRConverter("uint16" if it == 1 else "float")
    conv.par = lib_params()
    conv.keep_intermediates(True)
    apr = A.APR()
    if e == 2:  # the reference's uint16 overflow check threw: the GPU must refuse too
        with pytest.raises(ValueError):
            conv.get_apr(apr, img)
        pytest.skip("the reference's uint16 B-spline overflow check throws on this volume")
    assert e == 0
    assert conv.get_apr(apr, img)
    return it, ref, conv, apr


def test_intermediates(pair, img):
    it, ref, conv, apr = pair
    ds = ref.intermediate(1).shape
    assert apr.bspline_offset() == ref.offset()
    e, sm = B.ref_smooth(img, 3.0, it, ref.offset())
    assert e == 0 and bits_equal(conv.intermediate(0, SHAPE), sm), "smoothed image"
    for w in range(1, 7):
        assert bits_equal(conv.intermediate(w, ds), ref.intermediate(w)), "stage %d" % w


def test_structure_and_intensities(pair, img):
    it, ref, conv, apr = pair
    acc = ref.access()
    lx, xe, yv = apr.linear_access()
    assert np.array_equal(lx, acc.level_xz)
    assert np.array_equal(xe, acc.xz_end)
    assert np.array_equal(yv, acc.y_vec)
    assert apr.total_number_particles() == acc.P
    parts = A.ParticleData().sample_image(apr, img).data
    assert np.array_equal(parts, ref.sample(img)[: acc.P])


def test_level_decisions_and_margins(pair):
    """No level flips (the GPU's levels are the reference's), and the number
    of cells within 1e-5 of a level boundary, counted on the GPU, equals the
    count from the reference's own gradient and scale."""
    it, ref, conv, apr = pair
    ds = ref.intermediate(1).shape
    flips = int(np.count_nonzero(conv.intermediate(6, ds) != ref.intermediate(6)))
    assert flips == 0
    near, active = conv.level_margins(REL)
    acc = ref.access()
    assert (near, active) == level_margins_numpy(ref.intermediate(4), ref.intermediate(5), acc.l_max, REL)
    assert active > 0


def test_tree_conv_rl(pair, img):
    it, ref, conv, apr = pair
    acc = ref.access()
    parts = ref.sample(img)[: acc.P]
    pf = parts.astype(np.float32)
    assert bits_equal(A.APRTreeNumerics.fill_tree_mean(apr, pf), ref.tree_mean(pf))
    for ks in (3, 5):
        st = random_stencil(ks, 7 + ks)
        out = A.APRFilter.convolve_pencil(apr, st, pf)
        assert bits_equal(out, ref.convolve(st, pf)), "conv %d^3" % ks
    psf = gaussian_psf()
    out = A.APRNumerics.richardson_lucy(apr, parts, None, psf, 3)
    assert bits_equal(out, ref.richardson_lucy(parts, psf, 3))

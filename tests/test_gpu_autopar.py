"""GPU automatic parameters (threshold_li, autoParametersLiEntropy and
get_apr with auto_parameters on) against the oracle.

The GPU sums in FP64 in a fixed order; its thresholds equal the oracle's
FP64-sum restatement, and lie within LI_REL_TOL of the reference build's
FP32-sum thresholds.  Given the same thresholds the APR is bit-exact."""
import numpy as np
import pytest

import libapr_b200 as A
from oracle import bind as B
from tests.helpers import lib_params, oracle_params, volume
from tests.test_oracle_autopar import LI_REL_TOL, VECTORS, ref_missing

pytestmark = pytest.mark.gpu


def f32_equal(a, b):
    return np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32)


@pytest.mark.parametrize("name,v,integer", VECTORS, ids=[n for n, _, _ in VECTORS])
def test_threshold_li(name, v, integer):
    g = A.threshold_li(v, integer)
    assert f32_equal(g, B.orc_threshold_li(v, integer, fp32_sums=False)), (g, B.orc_threshold_li(v, integer, False))
    r = B.orc_threshold_li(v, integer, fp32_sums=True)
    assert abs(g - r) <= LI_REL_TOL * abs(r) + 1e-30


@pytest.mark.parametrize("grad_integer", [True, False])
@pytest.mark.parametrize("shape,frac", [((64, 80, 96), 0.6), ((300, 300, 190), 0.99)])
def test_auto_parameters_arrays(grad_integer, shape, frac):
    """Foreground compaction, the stride above 32*512*512 foreground cells, and
    both thresholds."""
    rng = np.random.default_rng(11)
    ids = rng.uniform(0, 100, shape).astype(np.float32)
    grad = rng.gamma(2.0, 20.0, shape).astype(np.float32)
    if grad_integer:
        grad = np.floor(grad)
    lis = rng.gamma(3.0, 10.0, shape).astype(np.float32)
    par = A.APRParameters(Ip_th=95.0 - 100.0 * frac)
    off = 5.0
    A.auto_parameters_li_entropy(par, ids, lis, grad, off, grad_integer)
    thr = np.float32(np.float32(par.Ip_th) + np.float32(off))
    eg, es, _, _ = B.orc_auto_parameters(ids, lis, grad, thr, grad_integer, fp32_sums=False)
    assert f32_equal(par.grad_th, eg) and f32_equal(par.sigma_th, es), (par.grad_th, eg, par.sigma_th, es)


def test_auto_parameters_without_foreground():
    z = np.zeros((8, 9, 10), np.float32)
    par = A.APRParameters(Ip_th=1.0, grad_th=7.0, sigma_th=9.0)
    A.auto_parameters_li_entropy(par, z, z + 1, z + 2, 0.0, True)
    assert (par.grad_th, par.sigma_th) == (0.0, 0.0)


CASES = [((40, 48, 56), 1, 0.0), ((33, 65, 31), 6, 150.0), ((96, 100, 64), 4, 0.0)]


@pytest.mark.parametrize("image_type", ["uint16", "float"])
@pytest.mark.parametrize("shape,seed,Ip_th", CASES)
def test_get_apr_auto_parameters(image_type, shape, seed, Ip_th):
    """get_apr with auto_parameters: the thresholds are the oracle's (FP64
    sums on the pipeline's ds arrays), the APR is the oracle's APR built with
    those thresholds, and the converter's par holds them afterwards."""
    it = 1 if image_type == "uint16" else 0
    img = volume(shape, 30, seed)
    e, _, (off, inter) = B.orc_get_apr(img, oracle_params(Ip_th=Ip_th), it)
    assert e == 0
    thr = np.float32(np.float32(Ip_th) + np.float32(off))
    eg, es, _, _ = B.orc_auto_parameters(inter[2], inter[3], inter[1], thr, it == 1, fp32_sums=False)

    conv = A.APRConverter(image_type)
    conv.par = lib_params(Ip_th=Ip_th, auto_parameters=True)
    apr = A.APR()
    assert conv.get_apr(apr, img)
    used = apr.get_apr_parameters()
    assert used.auto_parameters
    assert f32_equal(used.grad_th, eg) and f32_equal(used.sigma_th, es), (used.grad_th, eg, used.sigma_th, es)
    assert f32_equal(conv.par.grad_th, eg) and f32_equal(conv.par.sigma_th, es)

    e, acc, _ = B.orc_get_apr(img, oracle_params(Ip_th=Ip_th, grad_th=float(eg), sigma_th=float(es)), it,
                              keep=False)
    lx, xe, yv = apr.linear_access()
    assert np.array_equal(lx, acc.level_xz) and np.array_equal(xe, acc.xz_end) and np.array_equal(yv, acc.y_vec)


@ref_missing
@pytest.mark.parametrize("image_type", ["uint16", "float"])
def test_get_apr_auto_parameters_near_reference(image_type):
    it = 1 if image_type == "uint16" else 0
    img = volume((96, 100, 64), 30, 4)
    e, _, rg, rs = B.ref_get_apr_auto(img, oracle_params(), it, nthreads=4)
    assert e == 0
    conv = A.APRConverter(image_type)
    conv.par = lib_params(auto_parameters=True)
    apr = A.APR()
    assert conv.get_apr(apr, img)
    used = apr.get_apr_parameters()
    assert abs(used.grad_th - rg) <= LI_REL_TOL * abs(rg) and abs(used.sigma_th - rs) <= LI_REL_TOL * abs(rs)


def test_blocked_converter_auto_parameters():
    """One tile: the blocked converter chooses get_apr's thresholds and APR;
    several tiles: each tile chooses its own, the APR and the converter's par
    keep the last tile's (APRConverterBatch.hpp:243-247)."""
    img = volume((64, 72, 80), 30, 9)
    conv = A.APRConverter("uint16")
    conv.par = lib_params(auto_parameters=True)
    apr = A.APR()
    assert conv.get_apr(apr, img)
    one = A.APRConverterBatch("uint16", z_block_size=128, ghost_z=32)
    one.par = lib_params(auto_parameters=True)
    apr1 = A.APR()
    assert one.get_apr(apr1, img)
    a, b = apr.get_apr_parameters(), apr1.get_apr_parameters()
    assert f32_equal(a.grad_th, b.grad_th) and f32_equal(a.sigma_th, b.sigma_th)
    for x, y in zip(apr.linear_access(), apr1.linear_access()):
        assert np.array_equal(x, y)
    many = A.APRConverterBatch("uint16", z_block_size=16, ghost_z=8)
    many.par = lib_params(auto_parameters=True)
    apr2 = A.APR()
    assert many.get_apr(apr2, img)
    c = apr2.get_apr_parameters()
    assert c.grad_th > 0 and c.sigma_th > 0
    assert f32_equal(many.par.grad_th, c.grad_th) and f32_equal(many.par.sigma_th, c.sigma_th)


@ref_missing
@pytest.mark.parametrize("shape,z_block,ghost", [((64, 72, 80), 24, 8), ((60, 64, 64), 16, 4)])
def test_blocked_converter_auto_parameters_near_reference(shape, z_block, ghost):
    """Per-tile automatic parameters of the blocked converter against the
    reference's APRConverterBatch with auto_parameters on: the last tile's
    thresholds, which both APRs keep (tilings the reference keeps in bounds)."""
    assert B.block_tiling_in_bounds(shape, z_block, ghost)
    img = volume(shape, 30, 9)
    e, _, rg, rs = B.ref_get_apr_by_block_auto(img, oracle_params(), 1, z_block, ghost, nthreads=1)
    assert e == 0
    conv = A.APRConverterBatch("uint16", z_block_size=z_block, ghost_z=ghost)
    conv.par = lib_params(auto_parameters=True)
    apr = A.APR()
    assert conv.get_apr(apr, img)
    used = apr.get_apr_parameters()
    assert abs(used.grad_th - rg) <= LI_REL_TOL * abs(rg) and abs(used.sigma_th - rs) <= LI_REL_TOL * abs(rs), \
        (used.grad_th, rg, used.sigma_th, rs)

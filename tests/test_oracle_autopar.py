"""The oracle's automatic parameters (threshold_li, autoParametersLiEntropy,
src/algorithm/AutoParameters.hpp) pinned against the reference build.

With float sums in index order the restatement is the reference at one OpenMP
thread, bit for bit.  With FP64 sums (the GPU's definition) it differs from
the reference by the reference's own FP32 rounding, which also moves the
reference's answer when its thread count changes; that gap is bounded here by
LI_REL_TOL."""
import numpy as np
import pytest

from oracle import bind as B
from tests.helpers import oracle_params, volume

ref_missing = pytest.mark.skipif(not B.ref_available(), reason="oracle/_ref not built (needs the LibAPR tree)")

# relative gap allowed between FP64-sum thresholds and the reference's FP32 sums
LI_REL_TOL = 1e-3


def li_vectors():
    rng = np.random.default_rng(7)
    out = []
    for n in (10, 1000, 200_000):
        out.append(("gamma_f%d" % n, rng.gamma(2.0, 3.0, n).astype(np.float32), False))
        out.append(("gamma_u%d" % n, np.floor(rng.gamma(2.0, 30.0, n)).astype(np.float32), True))
    bi = np.concatenate([rng.normal(10, 2, 50_000), rng.normal(200, 30, 5_000)]).clip(0).astype(np.float32)
    out.append(("bimodal_f", bi, False))
    out.append(("bimodal_u", np.floor(bi), True))
    # integer input whose mean is below 1: the initial value is raised (:74-78)
    low = np.zeros(10_000, np.float32)
    low[:300] = 1
    low[:40] = 3
    out.append(("low_u", low, True))
    # every value at or below the threshold is 0: mean_back == 0 (:89-92)
    z = np.concatenate([np.zeros(500), rng.uniform(5, 9, 100)]).astype(np.float32)
    out.append(("zero_back_f", z, False))
    out.append(("constant_f", np.full(77, 4.25, np.float32), False))
    out.append(("constant_u", np.full(77, 12, np.float32), True))
    out.append(("empty_f", np.zeros(0, np.float32), False))
    return out


VECTORS = li_vectors()


@ref_missing
@pytest.mark.parametrize("name,v,integer", VECTORS, ids=[n for n, _, _ in VECTORS])
def test_threshold_li_fp32_sums_match_reference_bitwise(name, v, integer):
    r = B.ref_threshold_li(v, integer, nthreads=1)
    o = B.orc_threshold_li(v, integer, fp32_sums=True)
    assert np.float32(r).view(np.uint32) == np.float32(o).view(np.uint32), (r, o)


@ref_missing
@pytest.mark.parametrize("name,v,integer", VECTORS, ids=[n for n, _, _ in VECTORS])
def test_threshold_li_fp64_sums_near_reference(name, v, integer):
    o = B.orc_threshold_li(v, integer, fp32_sums=False)
    for nt in (1, 4):
        r = B.ref_threshold_li(v, integer, nthreads=nt)
        assert abs(o - r) <= LI_REL_TOL * abs(r) + 1e-30, (nt, r, o)


def test_threshold_li_edge_values():
    assert B.orc_threshold_li(np.zeros(0, np.float32), False, False) == 0.0
    assert B.orc_threshold_li(np.full(5, 3.5, np.float32), False, False) == 3.5
    # two separated clusters: the threshold falls between them
    v = np.concatenate([np.full(100, 10.0), np.full(100, 100.0)]).astype(np.float32)
    t = B.orc_threshold_li(v, False, False)
    assert 10.0 < t < 100.0


def _intermediates(shape, seed, image_type):
    img = volume(shape, 30, seed)
    e, acc, (off, inter) = B.orc_get_apr(img, oracle_params(), image_type)
    assert e == 0
    return img, off, inter


@ref_missing
@pytest.mark.parametrize("image_type", [1, 0])
@pytest.mark.parametrize("shape,seed,Ip_th", [((40, 48, 56), 1, 0.0), ((33, 65, 31), 6, 150.0)])
def test_auto_parameters_restatement_matches_reference(image_type, shape, seed, Ip_th):
    """orc_auto_parameters on the pipeline's ds arrays == the reference's
    autoParametersLiEntropy on the same arrays (one thread), and == the
    thresholds the reference's own get_apr chooses with auto_parameters on."""
    img, off, inter = _intermediates(shape, seed, image_type)
    grad, ids, lis = inter[1], inter[2], inter[3]
    integer = image_type == 1
    thr = np.float32(np.float32(Ip_th) + np.float32(off))
    g32, s32, _, _ = B.orc_auto_parameters(ids, lis, grad, thr, integer, fp32_sums=True)
    rg, rs = B.ref_auto_parameters(ids, lis, grad, Ip_th, off, integer, nthreads=1)
    assert (np.float32(g32), np.float32(s32)) == (np.float32(rg), np.float32(rs))
    e, _, ag, as_ = B.ref_get_apr_auto(img, oracle_params(Ip_th=Ip_th), image_type, nthreads=1)
    assert e == 0
    assert (np.float32(ag), np.float32(as_)) == (np.float32(g32), np.float32(s32))
    g64, s64, _, _ = B.orc_auto_parameters(ids, lis, grad, thr, integer, fp32_sums=False)
    assert abs(g64 - rg) <= LI_REL_TOL * abs(rg) and abs(s64 - rs) <= LI_REL_TOL * abs(rs)


@ref_missing
def test_auto_parameters_subsample_stride_matches_reference():
    """More than 32*512*512 foreground cells: the reference keeps every
    (n_fg // 32*512*512)-th one (:139-147)."""
    rng = np.random.default_rng(3)
    shape = (300, 300, 190)  # 17.1M cells, about 16.9M foreground
    ids = rng.uniform(0, 100, shape).astype(np.float32)
    grad = np.floor(rng.gamma(2.0, 20.0, shape)).astype(np.float32)
    lis = rng.gamma(3.0, 10.0, shape).astype(np.float32)
    g32, s32, sg, sl = B.orc_auto_parameters(ids, lis, grad, np.float32(1.0), True, fp32_sums=True)
    fg = ids.ravel() > np.float32(1.0)
    nf = int(fg.sum())
    m = min(32 * 512 * 512, nf)
    delta = nf // m
    assert delta == 2 and len(sg) == m
    assert np.array_equal(sg, grad.ravel()[fg][: m * delta: delta])
    assert np.array_equal(sl, lis.ravel()[fg][: m * delta: delta])
    rg, rs = B.ref_auto_parameters(ids, lis, grad, 1.0, 0.0, True, nthreads=1)
    assert (np.float32(g32), np.float32(s32)) == (np.float32(rg), np.float32(rs))


def test_auto_parameters_without_foreground():
    z = np.zeros((4, 5, 6), np.float32)
    g, s, sg, sl = B.orc_auto_parameters(z, z + 1, z + 2, np.float32(0.5), True, fp32_sums=False)
    assert (g, s, len(sg)) == (0.0, 0.0, 0)

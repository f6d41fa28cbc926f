"""Pins the CPU oracle (oracle/apr_oracle.c) against the reference's golden
fixtures (tests/golden, built by tests/golden/make_golden.py from LibAPR's
test/files) and, where oracle/_ref was built, against the reference's own CPU
code on seeded synthetic volumes."""
import os

import numpy as np
import pytest

from oracle import bind as B
from tests.helpers import bits_equal, gaussian_psf, oracle_params, random_stencil, volume

CASES = ["sphere_diff_dims", "sphere_120", "sphere_2D", "sphere_1D"]


def load(golden_dir, case):
    return np.load(os.path.join(golden_dir, case + ".npz"))


def case_params(d):
    lam, E, gth, sth, sthm = [float(v) for v in d["params"]]
    # test_pipeline_u16 (test/APRTest.cpp:2779-2790): sigma thresholds floored at 0.1
    return B.make_params(lambda_=lam, rel_error=E, grad_th=gth, sigma_th=max(sth, 0.1), sigma_th_max=max(sthm, 0.1))


@pytest.mark.parametrize("case", CASES)
def test_gradient_and_scale_match_saved(golden_dir, case):
    """gradient_step / local_intensity_scale_step vs the saved TIFFs at
    tolerance 1 (test/APRTest.cpp:2806-2813)."""
    d = load(golden_dir, case)
    e, acc, (off, inter) = B.orc_get_apr(d["original"], case_params(d), 1)
    assert e == 0
    assert np.abs(inter[1] - d["gradient_saved"].astype(np.float32)).max() <= 1
    assert np.abs(inter[3] - d["scale_saved"]).max() <= 1


@pytest.mark.parametrize("case", CASES)
def test_structure_from_saved_grad_scale(golden_dir, case):
    """get_apr_custom_grad_scale on the saved gradient/scale reproduces the
    stored APR: particle count, and each particle's level / x / y / z and its
    sampled intensity at its nearest pixel (test/APRTest.cpp:2600-2665,
    2815-2837)."""
    d = load(golden_dir, case)
    img = d["original"]
    acc = B.orc_get_apr_custom(d["gradient_saved"].astype(np.float32), d["scale_saved"], img.shape, case_params(d))
    assert acc.P == int(d["total_number_particles"][0])
    lev, zz, xx, yy = acc.particle_coords()
    size = 2 ** (acc.l_max - lev)
    Z, X, Y = img.shape
    yp, xp, zp = [np.floor((c + 0.5) * size).astype(np.int64) for c in (yy, xx, zz)]
    ok = (yp < Y) & (xp < X) & (zp < Z)
    parts = B.orc_sample(acc, img)
    for name, val in [("level", lev), ("x", xx), ("y", yy), ("z", zz), ("pc", parts)]:
        ref = d["img_" + name][zp[ok], xp[ok], yp[ok]]
        assert np.array_equal(ref.astype(np.int64), val[ok].astype(np.int64)), name


@pytest.mark.parametrize("case", CASES)
def test_reconstruction_matches_saved_images(golden_dir, case):
    """reconstruct_level and reconstruct_constant of the stored APR are the
    reference's per-pixel level and piecewise-constant images
    (APRReconstruction.hpp:80, 132; the fixtures of test/APRTest.cpp:2600-2665)."""
    d = load(golden_dir, case)
    img = d["original"]
    acc = B.orc_get_apr_custom(d["gradient_saved"].astype(np.float32), d["scale_saved"], img.shape, case_params(d))
    assert np.array_equal(B.orc_reconstruct(acc).astype(np.uint16), d["img_level"])
    assert np.array_equal(B.orc_reconstruct(acc, B.orc_sample(acc, img)), d["img_pc"])


ref_missing = pytest.mark.skipif(not B.ref_available(), reason="oracle/_ref not built (needs the LibAPR tree)")


@ref_missing
@pytest.mark.parametrize("image_type", [1, 0])
@pytest.mark.parametrize("shape,blobs,seed", [((40, 48, 56), 30, 1), ((17, 33, 70), 12, 2), ((5, 64, 9), 4, 3),
                                              ((1, 63, 64), 6, 4), ((1, 1, 100), 2, 5)])
def test_oracle_matches_reference_build(shape, blobs, seed, image_type):
    img = volume(shape, blobs, seed)
    p = oracle_params()
    e, acc, (off, inter) = B.orc_get_apr(img, p, image_type)
    e2, r = B.ref_get_apr(img, p, image_type)
    assert e == e2 == 0
    ra = r.access()
    assert np.array_equal(acc.xz_end, ra.xz_end) and np.array_equal(acc.y_vec, ra.y_vec)
    assert off == r.offset()
    for w in range(1, 7):
        assert bits_equal(inter[w], r.intermediate(w)), w
    assert np.array_equal(B.orc_sample(acc, img), r.sample(img))


@ref_missing
def test_oracle_filters_match_reference_build():
    img = volume((40, 48, 56), 30, 1)
    e, acc, _ = B.orc_get_apr(img, oracle_params(), 1)
    _, r = B.ref_get_apr(img, oracle_params(), 1)
    tr, rt = B.orc_tree(acc), r.tree()
    assert np.array_equal(tr.xz_end, rt.xz_end) and np.array_equal(tr.y_vec, rt.y_vec)
    parts = B.orc_sample(acc, img).astype(np.float32)
    assert bits_equal(B.orc_tree_mean(acc, tr, parts), r.tree_mean(parts))
    for ks in (3, 5):
        st = random_stencil(ks, 10 + ks)
        for reflect in (True, False):
            o, stale = B.orc_convolve(acc, tr, st, parts, reflect=reflect)
            assert stale == 0
            assert bits_equal(o, r.convolve(st, parts, reflect=reflect))
    pu = B.orc_sample(acc, img)
    psf = gaussian_psf()
    assert bits_equal(B.orc_richardson_lucy(acc, tr, pu, psf, 3), r.richardson_lucy(pu, psf, 3))
    o64 = B.orc_richardson_lucy(acc, tr, pu, psf, 2, use_double=True)
    assert np.array_equal(o64, r.richardson_lucy(pu, psf, 2, use_double=True))


@ref_missing
@pytest.mark.parametrize("shape", [(40, 48, 56), (1, 63, 64), (17, 33, 70)])
def test_oracle_gradients_match_reference_build(shape):
    """APRNumerics::gradient_cfd / gradient_sobel and the two gradient
    magnitudes (APRNumerics.hpp:165-287), computed by the oracle convolution
    with the reference's 1-D / 2-D stencils embedded in 3x3x3 cubes, equal the
    reference's own results bit for bit."""
    img = volume(shape, 12, 5)
    e, acc, _ = B.orc_get_apr(img, oracle_params(), 1)
    _, r = B.ref_get_apr(img, oracle_params(), 1)
    tr = B.orc_tree(acc)
    parts = B.orc_sample(acc, img).astype(np.float32)
    deltas = (1.0, 0.5, 2.0)
    for sobel in (False, True):
        for dim in (0, 1, 2):
            assert bits_equal(B.orc_gradient(acc, tr, parts, dim, sobel, deltas), r.gradient(parts, dim, sobel, deltas))
        assert bits_equal(B.orc_gradient(acc, tr, parts, -1, sobel, deltas), r.gradient(parts, -1, sobel, deltas))


@ref_missing
def test_overflow_detected_like_reference():
    """test_u16_overflow_detection (test/APRTest.cpp:2850-2867)."""
    img = volume((20, 24, 28), 5, 7)
    img[10, 12, 14] = 65535 - 100
    img[0, 0, 0] = 0
    e, _, _ = B.orc_get_apr(img, oracle_params(), 1)
    e2, _ = B.ref_get_apr(img, oracle_params(), 1)
    assert e == 2 and e2 == 2


# z-tilings of the blocked converter, all inside every level (the reference
# writes outside a level's array for tilings that fail block_tiling_in_bounds)
BLOCK_CASES = [((100, 40, 48), 32, 8), ((96, 30, 40), 20, 8), ((65, 37, 29), 16, 4), ((200, 32, 32), 128, 16),
               ((80, 24, 70), 16, 16), ((64, 40, 30), 128, 32)]


@pytest.mark.parametrize("shape,zb,ghost", BLOCK_CASES)
def test_block_cases_stay_in_bounds(shape, zb, ghost):
    assert B.block_tiling_in_bounds(shape, zb, ghost)


def test_block_bounds_predicate_flags_overrun():
    # 70 planes in tiles of 16 with ghost 4: the last tile reaches plane 9 of
    # a 9-plane level at 1/8 resolution
    assert not B.block_tiling_in_bounds((70, 33, 50), 16, 4)


@ref_missing
@pytest.mark.parametrize("image_type", [1, 0])
@pytest.mark.parametrize("shape,zb,ghost", BLOCK_CASES[:4])
def test_block_oracle_matches_reference_build(shape, zb, ghost, image_type):
    img = volume(shape, 30, 3)
    p = oracle_params()
    e, acc = B.orc_get_apr_by_block(img, p, image_type, zb, ghost)
    e2, r = B.ref_get_apr_by_block(img, p, image_type, zb, ghost)
    assert e == e2 == 0
    ra = r.access()
    assert np.array_equal(acc.level_xz, ra.level_xz)
    assert np.array_equal(acc.xz_end, ra.xz_end) and np.array_equal(acc.y_vec, ra.y_vec)
    assert np.array_equal(B.orc_sample_by_block(acc, img, zb, ghost), r.sample_by_block(img, zb, ghost)[:ra.P])

"""GPU parity of get_apr and sample_image, through the C ABI, against the CPU
oracle (bit-exact structure, intermediates and uint16 intensities) and against
the reference's golden fixtures."""
import os

import numpy as np
import pytest

import libapr_b200 as A
from oracle import bind as B
from tests.helpers import bits_equal, lib_params, oracle_params, volume

pytestmark = pytest.mark.gpu

STAGE_SHAPE_DS = lambda s: ((s[0] + 1) // 2, (s[1] + 1) // 2, (s[2] + 1) // 2)

SHAPES = [((40, 48, 56), 30, 1), ((17, 33, 70), 12, 2), ((5, 64, 9), 4, 3), ((33, 65, 31), 20, 6),
          ((1, 63, 64), 6, 4), ((1, 1, 100), 2, 5), ((64, 64, 64), 60, 8)]


def gpu_apr(img, image_type, **kw):
    conv = A.APRConverter("uint16" if image_type == 1 else "float")
    conv.par = lib_params(**kw)
    conv.keep_intermediates(True)
    apr = A.APR()
    assert conv.get_apr(apr, img)
    return conv, apr


@pytest.mark.parametrize("image_type", [1, 0])
@pytest.mark.parametrize("shape,blobs,seed", SHAPES)
def test_get_apr_bit_exact(shape, blobs, seed, image_type):
    img = volume(shape, blobs, seed)
    e, acc, (off, inter) = B.orc_get_apr(img, oracle_params(), image_type)
    assert e == 0
    conv, apr = gpu_apr(img, image_type)
    ds = STAGE_SHAPE_DS(shape)
    assert apr.bspline_offset() == off
    assert bits_equal(conv.intermediate(0, shape), inter[0]), "smoothed image"
    for w in range(1, 7):
        assert bits_equal(conv.intermediate(w, ds), inter[w]), "stage %d" % w
    lx, xe, yv = apr.linear_access()
    assert np.array_equal(lx, acc.level_xz)
    assert np.array_equal(xe, acc.xz_end)
    assert np.array_equal(yv, acc.y_vec)
    parts = A.ParticleData().sample_image(apr, img).data
    assert np.array_equal(parts, B.orc_sample(acc, img))


# shapes that take the TMA-staged smoothing (float ImageType): x / z passes
# with y_num a multiple of 4 and >= 256 and >= 16 samples along the axis --
# partial TMA boxes (y_num 600, 260), partial 16-sample segments, an x extent
# below 16 that keeps the register-staged x pass; the y pass with y_num a
# multiple of 8 and >= 64 and >= 32 lines -- one tile (64), a last tile of 8
# or 24 samples (72, 600), line counts that are not multiples of 32; the
# inverse B-spline with a ds y extent that is a multiple of 4 and >= 256 and
# an x extent >= 18 (600, 520: two y blocks, two x blocks, two z runs)
TMA_SHAPES = [((37, 45, 600), 25, 21), ((16, 300, 260), 30, 22), ((130, 17, 512), 40, 23), ((20, 9, 256), 6, 24),
              ((7, 11, 72), 4, 25), ((9, 5, 64), 3, 26), ((33, 40, 136), 12, 27), ((70, 40, 520), 30, 28)]


@pytest.mark.parametrize("shape,blobs,seed", TMA_SHAPES)
@pytest.mark.parametrize("lam", [3.0, 0.5, 10.0])
def test_tma_smoothing_bit_exact(shape, blobs, seed, lam):
    img = volume(shape, blobs, seed)
    e, acc, (off, inter) = B.orc_get_apr(img, oracle_params(lambda_=lam), 0)
    assert e == 0
    conv, apr = gpu_apr(img, 0, lambda_=lam)
    assert bits_equal(conv.intermediate(0, shape), inter[0]), "smoothed image"
    for w in range(1, 7):  # the TMA-staged inverse B-spline writes stage 2 where the ds image allows
        assert bits_equal(conv.intermediate(w, STAGE_SHAPE_DS(shape)), inter[w]), "stage %d" % w
    lx, xe, yv = apr.linear_access()
    assert np.array_equal(xe, acc.xz_end) and np.array_equal(yv, acc.y_vec)


@pytest.mark.parametrize("kw", [dict(lambda_=0.5), dict(lambda_=10.0), dict(sigma_th=0.0, grad_th=0.0),
                                dict(neighborhood_optimization=False), dict(Ip_th=150.0, rel_error=0.05),
                                dict(constant_intensity_scale=True), dict(lambda_=0.0),
                                dict(dx=0.5, dy=0.25, dz=2.0), dict(dx=0.7, dy=1.3, dz=1.0)])
def test_get_apr_parameter_variants(kw):
    img = volume((24, 40, 36), 10, 11)
    e, acc, (off, inter) = B.orc_get_apr(img, oracle_params(**kw), 1)
    assert e == 0
    conv, apr = gpu_apr(img, 1, **kw)
    lx, xe, yv = apr.linear_access()
    assert np.array_equal(xe, acc.xz_end) and np.array_equal(yv, acc.y_vec)
    for w in range(1, 7):
        assert bits_equal(conv.intermediate(w, STAGE_SHAPE_DS(img.shape)), inter[w]), w


@pytest.mark.parametrize("case", ["sphere_diff_dims", "sphere_120", "sphere_2D", "sphere_1D"])
def test_golden_spheres(golden_dir, case):
    d = np.load(os.path.join(golden_dir, case + ".npz"))
    lam, E, gth, sth, sthm = [float(v) for v in d["params"]]
    img = d["original"]
    conv, apr = gpu_apr(img, 1, lambda_=lam, rel_error=E, grad_th=gth, sigma_th=max(sth, 0.1),
                        sigma_th_max=max(sthm, 0.1), Ip_th=0.0)
    ds = STAGE_SHAPE_DS(img.shape)
    assert np.abs(conv.intermediate(1, ds) - d["gradient_saved"].astype(np.float32)).max() <= 1
    assert np.abs(conv.intermediate(3, ds) - d["scale_saved"]).max() <= 1
    assert apr.total_number_particles() == int(d["total_number_particles"][0])


def test_overflow_raises_value_error():
    img = volume((20, 24, 28), 5, 7)
    img[10, 12, 14] = 65535 - 100
    img[0, 0, 0] = 0
    conv = A.APRConverter("uint16")
    conv.par = lib_params()
    with pytest.raises(ValueError):
        conv.get_apr(A.APR(), img)
    # float ImageType has no overflow check
    conv = A.APRConverter("float")
    conv.par = lib_params()
    assert conv.get_apr(A.APR(), img)


def test_dimension_check():
    conv = A.APRConverter("uint16")
    conv.par = lib_params(check_input=True)
    img = volume((40, 1, 1), 2, 3)  # data along z only: fails the check
    assert conv.get_apr(A.APR(), img) is False
    conv.par = lib_params(check_input=True, swap_dimensions=True)
    assert conv.get_apr(A.APR(), img) is True


def test_empty_and_flat_inputs():
    conv = A.APRConverter("uint16")
    conv.par = lib_params()
    flat = np.full((16, 16, 16), 100, np.uint16)
    apr = A.APR()
    assert conv.get_apr(apr, flat)
    e, acc, _ = B.orc_get_apr(flat, oracle_params(), 1)
    lx, xe, yv = apr.linear_access()
    assert np.array_equal(xe, acc.xz_end) and np.array_equal(yv, acc.y_vec)
    tiny = np.array([[[7, 9, 200]]], np.uint16)
    assert conv.get_apr(apr, tiny)
    e, acc, _ = B.orc_get_apr(tiny, oracle_params(), 1)
    assert np.array_equal(apr.linear_access()[2], acc.y_vec)


def test_gradient_magnitudes_beyond_uint16_range():
    """uint16 ImageType whose gradient magnitudes exceed 65535 (steps of 65000
    with dy = 0.25 and no smoothing): the stored gradient wraps as the
    reference's conversion does, so the per-cell maximum is taken over the
    converted magnitudes there."""
    img = np.full((12, 20, 24), 100, np.uint16)
    img[:, :, 12:] = 65000
    img[4:8, 5:15, 3:9] = 40000
    kw = dict(lambda_=0.0, dy=0.25, dx=0.5)
    e, acc, (off, inter) = B.orc_get_apr(img, oracle_params(**kw), 1)
    assert e == 0
    conv, apr = gpu_apr(img, 1, **kw)
    ds = STAGE_SHAPE_DS(img.shape)
    assert inter[1].max() > 0
    for w in range(1, 7):
        assert bits_equal(conv.intermediate(w, ds), inter[w]), "stage %d" % w
    lx, xe, yv = apr.linear_access()
    assert np.array_equal(xe, acc.xz_end) and np.array_equal(yv, acc.y_vec)


@pytest.mark.parametrize("image_type", ["float", "uint16"])
def test_host_calls_copy_in_chunks_like_device_calls(image_type):
    """Host-buffer get_apr and sample_image copy a volume with large planes in
    z-chunks, overlapped with the smoothing and the sampling; the structure
    and the particles equal those of the device-buffer calls.  2048 x 2048
    planes, 33 of them: several chunks, an odd last plane."""
    import ctypes as C

    import torch
    from libapr_b200._lib import check, lib

    z, x, y = 33, 2048, 2048
    dev = torch.empty((z, x, y), dtype=torch.int16, device="cuda")
    A.synth_blobs_device(dev, 2000, sigma=(2.0, 8.0), amp=(500.0, 6000.0), seed=17)
    torch.cuda.synchronize()
    host = dev.cpu().numpy().view(np.uint16)
    conv = A.APRConverter(image_type)
    conv.par = lib_params()
    a_dev, a_host = A.APR(), A.APR()
    assert conv.get_apr(a_dev, dev)
    assert conv.get_apr(a_host, host)
    for u, v in zip(a_dev.linear_access(), a_host.linear_access()):
        assert np.array_equal(u, v)
    P = a_dev.total_number_particles()
    assert a_dev.level_max() > a_dev.level_min() and P > 0
    pd = torch.empty(P, dtype=torch.int16, device="cuda")
    check(lib().aprb_sample_image_device(a_dev._h, C.c_void_p(dev.data_ptr()), C.c_void_p(pd.data_ptr()), None))
    torch.cuda.synchronize()
    ph = A.ParticleData().sample_image(a_host, host).data
    assert np.array_equal(ph, pd.cpu().numpy().view(np.uint16))


def test_keep_input_samples_the_uploaded_copy():
    """keep_input: the host-buffer get_apr hands its device copy to the APR,
    sample_image from the same array uses it (no second upload) and equals
    the plain call; a different array is uploaded as usual."""
    img = volume((48, 64, 72), 30, 31)
    conv = A.APRConverter("float")
    conv.par = lib_params()
    ref_apr = A.APR()
    assert conv.get_apr(ref_apr, img)
    ref_parts = A.ParticleData().sample_image(ref_apr, img).data
    conv.keep_input(True)
    apr = A.APR()
    assert conv.get_apr(apr, img)
    assert np.array_equal(A.ParticleData().sample_image(apr, img).data, ref_parts)
    # the kept copy was consumed: a second sampling uploads the array again
    assert np.array_equal(A.ParticleData().sample_image(apr, img).data, ref_parts)
    other = img.copy()
    other[::2] //= 2
    apr2 = A.APR()
    assert conv.get_apr(apr2, img)
    assert np.array_equal(A.ParticleData().sample_image(apr2, other).data,
                          A.ParticleData().sample_image(ref_apr, other).data)


@pytest.fixture(scope="module")
def tma_case():
    shape = (37, 45, 600)  # takes the TMA kernels on every axis
    img = volume(shape, 25, 21)
    e, acc, (off, inter) = B.orc_get_apr(img, oracle_params(), 0)
    assert e == 0
    return img, acc, inter[0]


@pytest.mark.parametrize("axis,variant", [("y", v) for v in range(3)] + [("x", v) for v in range(5)] +
                         [("z", v) for v in range(5)])
def test_every_smoothing_variant_bit_exact(tma_case, axis, variant):
    """Each kernel variant of the smoothing schedule (the autotuner's choices)
    gives the reference's smoothed image and structure bit for bit."""
    img, acc, smoothed = tma_case
    old = A.smoothing_schedule()
    try:
        A.set_smoothing_schedule({axis: [variant] * len(A.SCHEDULE_BUCKETS)})
        conv, apr = gpu_apr(img, 0)
        assert bits_equal(conv.intermediate(0, img.shape), smoothed)
        assert np.array_equal(apr.linear_access()[2], acc.y_vec)
    finally:
        A.set_smoothing_schedule(old)


def test_host_calls_from_two_threads_match_one_thread():
    """Two host threads, each with its own converter (keep_input on), convert
    and sample different volumes through the host-buffer calls at the same
    time: their uploads take turns on the device and their APRs are freed
    without a device-wide wait.  Every structure and every particle equals
    the one-thread result of the same volume."""
    import threading

    import torch

    shape = (40, 512, 512)
    vols = []
    for seed in (31, 32, 33, 34):
        dev = torch.empty(shape, dtype=torch.int16, device="cuda")
        A.synth_blobs_device(dev, 300, sigma=(2.0, 6.0), amp=(500.0, 6000.0), seed=seed)
        torch.cuda.synchronize()
        vols.append(np.ascontiguousarray(dev.cpu().numpy().view(np.uint16)))

    def convert(conv, img):
        apr = A.APR()
        assert conv.get_apr(apr, img)
        parts = A.ParticleData().sample_image(apr, img).data.copy()
        return [a.copy() for a in apr.linear_access()], parts

    ref_conv = A.APRConverter("float")
    ref_conv.par = lib_params()
    ref = [convert(ref_conv, v) for v in vols]

    results = [None] * len(vols)
    errors = []

    def worker(t):
        try:
            torch.cuda.set_device(0)
            conv = A.APRConverter("float")
            conv.par = lib_params()
            conv.keep_input(True)
            for k in range(t, len(vols), 2):
                results[k] = convert(conv, vols[k])
        except Exception as e:  # noqa: BLE001 -- reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(2)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
    for (sr, pr), (s, p) in zip(ref, results):
        for u, v in zip(sr, s):
            assert np.array_equal(u, v)
        assert np.array_equal(pr, p)

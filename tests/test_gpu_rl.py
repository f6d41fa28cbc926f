"""APR Richardson-Lucy on a deconvolution workload (blob ground truth blurred
by a normalised 5x5x5 Gaussian PSF, sigma 1.2, Poisson noise, uint16; APR with
lambda=3, E=0.1, Ip_th=0, sigma_th=50, grad_th=10), at a size the CPU oracle
runs in seconds: the FP32 GPU estimate against the FP64 oracle after 20, 100
and 200 iterations, and the GPU FP64 path bit-exact against the oracle."""
import numpy as np
import pytest

import libapr_b200 as A
from oracle import bind as B
from tests.helpers import gaussian_psf, lib_params, oracle_params

pytestmark = pytest.mark.gpu

# FP32 against FP64 RL after k iterations, relative L2 (measured ~1e-6..1e-5;
# bound with margin)
FP32_VS_FP64_RTOL = 1e-4


def deconv_volume(shape=(32, 64, 64), n_blobs=12, seed=31):
    from scipy.ndimage import convolve
    rng = np.random.default_rng(seed)
    z, x, y = shape
    zz, xx, yy = np.meshgrid(np.arange(z) + 0.5, np.arange(x) + 0.5, np.arange(y) + 0.5, indexing="ij")
    gt = np.full(shape, 50.0)
    for _ in range(n_blobs):
        c = rng.uniform(0, 1, 3) * np.array(shape)
        s = rng.uniform(1.0, 4.0)
        a = rng.uniform(500.0, 5000.0)
        gt += a * np.exp(-((zz - c[0]) ** 2 + (xx - c[1]) ** 2 + (yy - c[2]) ** 2) / (2 * s * s))
    blurred = convolve(gt, gaussian_psf(1.2, 5).astype(np.float64), mode="reflect")
    return np.clip(rng.poisson(blurred), 0, 65535).astype(np.uint16)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_rl_fp32_against_fp64_oracle():
    img = deconv_volume()
    e, acc, _ = B.orc_get_apr(img, oracle_params(), 0)
    assert e == 0
    tr = B.orc_tree(acc)
    parts = B.orc_sample(acc, img)
    conv = A.APRConverter("float")
    conv.par = lib_params()
    apr = A.APR()
    assert conv.get_apr(apr, img)
    assert np.array_equal(apr.linear_access()[2], acc.y_vec)
    psf = gaussian_psf(1.2, 5)
    f32 = A.ParticleData()
    f64 = None
    done = 0
    for k in (20, 100, 200):
        A.APRNumerics.richardson_lucy(apr, parts, f32, psf, k - done, normalize=True, resume=done > 0)
        f64 = B.orc_richardson_lucy(acc, tr, parts, psf, k - done, normalize=True, use_double=True, init=f64)
        done = k
        err = rel_l2(f32.data, f64)
        print("RL iterations %d: FP32 GPU vs FP64 oracle relative L2 %.3e" % (k, err))
        assert err < FP32_VS_FP64_RTOL
    g64 = A.APRNumerics.richardson_lucy(apr, parts, None, psf, 200, normalize=True, dtype=np.float64)
    assert np.array_equal(g64.view(np.uint64), f64.view(np.uint64))

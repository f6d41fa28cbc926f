"""The reconstruction condition of the reference's pipeline tests
(test_pipeline_bound / test_pipeline_bound_blocked, test/APRTest.cpp:2930-3045,
compare_gt test/TestTools.hpp:147-192): the piecewise-constant reconstruction
differs from the input by at most rel_error times the local intensity scale,
at every pixel brighter than 1000."""
import numpy as np

# parameters of test_pipeline_bound (test/APRTest.cpp:2941-2949)
BOUND_PARAMS = dict(lambda_=0.0, Ip_th=0.0, sigma_th=100.0, sigma_th_max=50.0, grad_th=0.0)
REL_ERRORS = (0.2, 0.1, 0.05, 0.01, 0.001)


def inf_norm(img, recon, scale_ds, background=1000):
    """max |img - recon| / scale(y/2, x/2, z/2) over pixels > background."""
    img = np.asarray(img)
    z, x, y = img.shape
    sc = scale_ds[np.arange(z)[:, None, None] // 2, np.arange(x)[None, :, None] // 2,
                  np.arange(y)[None, None, :] // 2].astype(np.float64)
    m = img > background
    if not m.any():
        return 0.0
    d = np.abs(img.astype(np.float64) - np.asarray(recon).astype(np.float64))
    return float((d[m] / sc[m]).max())

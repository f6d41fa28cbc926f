"""Shared helpers for the parity tests: seeded inputs and the parameter sets
of the benchmark configurations (synthetic, seeded: no dataset is read)."""
import numpy as np

from libapr_b200.synth import blob_volume
from oracle import bind as B

# APR parameters of the get_apr configurations: lambda=3, E=0.1, Ip_th=0,
# sigma_th=50, grad_th=10.
CFG_PARAMS = dict(lambda_=3.0, rel_error=0.1, Ip_th=0.0, sigma_th=50.0, grad_th=10.0)


def oracle_params(**kw):
    d = dict(CFG_PARAMS)
    d.update(kw)
    return B.make_params(**d)


def lib_params(**kw):
    import libapr_b200 as A
    d = dict(CFG_PARAMS)
    d.update(kw)
    p = A.APRParameters()
    for k, v in d.items():
        setattr(p, k, v)
    return p


def volume(shape, n_blobs, seed, sigma=(2.0, 6.0), amp=(800.0, 4000.0), background=100.0):
    return blob_volume(shape, n_blobs, sigma=sigma, amp=amp, background=background, seed=seed)


def random_stencil(ks, seed):
    """Stencil uniform in [-1, 1], normalised to sum 1 (the conv configuration)."""
    rng = np.random.default_rng(seed)
    st = rng.uniform(-1, 1, ks ** 3).astype(np.float32)
    return (st / st.sum()).astype(np.float32)


def gaussian_psf(sigma=1.2, ks=5):
    g = np.exp(-((np.arange(ks) - ks // 2) ** 2) / (2 * sigma * sigma)).astype(np.float32)
    p = (g[:, None, None] * g[None, :, None] * g[None, None, :]).astype(np.float32)
    return (p / p.sum()).astype(np.float32)


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype == np.float32:
        return np.array_equal(a.view(np.uint32), b.view(np.uint32))
    return np.array_equal(a, b)

"""Seeded synthetic volumes with the shapes and value model of the benchmark
configurations: a constant background, isotropic Gaussian blobs (centres
uniform in the volume, sigma and peak amplitude uniform in given ranges) and
Poisson noise, clipped to uint16.  Arrays are (z, x, y) in C order, i.e. the
reference's PixelData memory order.

This host version (numpy, float64 rendering) is for test-sized volumes; the
library's device generator (``aprb_synth_blobs_u16``) produces the
benchmark-sized ones with the same model.
"""
import numpy as np


def blob_params(shape_zxy, n_blobs, sigma=(2.0, 6.0), amp=(800.0, 4000.0), seed=0):
    rng = np.random.default_rng(seed)
    z, x, y = shape_zxy
    c = rng.uniform(0, 1, size=(n_blobs, 3)) * np.array([z, x, y])
    s = rng.uniform(sigma[0], sigma[1], size=n_blobs)
    a = rng.uniform(amp[0], amp[1], size=n_blobs)
    return c, s, a, rng


def blob_volume(shape_zxy, n_blobs, sigma=(2.0, 6.0), amp=(800.0, 4000.0), background=100.0, seed=0,
                noise=True, dtype=np.uint16):
    z, x, y = shape_zxy
    c, s, a, rng = blob_params(shape_zxy, n_blobs, sigma, amp, seed)
    vol = np.full(shape_zxy, background, dtype=np.float64)
    for (cz, cx, cy), sg, am in zip(c, s, a):
        r = int(np.ceil(4 * sg))
        z0, z1 = max(int(cz) - r, 0), min(int(cz) + r + 1, z)
        x0, x1 = max(int(cx) - r, 0), min(int(cx) + r + 1, x)
        y0, y1 = max(int(cy) - r, 0), min(int(cy) + r + 1, y)
        if z0 >= z1 or x0 >= x1 or y0 >= y1:
            continue
        gz = np.exp(-((np.arange(z0, z1) + 0.5 - cz) ** 2) / (2 * sg * sg))
        gx = np.exp(-((np.arange(x0, x1) + 0.5 - cx) ** 2) / (2 * sg * sg))
        gy = np.exp(-((np.arange(y0, y1) + 0.5 - cy) ** 2) / (2 * sg * sg))
        vol[z0:z1, x0:x1, y0:y1] += am * gz[:, None, None] * gx[None, :, None] * gy[None, None, :]
    if noise:
        vol = rng.poisson(vol).astype(np.float64)
    if dtype == np.float32:
        return vol.astype(np.float32)
    return np.clip(np.rint(vol), 0, 65535).astype(np.uint16)

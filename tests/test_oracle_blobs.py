"""The CPU twin of the benchmark generator (oracle/blobs.c): its noise-free
intensities against a float64 rendering of the same blob parameters, its
Poisson deviates' moments in both sampler branches, and determinism.  The
GPU test (test_gpu_synth.py) checks that the device generator writes the
same bytes."""
import numpy as np
import pytest

from oracle import bind as B

M64 = (1 << 64) - 1


def _splitmix_params(shape, n_blobs, sigma, amp, seed):
    """The generator's blob parameter stream restated (splitmix64)."""
    st = [(seed * 0x2545F4914F6CDD1D + 0x632BE59BD9B4E019) & M64]

    def unif():
        st[0] = (st[0] + 0x9E3779B97F4A7C15) & M64
        z = st[0]
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        z ^= z >> 31
        return (z >> 11) * (1.0 / 9007199254740992.0)

    z, x, y = shape
    out = []
    for _ in range(n_blobs):
        cz, cx, cy = np.float32(unif() * z), np.float32(unif() * x), np.float32(unif() * y)
        sg = np.float32(np.float32(sigma[0]) + unif() * float(np.float32(sigma[1]) - np.float32(sigma[0])))
        a = np.float32(np.float32(amp[0]) + unif() * float(np.float32(amp[1]) - np.float32(amp[0])))
        out.append((float(cz), float(cx), float(cy), float(sg), float(a)))
    return out


def test_noise_free_intensities_match_float64_rendering():
    shape, nb, sigma, amp, bg = (24, 40, 56), 25, (2.0, 6.0), (800.0, 4000.0), 100.0
    img = B.blob_volume_cpu(shape, nb, sigma, amp, bg, seed=11, noise=False)
    ref = np.full(shape, bg, np.float64)
    zz, xx, yy = np.meshgrid(*(np.arange(n) + 0.5 for n in shape), indexing="ij")
    for cz, cx, cy, sg, a in _splitmix_params(shape, nb, sigma, amp, 11):
        d2 = (zz - cz) ** 2 + (xx - cx) ** 2 + (yy - cy) ** 2
        # the generator sums a blob over the 16^3 bricks its 4-sigma box meets
        bz = [(int(np.floor((c - 4 * sg) / 16)), int(np.floor((c + 4 * sg) / 16))) for c in (cz, cx, cy)]
        m = np.ones(shape, bool)
        for ax, (lo, hi), g in zip(range(3), bz, (zz, xx, yy)):
            b = np.floor(g / 16)
            m &= (b >= lo) & (b <= hi)
        ref += np.where(m, a * np.exp(-d2 / (2 * sg * sg)), 0.0)
    rel = np.abs(img - ref) / ref
    assert rel.max() < 2e-6


@pytest.mark.parametrize("bg", [0.5, 3.0, 9.5, 10.0, 100.0, 5000.0])
def test_poisson_moments(bg):
    a = B.blob_volume_cpu((64, 64, 64), 0, (2.0, 6.0), (800.0, 4000.0), bg, seed=5).astype(np.float64)
    n = a.size
    tol = 5 * np.sqrt(bg / n)  # five standard errors of the mean
    assert abs(a.mean() - bg) < tol
    assert abs(a.var() / bg - 1) < 0.03


def test_deterministic_and_seeded():
    a = B.blob_volume_cpu((20, 33, 47), 12, (2.0, 8.0), (500.0, 6000.0), 100.0, seed=3)
    b = B.blob_volume_cpu((20, 33, 47), 12, (2.0, 8.0), (500.0, 6000.0), 100.0, seed=3)
    c = B.blob_volume_cpu((20, 33, 47), 12, (2.0, 8.0), (500.0, 6000.0), 100.0, seed=4)
    assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_clipped_to_uint16():
    a = B.blob_volume_cpu((16, 16, 16), 0, (2.0, 6.0), (800.0, 4000.0), 70000.0, seed=1)
    assert a.max() == 65535

"""The device generator (aprb_synth_blobs_u16 / _f32) writes the same bytes
as its CPU twin (oracle/blobs.c), so a CPU-only run of the benchmark workload
(the reference arm) converts exactly the volume the GPU converts."""
import numpy as np
import pytest

from oracle import bind as B

pytestmark = pytest.mark.gpu

CASES = [
    ((20, 33, 47), 12, (2.0, 8.0), (500.0, 6000.0), 100.0, 3),
    ((64, 64, 64), 40, (2.0, 6.0), (800.0, 4000.0), 100.0, 9),
    ((128, 256, 256), 400, (2.0, 6.0), (800.0, 4000.0), 100.0, 1),  # the config-0 volume
    ((96, 128, 160), 300, (1.0, 4.0), (500.0, 5000.0), 50.0, 3000),
    ((17, 18, 19), 5, (2.0, 6.0), (800.0, 4000.0), 4.0, 2),  # small-mean Poisson branch
]


@pytest.mark.parametrize("shape,nb,sigma,amp,bg,seed", CASES)
def test_device_generator_matches_cpu_twin(shape, nb, sigma, amp, bg, seed):
    import torch
    import libapr_b200 as A
    d = torch.empty(shape, dtype=torch.int16, device="cuda")
    A.synth_blobs_device(d, nb, sigma, amp, bg, seed=seed)
    gpu = d.cpu().numpy().view(np.uint16)
    cpu = B.blob_volume_cpu(shape, nb, sigma, amp, bg, seed)
    assert np.array_equal(gpu, cpu)
    f = torch.empty(shape, dtype=torch.float32, device="cuda")
    A.synth_ground_truth_device(f, nb, sigma, amp, bg, seed=seed)
    gf = f.cpu().numpy()
    cf = B.blob_volume_cpu(shape, nb, sigma, amp, bg, seed, noise=False)
    assert np.array_equal(gf.view(np.uint32), cf.view(np.uint32))

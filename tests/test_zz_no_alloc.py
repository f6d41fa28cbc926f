"""aprb_sample_image_noalloc: particle sampling for callers that cannot
allocate GPU memory while they run (real-time acquisition loops that may not
stall on an allocation, plugin hosts with a fixed device-memory budget).

The entry point keeps its down-sampling pyramid in a fixed 64 MiB device
buffer, reserved on a device when the library's module is first used there.
This file is collected last so that a run stopping at the first failure has
already run every other test; the test passes alone in a fresh process and
after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_sampling_matches_sample_image_on_two_calls():
    import torch

    import libapr_b200 as A
    from libapr_b200 import _lib
    from tests.helpers import lib_params, volume

    L = _lib.lib()
    img1 = volume((48, 64, 80), 20, 21)
    img2 = volume((48, 64, 80), 25, 22)
    conv = A.APRConverter("uint16")
    conv.par = lib_params()
    apr = A.APR()
    assert conv.get_apr(apr, img1)
    P = apr.total_number_particles()
    xz = C.c_void_p()
    yv = C.c_void_p()
    _lib.check(L.aprb_apr_device_arrays(apr._h, None, C.byref(xz), C.byref(yv)))
    z, x, y = img1.shape
    stream = torch.cuda.current_stream()
    out = torch.empty(P, dtype=torch.int16, device="cuda")
    for k, img in enumerate((img1, img2)):  # two calls in a row through the same scratch
        expected = A.ParticleData().sample_image(apr, img).data
        dimg = torch.from_numpy(img.view(np.int16)).cuda()
        out.fill_(-1)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = L.aprb_sample_image_noalloc(xz, yv, y, x, z, C.c_void_p(dimg.data_ptr()), C.c_void_p(out.data_ptr()),
                                         C.c_void_p(stream.cuda_stream))
        _lib.check(st)
        torch.cuda.synchronize()
        if k == 1:  # a warm call takes no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
        got = out.cpu().numpy().view(np.uint16)
        assert np.array_equal(got, expected)


def test_noalloc_rejects_volumes_beyond_its_scratch():
    from libapr_b200 import _lib

    L = _lib.lib()
    dummy = C.c_void_p(256)  # never dereferenced: the size check comes first
    st = L.aprb_sample_image_noalloc(dummy, dummy, 4096, 4096, 2048, dummy, dummy, None)
    assert st == 1
    assert b"scratch" in L.aprb_last_error()

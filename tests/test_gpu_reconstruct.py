"""GPU reconstruction (APRReconstruction::reconstruct_constant /
reconstruct_level, src/numerics/APRReconstruction.hpp:80, 132) against the
reference's per-pixel golden images and the numpy oracle."""
import ctypes as C
import os

import numpy as np
import pytest

import libapr_b200 as A
from oracle import bind as B
from tests.helpers import lib_params, oracle_params, volume

pytestmark = pytest.mark.gpu


def case_params(d):
    lam, E, gth, sth, sthm = [float(v) for v in d["params"]]
    return oracle_params(lambda_=lam, rel_error=E, grad_th=gth, sigma_th=max(sth, 0.1), sigma_th_max=max(sthm, 0.1),
                         Ip_th=0.0)


@pytest.mark.parametrize("case", ["sphere_diff_dims", "sphere_120", "sphere_2D", "sphere_1D"])
def test_reconstruction_of_stored_apr_matches_saved_images(golden_dir, case):
    d = np.load(os.path.join(golden_dir, case + ".npz"))
    img = d["original"]
    acc = B.orc_get_apr_custom(d["gradient_saved"].astype(np.float32), d["scale_saved"], img.shape, case_params(d))
    apr = A.APR.from_arrays(img.shape, acc.level_xz, acc.xz_end, acc.y_vec)
    assert np.array_equal(A.APRReconstruction.reconstruct_level(apr).astype(np.uint16), d["img_level"])
    parts = A.ParticleData().sample_image(apr, img).data
    assert np.array_equal(A.APRReconstruction.reconstruct_constant(apr, parts), d["img_pc"])


@pytest.mark.parametrize("shape,blobs,seed", [((40, 48, 56), 30, 1), ((17, 33, 70), 12, 2), ((1, 63, 64), 6, 4),
                                              ((64, 64, 64), 60, 8)])
def test_reconstruction_matches_oracle(shape, blobs, seed):
    img = volume(shape, blobs, seed)
    e, acc, _ = B.orc_get_apr(img, oracle_params(), 1)
    assert e == 0
    conv = A.APRConverter("uint16")
    conv.par = lib_params()
    apr = A.APR()
    assert conv.get_apr(apr, img)
    parts = A.ParticleData().sample_image(apr, img).data
    assert np.array_equal(A.APRReconstruction.reconstruct_level(apr), B.orc_reconstruct(acc))
    assert np.array_equal(A.APRReconstruction.reconstruct_constant(apr, parts), B.orc_reconstruct(acc, parts))
    pf = (parts.astype(np.float32) * np.float32(0.37)).astype(np.float32)
    assert np.array_equal(A.APRReconstruction.reconstruct_constant(apr, pf), B.orc_reconstruct(acc, pf))


def test_reconstruction_device_entry_points():
    import torch
    from libapr_b200._lib import check, lib

    img = volume((33, 65, 31), 20, 6)
    conv = A.APRConverter("float")
    conv.par = lib_params()
    apr = A.APR()
    assert conv.get_apr(apr, img)
    parts = A.ParticleData().sample_image(apr, img).data
    pd = torch.from_numpy(parts.view(np.int16)).cuda()
    out = torch.empty(img.shape, dtype=torch.int16, device="cuda")
    lv = torch.empty(img.shape, dtype=torch.uint8, device="cuda")
    check(lib().aprb_reconstruct_constant_u16_device(apr._h, C.c_void_p(pd.data_ptr()), C.c_void_p(out.data_ptr()),
                                                     None))
    check(lib().aprb_reconstruct_level_device(apr._h, C.c_void_p(lv.data_ptr()), None))
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint16), A.APRReconstruction.reconstruct_constant(apr, parts))
    assert np.array_equal(lv.cpu().numpy(), A.APRReconstruction.reconstruct_level(apr))

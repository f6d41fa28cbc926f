"""The GPU pipeline satisfies the reference's reconstruction bound
(test_pipeline_bound / test_pipeline_bound_blocked, test/APRTest.cpp:2930-3045):
a size-independent property checked on the golden spheres and on seeded
volumes up to 128 x 512 x 512, whole-volume and blocked."""
import os

import numpy as np
import pytest

import libapr_b200 as A
from tests.bound_helpers import BOUND_PARAMS, REL_ERRORS, inf_norm
from tests.conftest import ROOT
from tests.helpers import volume

pytestmark = pytest.mark.gpu

STAGE_LOCAL_SCALE = 3


def _params(rel_error):
    p = A.APRParameters(rel_error=rel_error)
    for k, v in BOUND_PARAMS.items():
        setattr(p, k, v)
    return p


INPUTS = ["sphere_120", "sphere_diff_dims", "blobs_64x96x80", "blobs_128x512x512"]
_CACHE = {}


def _image(name):
    if name not in _CACHE:
        if name.startswith("sphere"):
            _CACHE[name] = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))["original"]
        elif name == "blobs_64x96x80":
            _CACHE[name] = volume((64, 96, 80), 40, 3)
        else:
            _CACHE[name] = volume((128, 512, 512), 3000, 5, amp=(800.0, 6000.0))
    return _CACHE[name]


def _whole(img, rel_error):
    conv = A.APRConverter("uint16")
    conv.keep_intermediates(True)
    conv.par = _params(rel_error)
    apr = A.APR()
    assert conv.get_apr(apr, img)
    z, x, y = img.shape
    scale = conv.intermediate(STAGE_LOCAL_SCALE, ((z + 1) // 2, (x + 1) // 2, (y + 1) // 2))
    return apr, scale


@pytest.mark.parametrize("name", INPUTS)
@pytest.mark.parametrize("rel_error", REL_ERRORS)
def test_reconstruction_bound(name, rel_error):
    img = _image(name)
    apr, scale = _whole(img, rel_error)
    parts = A.ParticleData().sample_image(apr, img)
    rec = A.APRReconstruction.reconstruct_constant(apr, parts)
    assert inf_norm(img, rec, scale) <= rel_error


@pytest.mark.parametrize("name", INPUTS[1:3])
@pytest.mark.parametrize("rel_error", REL_ERRORS)
def test_reconstruction_bound_blocked(name, rel_error):
    """z blocks of 32 with 16 ghost planes, blocked sampling 32 / 32, scale of
    the whole-volume converter (test/APRTest.cpp:2988-3045)."""
    img = _image(name)
    _, scale = _whole(img, rel_error)
    conv = A.APRConverterBatch("uint16", z_block_size=32, ghost_z=16)
    conv.par = _params(rel_error)
    apr = A.APR()
    assert conv.get_apr(apr, img)
    parts = A.ParticleData().sample_parts_from_img_blocked(apr, img, 32, 32)
    rec = A.APRReconstruction.reconstruct_constant(apr, parts)
    assert inf_norm(img, rec, scale) <= rel_error

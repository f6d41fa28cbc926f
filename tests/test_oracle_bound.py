"""The oracle satisfies the reference's reconstruction bound on the golden
sphere inputs (test_pipeline_bound, test/APRTest.cpp:2930-2986)."""
import os

import numpy as np
import pytest

from oracle import bind as B
from tests.bound_helpers import BOUND_PARAMS, REL_ERRORS, inf_norm
from tests.conftest import ROOT


@pytest.mark.parametrize("name", ["sphere_120", "sphere_diff_dims"])
@pytest.mark.parametrize("rel_error", REL_ERRORS)
def test_oracle_reconstruction_bound(name, rel_error):
    img = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))["original"]
    e, acc, (off, inter) = B.orc_get_apr(img, B.make_params(rel_error=rel_error, **BOUND_PARAMS), 1)
    assert e == 0
    rec = B.orc_reconstruct(acc, B.orc_sample(acc, img))
    assert inf_norm(img, rec, inter[3]) <= rel_error

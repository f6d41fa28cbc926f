"""CPU-side checks of the drop-in boundary: libaprb200.so loads, exports every
entry point include/aprb200.h declares, and the host-side parameter mirror
keeps the reference defaults.  No compute call is made (no GPU here)."""
import os
import re

import pytest

from tests.conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "aprb200.h")).read()
    return sorted(set(re.findall(r"\b(aprb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from libapr_b200 import _lib
    L = _lib.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.SIGNATURES), "ctypes signatures must cover exactly the declared ABI"


def test_default_parameters_mirror_reference():
    import libapr_b200 as A
    p = A.APRParameters()
    # APRParameters.hpp:14-41
    assert (p.dx, p.dy, p.dz, p.psfx, p.Ip_th, p.lambda_, p.sigma_th, p.grad_th) == (1, 1, 1, 2, 0, 3, 0, 0)
    assert abs(p.rel_error - 0.1) < 1e-7
    assert p.reflect_bc_lis and p.neighborhood_optimization and not p.constant_intensity_scale
    setattr(p, "lambda", 2.0)
    assert p.lambda_ == 2.0
    with pytest.raises(AttributeError):
        p.not_a_field = 1


def test_status_strings():
    from libapr_b200 import _lib
    L = _lib.lib()
    for s in range(9):
        assert L.aprb_status_string(s)

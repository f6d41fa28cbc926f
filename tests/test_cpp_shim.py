"""The C++ host layer (include/aprb200.hpp) compiles against the C ABI and, on
a GPU, produces the same APR as the Python path."""
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "shim_example.cpp")


def build(tmp_path):
    exe = str(tmp_path / "shim_example")
    libdir = os.path.join(ROOT, "libapr_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-L", libdir,
                    "-laprb200", "-Wl,-rpath," + libdir, "-o", exe], check=True)
    return exe


def test_cpp_shim_compiles_and_links(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_cpp_shim_matches_python_path(tmp_path):
    import libapr_b200 as A
    from tests.helpers import lib_params, volume
    exe = build(tmp_path)
    img = volume((24, 40, 48), 10, 31)
    raw = tmp_path / "img.raw"
    img.tofile(raw)
    out = subprocess.run([exe, str(raw)], check=True, capture_output=True, text=True).stdout.strip()
    conv = A.APRConverter("uint16")
    conv.par = lib_params()
    apr = A.APR()
    assert conv.get_apr(apr, img)
    parts = A.ParticleData().sample_image(apr, img).data
    c = A.APRFilter.convolve_pencil(apr, np.full(27, 1.0 / 27, np.float32), parts.astype(np.float32))
    P, s, cs, rs, ls, gs, aP, gth, sth = out.split()
    g = A.APRNumerics.gradient_magnitude_cfd(apr, parts.astype(np.float32))
    assert abs(float(gs.split("=")[1]) - float(g.astype(np.float64).sum())) <= 1e-3 * max(1.0, abs(float(g.sum())))
    conv_auto = A.APRConverter("uint16")
    conv_auto.par = lib_params(auto_parameters=True)
    apr_auto = A.APR()
    assert conv_auto.get_apr(apr_auto, img)
    used = apr_auto.get_apr_parameters()
    assert np.float32(float(gth.split("=")[1])) == np.float32(used.grad_th)
    assert np.float32(float(sth.split("=")[1])) == np.float32(used.sigma_th)
    assert int(aP.split("=")[1]) == apr_auto.total_number_particles()
    assert int(rs.split("=")[1]) == int(A.APRReconstruction.reconstruct_constant(apr, parts).astype(np.uint64).sum())
    assert int(ls.split("=")[1]) == int(A.APRReconstruction.reconstruct_level(apr).astype(np.uint64).sum())
    assert int(P.split("=")[1]) == apr.total_number_particles()
    assert int(s.split("=")[1]) == int(parts.astype(np.uint64).sum())
    assert abs(float(cs.split("=")[1]) - float(c.astype(np.float64).sum())) <= 1e-3 * max(1.0, abs(float(c.sum())))

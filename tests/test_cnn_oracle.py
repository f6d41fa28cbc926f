"""The FP64 oracle of the learned proposal's layer: its backward pass
against central finite differences of its forward pass (CPU only)."""
import numpy as np
import pytest

from oracle import bind as B
from oracle import cnn_oracle as O
from tests.helpers import oracle_params, volume


@pytest.fixture(scope="module")
def geo():
    img = volume((12, 16, 20), 6, 3)
    e, acc, _ = B.orc_get_apr(img, oracle_params(), 1)
    assert e == 0
    return O.Geometry(acc, B.orc_tree(acc))


@pytest.mark.parametrize("relu", [False, True])
def test_backward_matches_finite_differences(geo, relu):
    rng = np.random.default_rng(11)
    H = rng.normal(size=(geo.P, O.C))
    W = rng.normal(size=(27, O.C, O.C)) * 0.2
    b = rng.normal(size=O.C) * 0.1
    R = rng.normal(size=(geo.P, O.C))

    def loss(H_, W_, b_):
        return float((O.layer_forward(geo, H_, W_, b_, relu) * R).sum())

    out = O.layer_forward(geo, H, W, b, relu)
    g_in, dW, db = O.layer_backward(geo, H, W, out, R, relu)
    eps = 1e-6
    for _ in range(6):
        i, c = rng.integers(geo.P), rng.integers(O.C)
        Hp, Hm = H.copy(), H.copy()
        Hp[i, c] += eps
        Hm[i, c] -= eps
        fd = (loss(Hp, W, b) - loss(Hm, W, b)) / (2 * eps)
        assert abs(fd - g_in[i, c]) <= 1e-5 * max(1.0, abs(fd)), (i, c, fd, g_in[i, c])
    for _ in range(6):
        t, o, c = rng.integers(27), rng.integers(O.C), rng.integers(O.C)
        Wp, Wm = W.copy(), W.copy()
        Wp[t, o, c] += eps
        Wm[t, o, c] -= eps
        fd = (loss(H, Wp, b) - loss(H, Wm, b)) / (2 * eps)
        assert abs(fd - dW[t, o, c]) <= 1e-5 * max(1.0, abs(fd))
    c = rng.integers(O.C)
    bp, bm = b.copy(), b.copy()
    bp[c] += eps
    bm[c] -= eps
    fd = (loss(H, W, bp) - loss(H, W, bm)) / (2 * eps)
    assert abs(fd - db[c]) <= 1e-5 * max(1.0, abs(fd))


def test_tree_gradient_reaches_fine_particles(geo):
    """A gradient on coarse particles flows to finer particles through the tree means."""
    W = np.zeros((27, O.C, O.C))
    W[:, 0, 0] = 1.0
    H = np.zeros((geo.P, O.C))
    out = O.layer_forward(geo, H, W, np.zeros(O.C), False)
    g = np.zeros((geo.P, O.C))
    lmin = geo.acc.l_min
    g[geo.plev == geo.plev.min(), 0] = 1.0
    g_in, _, _ = O.layer_backward(geo, H, W, out, g, False)
    assert np.abs(g_in[geo.plev > lmin + 1, 0]).sum() > 0


def test_bf16_rounding():
    # 1 + 2^-8 is half-way between bfloat16 neighbours 1 and 1 + 2^-7: ties to even
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 3.14159265], np.float32)
    assert list(O.bf16(v)) == [1.0, 1.0, 1.0078125, 3.140625]

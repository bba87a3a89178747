"""The U-Net CPU oracle pinned by central finite differences (float64), and its BF16 emulation
close to the exact network."""
import numpy as np

import unet_oracle as UO


def _problem(G=9, B=2, seed=0):
    rng = np.random.default_rng(seed)
    from featb200.unet import init_params, num_params
    theta = init_params(seed).astype(np.float64)
    # non-zero biases so that every path carries signal
    theta += 0.05 * rng.standard_normal(theta.size) * (np.abs(theta) == 0)
    inp = rng.standard_normal((B, 2, G, G))
    tgt = rng.standard_normal((B, G, G))
    assert theta.size == num_params() == UO.num_params()
    return theta, inp, tgt


def _loss(theta, inp, tgt):
    y, _ = UO.forward(theta, inp, exact=True)
    return UO.mse(y, tgt)[0]


def test_oracle_gradient_matches_finite_differences():
    theta, inp, tgt = _problem()
    y, cache = UO.forward(theta, inp, exact=True)
    _, dy = UO.mse(y, tgt)
    g = UO.backward(cache, dy, exact=True)
    rng = np.random.default_rng(1)
    # a few coordinates of every layer's weights and biases
    off = 0
    idx = []
    for ci, co, _, _, _ in UO.LAYERS:
        nw = co * 9 * ci
        idx += list(off + rng.choice(nw, 4, replace=False))
        idx += list(off + nw + rng.choice(co, min(co, 2), replace=False))
        off += nw + co
    h = 1e-6
    for k in idx:
        tp = theta.copy()
        tm = theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (_loss(tp, inp, tgt) - _loss(tm, inp, tgt)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(g[k])) + 1e-7, (k, fd, g[k])


def test_grid_transfers_are_adjoint():
    rng = np.random.default_rng(2)
    c = rng.standard_normal((2, 5, 5, 3))
    f = rng.standard_normal((2, 9, 9, 3))
    assert np.isclose(np.sum(UO.up(c) * f), np.sum(c * UO.up_T(f)))
    assert np.isclose(np.sum(UO.sub(f) * c), np.sum(f * UO.sub_T(c, 9)))
    # U interpolates bilinear functions exactly
    y, x = np.meshgrid(np.arange(5), np.arange(5), indexing="ij")
    lin = (2.0 * x + 3.0 * y + 0.5 * x * y)[None, :, :, None]
    yf, xf = np.meshgrid(np.arange(9) / 2.0, np.arange(9) / 2.0, indexing="ij")
    linf = (2.0 * xf + 3.0 * yf + 0.5 * xf * yf)[None, :, :, None]
    assert np.allclose(UO.up(lin), linf)


def test_bf16_emulation_close_to_exact():
    theta, inp, tgt = _problem(G=17, B=2, seed=3)
    y, c = UO.forward(theta, inp, exact=True)
    yb, cb = UO.forward(theta, inp, exact=False)
    assert np.linalg.norm(yb - y) <= 3e-2 * np.linalg.norm(y)
    _, dy = UO.mse(y, tgt)
    g = UO.backward(c, dy, exact=True)
    gb = UO.backward(cb, UO.mse(yb, tgt)[1], exact=False)
    assert np.linalg.norm(gb - g) <= 5e-2 * np.linalg.norm(g)


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0, 3.0e38])
    r = UO.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0          # tie -> even
    assert r[2] == 1.0 + 2 ** -7                 # above the tie -> up
    assert r[3] == -2.5 and r[4] == 0.0


def test_dilated_conv_gradients():
    """conv / conv_bwd with tap spacing 2 and 4 (the bottleneck layers): the data gradient is the
    adjoint of the convolution, the weight gradient matches central differences."""
    rng = np.random.default_rng(4)
    x = rng.standard_normal((2, 11, 11, 3))
    W = rng.standard_normal((4, 9, 3))
    b = rng.standard_normal(4)
    dy = rng.standard_normal((2, 11, 11, 4))
    for dil in (1, 2, 4):
        y = UO.conv(x, W, b, dil)
        dx, dW, db = UO.conv_bwd(x, W, dy, dil)
        # adjoint in x: <conv(x) - b, dy> = <x, dx>
        assert np.isclose(np.sum((y - b) * dy), np.sum(x * dx))
        assert np.allclose(db, dy.sum(axis=(0, 1, 2)))
        for (o, t, c) in [(0, 0, 0), (3, 8, 2), (1, 4, 1), (2, 2, 0)]:
            Wp = W.copy()
            Wm = W.copy()
            Wp[o, t, c] += 1e-6
            Wm[o, t, c] -= 1e-6
            fd = (np.sum(UO.conv(x, Wp, b, dil) * dy) - np.sum(UO.conv(x, Wm, b, dil) * dy)) / 2e-6
            assert abs(fd - dW[o, t, c]) <= 1e-5 * max(1.0, abs(fd))

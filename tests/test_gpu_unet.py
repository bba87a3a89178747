"""GPU parity of the learned warm-start network (fb_unet_*) with its CPU oracle.

The GPU runs BF16 GEMM operands with FP32 accumulation in a different summation order than the
oracle's BF16 emulation, so agreement is to BF16 noise: 2e-2 relative (L2) for the output and 5e-2
per parameter tensor for the gradients.  The oracle itself is pinned by finite differences
(test_unet_oracle)."""
import numpy as np
import pytest

import unet_oracle as UO

pytestmark = pytest.mark.gpu

FWD_TOL = 2e-2
GRAD_TOL = 5e-2


def _setup(torch, G, B, seed):
    from featb200.unet import UNet, init_params
    rng = np.random.default_rng(seed)
    theta = init_params(seed)
    theta = theta + (0.05 * rng.standard_normal(theta.size) * (theta == 0)).astype(np.float32)
    inp = rng.standard_normal((B, 2, G, G)).astype(np.float32)
    tgt = rng.standard_normal((B, G, G)).astype(np.float32)
    net = UNet(G, B, params=theta)
    return net, theta, inp, tgt, torch.tensor(inp, device="cuda"), torch.tensor(tgt, device="cuda")


def _layer_slices():
    out = []
    k = 0
    for ci, co, _, _, _ in UO.LAYERS:
        out.append(slice(k, k + co * 9 * ci))
        k += co * 9 * ci
        out.append(slice(k, k + co))
        k += co
    return out


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("G,B", [(17, 3), (33, 2), (129, 1)])
def test_forward_backward_match_oracle(featlib, cuda, G, B):
    torch = cuda
    net, theta, inp, tgt, inp_d, tgt_d = _setup(torch, G, B, seed=G)
    y = net.forward(inp_d)
    grad = torch.empty_like(y)
    loss = net.mse(y, tgt_d, grad)
    net.backward(grad)
    torch.cuda.synchronize()
    y_h = y.cpu().numpy()
    yo, cache = UO.forward(theta.astype(np.float64), inp, exact=False)
    assert _rel(y_h, yo) <= FWD_TOL
    l_ref, g_ref = UO.mse(y_h, tgt)
    assert abs(float(loss.item()) - l_ref) <= 1e-6 * l_ref
    assert np.allclose(grad.cpu().numpy(), g_ref, rtol=1e-5, atol=1e-12)
    go = UO.backward(cache, grad.cpu().numpy().astype(np.float64), exact=False)
    g = net.get_grads()
    for sl in _layer_slices():
        assert _rel(g[sl], go[sl]) <= GRAD_TOL, (sl, _rel(g[sl], go[sl]))


def test_backward_accumulates(featlib, cuda):
    torch = cuda
    net, theta, inp, tgt, inp_d, tgt_d = _setup(torch, 17, 2, seed=5)
    y = net.forward(inp_d)
    grad = torch.empty_like(y)
    net.mse(y, tgt_d, grad)
    net.backward(grad)
    g1 = net.get_grads()
    net.backward(grad, accumulate=True)
    g2 = net.get_grads()
    assert np.allclose(g2, 2.0 * g1, rtol=1e-6, atol=1e-12)


def test_adam_step_matches_formula(featlib, cuda):
    torch = cuda
    net, theta, inp, tgt, inp_d, tgt_d = _setup(torch, 17, 2, seed=6)
    y = net.forward(inp_d)
    grad = torch.empty_like(y)
    net.mse(y, tgt_d, grad)
    net.backward(grad)
    g = net.get_grads().astype(np.float64)
    p0 = net.get_params().astype(np.float64)
    lr, b1, b2, eps = 1e-3, 0.9, 0.999, 1e-8
    net.adam(lr, b1, b2, eps)
    p1 = net.get_params().astype(np.float64)
    m = (1 - b1) * g
    v = (1 - b2) * g * g
    ref = p0 - lr * (m / (1 - b1)) / (np.sqrt(v / (1 - b2)) + eps)
    assert np.allclose(p1, ref, rtol=1e-5, atol=1e-7)


def test_training_reduces_loss(featlib, cuda):
    """Adam on one fixed batch of a smooth target: the loss falls by an order of magnitude."""
    torch = cuda
    from featb200.unet import UNet
    G, B = 33, 4
    xs = np.linspace(0.0, 1.0, G)
    X, Y = np.meshgrid(xs, xs)
    rng = np.random.default_rng(9)
    inp = np.zeros((B, 2, G, G), np.float32)
    tgt = np.zeros((B, G, G), np.float32)
    for b in range(B):
        a, c = rng.uniform(0.5, 1.5, 2)
        inp[b, 0] = a * np.sin(np.pi * X) * np.sin(np.pi * Y)
        inp[b, 1] = c
        tgt[b] = a / c * np.sin(np.pi * X) * np.sin(np.pi * Y) / (2 * np.pi ** 2)
    tgt *= 10.0
    net = UNet(G, B, seed=1)
    inp_d = torch.tensor(inp, device="cuda")
    tgt_d = torch.tensor(tgt, device="cuda")
    g = torch.empty((B, G, G), dtype=torch.float32, device="cuda")
    first = float(net.train_step(inp_d, tgt_d, 3e-3, g).item())
    for _ in range(150):
        loss = net.train_step(inp_d, tgt_d, 3e-3, g)
    last = float(loss.item())
    assert np.isfinite(last) and last < 0.1 * first, (first, last)


def test_rejects_bad_arguments(featlib, cuda):
    from featb200.unet import UNet
    import featb200 as fb
    with pytest.raises(fb.FeatB200Error):
        UNet(20, 1)
    with pytest.raises(fb.FeatB200Error):
        UNet(5, 1)
    net = UNet(17, 2)
    x = cuda.zeros((3, 2, 17, 17), dtype=cuda.float32, device="cuda")
    with pytest.raises(fb.FeatB200Error):
        net.forward(x)

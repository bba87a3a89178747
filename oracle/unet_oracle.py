"""CPU oracle of the learned warm-start network (test infrastructure only: the tests import it as the
checker of the CUDA kernels in libfeatb200.so; the product never calls it).

A numpy restatement of the U-Net of fb_unet.cu: forward pass, backward pass (parameter gradients)
and the MSE loss, with the same parameter layout (per layer W[co][tap][ci], tap = (dy+1)*3 + dx+1,
then b[co]), the same grid transfers (injection S, bilinear vertex upsampling U) and the same
cross-correlation convention y[p] = sum_tap W[tap] x[p + off(tap)] with zero padding.

Two modes:
* exact=True: float64 throughout (checked against central finite differences);
* exact=False: BF16 rounding at the points the GPU rounds (input, weights, every activation and
  pre-activation gradient; FP32 data gradients; FP32 output), everything else in float64 -- the
  reference the GPU kernels are compared with (their FP32 accumulation order differs, so agreement
  is to BF16 noise, not bitwise).

The network has no counterpart in the reference (its solve path has no learned part); parity for it
is against this oracle, which is itself pinned by the finite-difference check.
"""
from __future__ import annotations

import numpy as np

# (cin, cout, level, relu, dilation): L1, L2, L3, L4 + two dilated bottleneck convolutions, L5..L8
LAYERS = [(2, 16, 0, True, 1), (16, 32, 1, True, 1), (32, 64, 2, True, 1), (64, 64, 3, True, 1),
          (64, 64, 3, True, 2), (64, 64, 3, True, 4), (128, 64, 2, True, 1), (96, 32, 1, True, 1),
          (48, 16, 0, True, 1), (16, 1, 0, False, 1)]


def num_params():
    return sum(co * 9 * ci + co for ci, co, _, _, _ in LAYERS)


def split_params(theta):
    """Flat vector -> [(W [co, 9, ci], b [co])] (views)."""
    out = []
    k = 0
    for ci, co, _, _, _ in LAYERS:
        W = theta[k:k + co * 9 * ci].reshape(co, 9, ci)
        k += co * 9 * ci
        b = theta[k:k + co]
        k += co
        out.append((W, b))
    return out


def bf16(a):
    """Round to BF16 (nearest even) through float32; returns float64 values."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(a):
    return np.asarray(a, dtype=np.float64).astype(np.float32).astype(np.float64)


def _shift(x, dy, dx):
    """s[:, y, x] = x[:, y + dy, x + dx] (zero outside)."""
    B, H, W, C = x.shape
    s = np.zeros_like(x)
    ys0, ys1 = max(0, -dy), min(H, H - dy)
    xs0, xs1 = max(0, -dx), min(W, W - dx)
    if ys0 < ys1 and xs0 < xs1:
        s[:, ys0:ys1, xs0:xs1] = x[:, ys0 + dy:ys1 + dy, xs0 + dx:xs1 + dx]
    return s


def _cols(x, dil=1):
    """im2col with tap spacing dil: [B, H, W, 9, C]."""
    return np.stack([_shift(x, (t // 3 - 1) * dil, (t % 3 - 1) * dil) for t in range(9)], axis=3)


def conv(x, W, b, dil=1):
    return np.einsum("bhwtc,otc->bhwo", _cols(x, dil), W, optimize=True) + b


def conv_bwd(x, W, dy, dil=1):
    """(dx, dW, db) of y = conv(x, W, b, dil) for upstream gradient dy."""
    cols = _cols(x, dil)
    dW = np.einsum("bhwo,bhwtc->otc", dy, cols, optimize=True)
    db = dy.sum(axis=(0, 1, 2))
    dx = np.zeros_like(x)
    for t in range(9):
        T = np.einsum("bhwo,oc->bhwc", dy, W[:, t, :], optimize=True)
        dx += _shift(T, -(t // 3 - 1) * dil, -(t % 3 - 1) * dil)
    return dx, dW, db


def sub(f):
    return f[:, ::2, ::2]


def sub_T(gc, Gf):
    B, _, _, C = gc.shape
    f = np.zeros((B, Gf, Gf, C))
    f[:, ::2, ::2] = gc
    return f


def _up_index(Gf):
    y = np.arange(Gf)
    y0 = y >> 1
    return y0, y0 + (y & 1)


def up(c, rnd=None):
    """Bilinear vertex upsampling: ((a00 + a01) + (a10 + a11)) * 0.25 per fine point."""
    Gc = c.shape[1]
    Gf = 2 * Gc - 1
    i0, i1 = _up_index(Gf)
    a00 = c[:, i0][:, :, i0]
    a01 = c[:, i0][:, :, i1]
    a10 = c[:, i1][:, :, i0]
    a11 = c[:, i1][:, :, i1]
    if rnd is None:
        return ((a00 + a01) + (a10 + a11)) * 0.25
    return rnd(f32(f32(f32(a00 + a01) + f32(a10 + a11)) * 0.25))


def up_T(gf):
    B, Gf, _, C = gf.shape
    Gc = (Gf + 1) // 2
    i0, i1 = _up_index(Gf)
    gc = np.zeros((B, Gc, Gc, C))
    q = 0.25 * gf
    for ya in (i0, i1):
        for xa in (i0, i1):
            np.add.at(gc, (slice(None), ya[:, None], xa[None, :]), q)
    return gc


def forward(theta, inp, exact=True):
    """inp: [B, 2, G, G] -> (out [B, G, G], cache)."""
    R = (lambda a: a) if exact else bf16
    P = [(R(W), b if exact else f32(b)) for W, b in split_params(np.asarray(theta, dtype=np.float64))]
    x = R(np.transpose(np.asarray(inp, dtype=np.float64), (0, 2, 3, 1)))
    cache = {"x": x, "P": P}

    def layer(l, a):
        W, b = P[l]
        pre = conv(a, W, b, LAYERS[l][4])
        return R(np.maximum(pre, 0.0)) if LAYERS[l][3] else pre

    e1 = layer(0, x)
    s1 = sub(e1)
    e2 = layer(1, s1)
    s2 = sub(e2)
    e3 = layer(2, s2)
    s3 = sub(e3)
    e4a = layer(3, s3)
    e4b = layer(4, e4a)
    e4 = layer(5, e4b)
    rup = None if exact else bf16
    c3 = np.concatenate([up(e4, rup), e3], axis=3)
    d3 = layer(6, c3)
    c2 = np.concatenate([up(d3, rup), e2], axis=3)
    d2 = layer(7, c2)
    c1 = np.concatenate([up(d2, rup), e1], axis=3)
    d1 = layer(8, c1)
    y = layer(9, d1)
    if not exact:
        y = f32(y)
    cache.update(e1=e1, s1=s1, e2=e2, s2=s2, e3=e3, s3=s3, e4a=e4a, e4b=e4b, e4=e4, c3=c3, d3=d3, c2=c2, d2=d2,
                 c1=c1, d1=d1)
    return y[..., 0], cache


def backward(cache, dout, exact=True):
    """Parameter gradients (flat, the layout of theta) for d loss / d out = dout [B, G, G]."""
    R = (lambda a: a) if exact else bf16
    F = (lambda a: a) if exact else f32
    P = cache["P"]
    grads = [None] * len(LAYERS)

    def bwd(l, a_in, dpre):
        W, _ = P[l]
        dx, dW, db = conv_bwd(a_in, W, dpre, LAYERS[l][4])
        grads[l] = (dW, db)
        return F(dx)

    def mask(post, g):
        return R(np.where(post > 0, g, 0.0))

    dy = R(np.asarray(dout, dtype=np.float64)[..., None])
    g_d1 = bwd(9, cache["d1"], dy)
    dc1 = bwd(8, cache["c1"], mask(cache["d1"], g_d1))
    G1 = dc1.shape[1]
    dc2 = bwd(7, cache["c2"], mask(cache["d2"], up_T(dc1[..., :32])))
    dc3 = bwd(6, cache["c3"], mask(cache["d3"], up_T(dc2[..., :64])))
    g_e4b = bwd(5, cache["e4b"], mask(cache["e4"], up_T(dc3[..., :64])))
    g_e4a = bwd(4, cache["e4a"], mask(cache["e4b"], g_e4b))
    g_s3 = bwd(3, cache["s3"], mask(cache["e4a"], g_e4a))
    G3 = dc3.shape[1]
    g_s2 = bwd(2, cache["s2"], mask(cache["e3"], dc3[..., 64:] + sub_T(g_s3, G3)))
    G2 = dc2.shape[1]
    g_s1 = bwd(1, cache["s1"], mask(cache["e2"], dc2[..., 64:] + sub_T(g_s2, G2)))
    bwd(0, cache["x"], mask(cache["e1"], dc1[..., 32:] + sub_T(g_s1, G1)))
    flat = []
    for dW, db in grads:
        flat.append(dW.ravel())
        flat.append(db.ravel())
    return np.concatenate(flat)


def mse(y, t):
    d = np.asarray(y, dtype=np.float64) - np.asarray(t, dtype=np.float64)
    return float(np.mean(d * d)), 2.0 * d / d.size

"""Host side of the learned warm start (fb_unet_* in libfeatb200.so).

``UNet`` owns the device network (FP32 master parameters, BF16 activations); its forward, backward,
loss and Adam step are the library's CUDA kernels, called on torch's current stream with CUDA
tensors.  There is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

# (cin, cout) of the ten convolutions, in parameter order (L1, L2, L3, L4, the two dilated
# bottleneck convolutions, L5, L6, L7, L8)
LAYERS = [(2, 16), (16, 32), (32, 64), (64, 64), (64, 64), (64, 64), (128, 64), (96, 32), (48, 16), (16, 1)]


def num_params():
    return sum(co * 9 * ci + co for ci, co in LAYERS)


def init_params(seed):
    """He-normal weights (std sqrt(2 / (9 cin))), zero biases; numpy PCG64 with `seed`."""
    rng = np.random.default_rng(seed)
    out = []
    for ci, co in LAYERS:
        out.append(rng.standard_normal(co * 9 * ci) * np.sqrt(2.0 / (9 * ci)))
        out.append(np.zeros(co))
    return np.concatenate(out).astype(np.float32)


class UNet:
    def __init__(self, grid, max_batch, params=None, seed=0):
        L = _lib.lib()
        h = C.c_void_p()
        _lib.check(L.fb_unet_create(C.byref(h), int(grid), int(max_batch)), "fb_unet_create")
        self._h = h
        self.grid = int(grid)
        self.max_batch = int(max_batch)
        n = C.c_uint64(0)
        _lib.check(L.fb_unet_num_params(h, C.byref(n)), "fb_unet_num_params")
        self.nparam = int(n.value)
        self.t = 0
        self.set_params(init_params(seed) if params is None else params)
        import torch
        self._loss = torch.zeros(1, dtype=torch.float64, device="cuda")

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                _lib.lib().fb_unet_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.nparam:
            raise ValueError("parameter count")
        _lib.check(_lib.lib().fb_unet_set_params(self._h, p.ctypes.data_as(C.c_void_p)), "fb_unet_set_params")
        self.t = 0

    def get_params(self):
        p = np.zeros(self.nparam, dtype=np.float32)
        _lib.check(_lib.lib().fb_unet_get_params(self._h, p.ctypes.data_as(C.c_void_p)), "fb_unet_get_params")
        return p

    def get_grads(self):
        g = np.zeros(self.nparam, dtype=np.float32)
        _lib.check(_lib.lib().fb_unet_get_grads(self._h, g.ctypes.data_as(C.c_void_p)), "fb_unet_get_grads")
        return g

    @staticmethod
    def _stream(stream):
        import torch
        return (stream or torch.cuda.current_stream()).cuda_stream

    def forward(self, inp, out=None, stream=None):
        """inp: CUDA float32 [B, 2, G, G] -> CUDA float32 [B, G, G]."""
        import torch
        B = int(inp.shape[0])
        if inp.dtype != torch.float32 or not inp.is_contiguous() or tuple(inp.shape[1:]) != (2, self.grid, self.grid):
            raise ValueError("input must be a contiguous float32 [B, 2, G, G] CUDA tensor")
        if out is None:
            out = torch.empty((B, self.grid, self.grid), dtype=torch.float32, device=inp.device)
        _lib.check(_lib.lib().fb_unet_forward(self._h, C.c_void_p(inp.data_ptr()), C.c_void_p(out.data_ptr()), B,
                                              C.c_void_p(self._stream(stream))), "fb_unet_forward")
        return out

    def backward(self, dout, accumulate=False, stream=None):
        _lib.check(_lib.lib().fb_unet_backward(self._h, C.c_void_p(dout.data_ptr()), int(dout.shape[0]),
                                               1 if accumulate else 0, C.c_void_p(self._stream(stream))),
                   "fb_unet_backward")

    def mse(self, y, t, grad=None, stream=None):
        """Device loss tensor (float64 [1]); writes d loss / d y into `grad` when given."""
        _lib.check(_lib.lib().fb_unet_mse(self._h, C.c_void_p(y.data_ptr()), C.c_void_p(t.data_ptr()),
                                          int(y.numel()), C.c_void_p(grad.data_ptr()) if grad is not None else None,
                                          C.c_void_p(self._loss.data_ptr()), C.c_void_p(self._stream(stream))),
                   "fb_unet_mse")
        return self._loss

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self.t += 1
        _lib.check(_lib.lib().fb_unet_adam(self._h, float(lr), float(beta1), float(beta2), float(eps), self.t,
                                           C.c_void_p(self._stream(stream))), "fb_unet_adam")

    def train_step(self, inp, target, lr, grad_buf=None, stream=None):
        """forward + MSE + backward + Adam; returns the device loss (before the update)."""
        import torch
        y = self.forward(inp, stream=stream)
        g = grad_buf if grad_buf is not None else torch.empty_like(y)
        loss = self.mse(y, target, g, stream=stream)
        self.backward(g, stream=stream)
        self.adam(lr, stream=stream)
        return loss


def _main():
    """A few training steps on random data (for profiling the network kernels):
    python -m featb200.unet --grid 129 --batch 32 --steps 5"""
    import argparse
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=129)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--steps", type=int, default=5)
    a = ap.parse_args()
    net = UNet(a.grid, a.batch, seed=0)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((a.batch, 2, a.grid, a.grid), device="cuda", generator=g)
    t = torch.randn((a.batch, a.grid, a.grid), device="cuda", generator=g)
    buf = torch.empty_like(t)
    for _ in range(a.steps):
        loss = net.train_step(x, t, 1e-3, buf)
    torch.cuda.synchronize()
    print({"loss": float(loss.item()), "steps": a.steps})


if __name__ == "__main__":
    _main()

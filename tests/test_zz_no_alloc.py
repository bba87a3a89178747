"""fb_dot_f64_noalloc: the dot product for callers that cannot allocate device memory (processes
that hand all device memory to their own pool at start-up, loops that must not stall on
cudaMalloc/cudaFree).  Called through the C ABI and compared with fb_dot_f64, twice in a row
(the shared scratch array keeps the previous call's contents), and its size limit is checked.
This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dot(lib, name, xd, yd, n):
    out = C.c_double()
    st = getattr(lib, name)(C.byref(out), C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), n, None)
    return st, out.value


def test_dot_noalloc_matches_dot(featlib, cuda):
    torch = cuda
    lib = featlib.lib()
    # the set-up call a caller makes before its pool takes the device memory: n = 0, null vectors
    out = C.c_double(1.0)
    assert lib.fb_dot_f64_noalloc(C.byref(out), None, None, 0, None) == 0, lib.fb_last_error()
    assert out.value == 0.0
    rng = np.random.default_rng(7)
    for n in (1, 4095, 4096, 4097, 1_000_003):
        x = rng.standard_normal(n)
        y = rng.standard_normal(n)
        xd = torch.tensor(x, device="cuda")
        yd = torch.tensor(y, device="cuda")
        torch.cuda.synchronize()
        st_ref, ref = _dot(lib, "fb_dot_f64", xd, yd, n)
        assert st_ref == 0
        tol = 1e-13 * float(np.abs(x * y).sum())
        for _ in range(2):                      # two calls in a row share the scratch array
            st, v = _dot(lib, "fb_dot_f64_noalloc", xd, yd, n)
            assert st == 0, lib.fb_last_error()
            assert abs(v - ref) <= tol
            assert abs(v - float(np.dot(x, y))) <= tol


def test_dot_noalloc_rejects_oversized(featlib, cuda):
    torch = cuda
    lib = featlib.lib()
    xd = torch.zeros(4, dtype=torch.float64, device="cuda")
    st, _ = _dot(lib, "fb_dot_f64_noalloc", xd, xd, 16_777_216 + 1)
    assert st == 1
    assert b"maximum" in lib.fb_last_error()

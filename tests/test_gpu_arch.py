"""GPU parity of the op-level seam (the LAFEM::Arch drop-ins) against the oracle and the
reference's known answers.  Device buffers are torch CUDA tensors (plumbing only)."""
import numpy as np
import pytest

from helpers import load_golden, rel_err

pytestmark = pytest.mark.gpu


def _t(torch, a, dtype=None):
    return torch.tensor(np.ascontiguousarray(a), device="cuda", dtype=dtype)


@pytest.mark.parametrize("index", ["u64", "u32"])
def test_apply_csr_bitwise(featlib, cuda, oracle_lib, index):
    """r = a A x + b y for alpha in {1, -1, 0, 4711.1}, r == y aliasing and the transposed form on
    the reference's level-5 Q1 matrix: non-transposed results are bitwise equal to the generic
    backend (Apply::csr_generic)."""
    torch = cuda
    fb = featlib
    A = load_golden("c1_L5")["levels"][0]["A"]
    n = A.shape[0]
    rng = np.random.default_rng(0)
    x = rng.standard_normal(n)
    y = rng.standard_normal(n)
    it = torch.int64 if index == "u64" else torch.int32
    val, col, rp = _t(torch, A.val), _t(torch, A.col_ind.astype(np.int64), it), _t(torch, A.row_ptr.astype(np.int64), it)
    xd, yd = _t(torch, x), _t(torch, y)
    for a, b in ((1.0, 0.0), (-1.0, 1.0), (0.5, 1.0), (4711.1, 1.0)):
        r = torch.empty_like(xd)
        fb.arch.apply_csr(r, a, xd, b, yd, val, col, rp, n)
        torch.cuda.synchronize()
        ref = oracle_lib.csr_apply(A, x, a, b, y)
        assert np.array_equal(r.cpu().numpy(), ref)
    r = yd.clone()
    fb.arch.apply_csr(r, -1.0, xd, 1.0, r, val, col, rp, n)
    assert np.array_equal(r.cpu().numpy(), oracle_lib.csr_apply(A, x, -1.0, 1.0, y))
    r = torch.empty_like(xd)
    fb.arch.apply_csr(r, 4711.1, xd, 1.0, yd, val, col, rp, n, transposed=True)
    ref = oracle_lib.csr_apply(A, x, 4711.1, 1.0, y, transposed=True)
    assert rel_err(r.cpu().numpy(), ref) <= 1e-14


def test_apply_csr_known_answer_f32(featlib, cuda):
    """kernel/lafem/sparse_matrix_csr-test.cpp:345-452 in FP32 (tolerances as in the reference)."""
    torch = cuda
    fb = featlib
    size = 1
    while size < 1000:
        i = np.arange(size)
        x = ((i % 100) * 1.234).astype(np.float32)
        y = (2.0 - (i % 42)).astype(np.float32)
        rows, cols, vals = [], [], []
        for r_ in range(size):
            for c in (r_ - 1, r_, r_ + 1):
                if 0 <= c < size:
                    rows.append(r_)
                    cols.append(c)
                    vals.append(2.0 if r_ == c else -1.0)
        rp = np.searchsorted(np.array(rows), np.arange(size + 1))
        Ad = (_t(torch, np.array(vals, np.float32)), _t(torch, np.array(cols), torch.int32), _t(torch, rp, torch.int32))
        A64 = np.zeros((size, size))
        A64[rows, cols] = vals
        xd, yd = _t(torch, x), _t(torch, y)
        r = torch.empty_like(xd)
        fb.arch.apply_csr(r, 4711.1, xd, 1.0, yd, *Ad, size)
        np.testing.assert_allclose(r.cpu().numpy(), 4711.1 * (A64 @ x) + y, atol=5e-2 * max(1, np.abs(A64 @ x).max()) / 1e2 + 5e-2, rtol=1e-5)
        fb.arch.apply_csr(r, 4711.1, xd, 1.0, yd, *Ad, size, transposed=True)
        np.testing.assert_allclose(r.cpu().numpy(), 4711.1 * (A64.T @ x) + y, atol=7e-2, rtol=1e-5)
        size *= 2


def test_blas1(featlib, cuda):
    torch = cuda
    fb = featlib
    rng = np.random.default_rng(1)
    n = 100003
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    xd, yd = _t(torch, x), _t(torch, y)
    r = torch.empty_like(xd)
    fb.arch.axpy(r, 0.3, xd, yd)
    assert np.array_equal(r.cpu().numpy(), 0.3 * x + y)
    r2 = xd.clone()
    fb.arch.axpy(r2, 0.3, r2, yd)                 # r == x
    assert np.array_equal(r2.cpu().numpy(), 0.3 * x + y)
    assert abs(fb.arch.dot(xd, yd) - np.dot(x, y)) <= 1e-13 * np.abs(x * y).sum()
    assert abs(fb.arch.norm2(xd) - np.linalg.norm(x)) <= 1e-14 * np.linalg.norm(x)
    fb.arch.component_product(r, xd, yd)
    assert np.array_equal(r.cpu().numpy(), x * y)
    fb.arch.component_invert(r, xd, 0.7)
    assert np.array_equal(r.cpu().numpy(), 0.7 / x)
    fb.arch.scale(r, xd, -2.5)
    assert np.array_equal(r.cpu().numpy(), x * -2.5)
    idx = np.array([0, 5, n - 1], dtype=np.int64)
    v = r.clone()
    fb.arch.unit_filter_rhs(v, _t(torch, [1.0, 2.0, 3.0]), _t(torch, idx))
    fb.arch.unit_filter_def(v, _t(torch, idx[:1]))
    vh = v.cpu().numpy()
    assert vh[0] == 0.0 and vh[5] == 2.0 and vh[-1] == 3.0
    f = torch.empty(n, dtype=torch.float32, device="cuda")
    fb.arch.convert(f, xd)
    assert np.array_equal(f.cpu().numpy(), x.astype(np.float32))
    assert abs(fb.arch.dot(f, f) - np.dot(x.astype(np.float32).astype(np.float64), x.astype(np.float32))) < 1e-8 * n


def test_diagonal(featlib, cuda):
    torch = cuda
    A = load_golden("c1_L4")["levels"][0]["A"]
    diag = torch.empty(A.shape[0], dtype=torch.int64, device="cuda")
    featlib.arch.diagonal_csr(diag, _t(torch, A.col_ind.astype(np.int64)), _t(torch, A.row_ptr.astype(np.int64)))
    d = diag.cpu().numpy()
    for r in range(A.shape[0]):
        assert A.col_ind[d[r]] == r


def test_pcg_jacobi_from_arch_known_answer(featlib, cuda):
    """The reference's PCG (kernel/solver/pcg.hpp:188-286) written over the op-level seam reproduces
    the reference's known answer on its own test problem (basic_solver-test.cpp:98-140):
    28 (+-2) iterations for CG and PCG-Jacobi, ||x - x_ref||^2 <= sqrt(eps)."""
    torch = cuda
    fb = featlib
    g = load_golden("fd17")["raw"]
    n = int(g["fd_A_shape"][0])
    val, col, rp = _t(torch, g["fd_A_val"]), _t(torch, g["fd_A_col_ind"].astype(np.int64)), \
        _t(torch, g["fd_A_row_ptr"].astype(np.int64))
    rhs = _t(torch, g["fd_rhs"])
    tol = np.sqrt(np.finfo(np.float64).eps)
    diag = torch.empty(n, dtype=torch.int64, device="cuda")
    fb.arch.diagonal_csr(diag, col, rp)
    inv = torch.empty(n, dtype=torch.float64, device="cuda")
    fb.arch.component_invert(inv, val[diag], 1.0)
    for jac, ref_iters in ((False, g_iters("cg_iters")), (True, g_iters("pcg_jac_iters"))):
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        r = torch.empty_like(x)
        fb.arch.apply_csr(r, -1.0, x, 1.0, rhs, val, col, rp, n)
        d0 = fb.arch.norm2(r)
        p = torch.empty_like(x)
        if jac:
            fb.arch.component_product(p, inv, r)
        else:
            p.copy_(r)
        gamma = fb.arch.dot(r, p)
        t = torch.empty_like(x)
        it = 0
        while True:
            fb.arch.apply_csr(t, 1.0, p, 0.0, t, val, col, rp, n)
            alpha = gamma / fb.arch.dot(t, p)
            fb.arch.axpy(x, alpha, p, x)
            fb.arch.axpy(r, -alpha, t, r)
            it += 1
            if fb.arch.norm2(r) <= tol * d0 or it >= 100:
                break
            if jac:
                fb.arch.component_product(t, inv, r)
            else:
                t.copy_(r)
            g2 = gamma
            gamma = fb.arch.dot(r, t)
            fb.arch.axpy(p, gamma / g2, p, t)
        assert abs(it - 28) <= 2 and abs(it - ref_iters) <= 1
        assert float(((x.cpu().numpy() - g["fd_ref"]) ** 2).sum()) <= tol


def g_iters(key):
    return load_golden("fd17")["summary"][key]

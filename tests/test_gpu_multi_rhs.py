"""Many right-hand sides with one hierarchy (fb_msolver_*): each right-hand side must follow the
single-RHS algorithm (same iterations, FP64 results within 1e-12 of the single-RHS solver and of the
reference), and the FP32 V-cycle variant stays within 1e-7 of FP64 at residual 1e-8."""
import numpy as np
import pytest

from helpers import load_golden, rel_err, to_lafem_levels

pytestmark = pytest.mark.gpu


def _rhs_family(level, dim, k, seed0=100):
    from featb200 import assembly as AS
    levels, _ = AS.poisson_hierarchy(level, dim, rhs="sine")
    fidx = levels[0]["filter"].indices.astype(np.int64)
    B = np.zeros((levels[0]["matrix"].rows(), k))
    for j in range(k):
        g = AS.gauss_params(seed0 + j, dim, width=(0.03, 0.12) if dim == 3 else (0.02, 0.1))
        b = AS.gauss_load_vector(level, g, dim)
        b[fidx] = 0.0
        B[:, j] = b
    return levels, B


@pytest.mark.parametrize("k,ordering", [(32, "native"), (64, "rcm")])
def test_multi_rhs_fp64_matches_single(featlib, cuda, k, ordering):
    fb = featlib
    levels, B = _rhs_family(3, 3, k)
    h = fb.build_hierarchy(levels)
    ms = fb.MultiRhsPCG(h, k, ordering=ordering)
    X = ms.solve(np.zeros_like(B), B)
    single = fb.build_pcg_multigrid(levels, ordering=ordering)
    for j in range(k):
        x = fb.DenseVector(B.shape[0])
        assert fb.solve(single, x, fb.DenseVector(B[:, j].copy())) == fb.Status.success
        assert ms.statuses()[j] == fb.Status.success
        assert ms.iterations()[j] == single.get_num_iter()
        assert rel_err(X[:, j], x.elements) <= 1e-12


def test_multi_rhs_reproduces_reference(featlib, cuda):
    """Column 0 = the reference's own 3D problem; its result matches the reference's solution."""
    fb = featlib
    g = load_golden("c3d_L3")
    lv = to_lafem_levels(g["levels"])
    h = fb.build_hierarchy(lv)
    ms = fb.MultiRhsPCG(h, 32)
    B = np.zeros((g["rhs"].size, 32))
    for j in range(32):
        B[:, j] = g["rhs"] * (1.0 + 0.25 * j)
    X = ms.solve(np.zeros_like(B), B)
    for j in range(32):
        assert ms.iterations()[j] == g["summary"]["iters"]
    assert rel_err(X[:, 0], g["sol"]) <= 1e-12


@pytest.mark.parametrize("level", [3, 6])
def test_multi_rhs_fp32_error(featlib, cuda, level):
    """The configured 3D case: level 6 (274,625 DOFs), 64 Gaussian right-hand sides, FP32 V-cycle
    inside FP64 PCG: residual <= 1e-8 and FP64 error <= 1e-7 for every right-hand side."""
    fb = featlib
    levels, B = _rhs_family(level, 3, 64)
    h = fb.build_hierarchy(levels)
    m64 = fb.MultiRhsPCG(h, 64, precision="f64")
    X64 = m64.solve(np.zeros_like(B), B)
    m32 = fb.MultiRhsPCG(h, 64, precision="f32")
    X32 = m32.solve(np.zeros_like(B), B)
    A = levels[0]["matrix"].to_scipy()
    fidx = levels[0]["filter"].indices.astype(np.int64)
    R = B - A @ X32
    R[fidx] = 0.0
    for j in range(64):
        assert m32.statuses()[j] == fb.Status.success
        assert np.linalg.norm(R[:, j]) <= 1.05e-8 * np.linalg.norm(B[:, j])
        assert rel_err(X32[:, j], X64[:, j]) <= 1e-7


@pytest.mark.parametrize("dim,level,precision", [(2, 5, "f64"), (3, 3, "f64"), (2, 6, "f32"), (3, 4, "f32")])
def test_multi_rhs_stencil_form(featlib, cuda, dim, level, precision):
    """Lexicographic Q1 levels run in the stencil form (strips of rows sharing their gathers, values
    without column indices).  Every row sum keeps the stored entry order; the per-RHS dot products
    are summed by FP64 atomics in an order that depends on the grid, so the two forms agree to
    rounding: FP64 within 1e-12 with the same iterations; with the FP32 V-cycle each form is within
    1e-7 of the FP64 solution, so the two within 2e-7."""
    fb = featlib
    levels, B = _rhs_family(level, dim, 64)
    h = fb.build_hierarchy(levels)
    out = {}
    for diag in (False, True):
        ms = fb.MultiRhsPCG(h, 64, precision=precision, ordering="native", stencil=diag)
        X = ms.solve(np.zeros_like(B), B)
        assert all(s == fb.Status.success for s in ms.statuses())
        out[diag] = (X, ms.iterations())
        ms.done()
    err = max(rel_err(out[True][0][:, j], out[False][0][:, j]) for j in range(64))
    if precision == "f64":
        assert err <= 1e-12, err
        assert out[True][1] == out[False][1]
    else:
        assert err <= 2e-7, err
        assert max(abs(a - b) for a, b in zip(out[True][1], out[False][1])) <= 1

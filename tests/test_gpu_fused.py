"""Fused V(2,2) passes on structured 2D levels (k_fz_down: pre-smoothing + defect + restriction;
k_fz_up: prolongation + both post-smoothing steps, with the skip test of the post-smoother resolved
by the last block).  The reference runs these steps one after the other
(kernel/solver/multigrid.hpp:1713-1838, :1845-2000, kernel/solver/richardson.hpp:187-228); the fused
passes must give the unfused V-cycle bit for bit in every precision, the FP64 V-cycle must equal the
oracle's, and the solves must agree (iteration counts equal; solutions within 1e-12 in FP64, where
only the order of the PCG's r.z sum differs)."""
import numpy as np
import pytest

from helpers import rel_err, to_oracle_levels

pytestmark = pytest.mark.gpu


def _problem(level, kappa=False, seed=4):
    from featb200 import assembly as AS
    field = AS.field_params(seed + 100) if kappa else None
    return AS.poisson_hierarchy(level, 2, rhs="gauss", gauss=AS.gauss_params(seed, 2), field=field)


def _solver(fb, levels, fused, precision="f64", **kw):
    return fb.build_pcg_multigrid(levels, precision=precision, ordering="native", fused=fused, **kw)


@pytest.mark.parametrize("level", [5, 7, 10])
@pytest.mark.parametrize("precision", ["f64", "f32", "f32_bf16"])
def test_fused_equals_unfused(featlib, cuda, level, precision):
    fb = featlib
    levels, b = _problem(level)
    s1 = _solver(fb, levels, True, precision)
    s0 = _solver(fb, levels, False, precision)
    z1 = s1.apply_precond(fb.DenseVector(b)).elements
    z0 = s0.apply_precond(fb.DenseVector(b)).elements
    assert np.array_equal(z1, z0)
    x1, x0 = fb.DenseVector(b.size), fb.DenseVector(b.size)
    assert fb.solve(s1, x1, fb.DenseVector(b)) == fb.Status.success
    assert fb.solve(s0, x0, fb.DenseVector(b)) == fb.Status.success
    assert s1.get_num_iter() == s0.get_num_iter()
    assert rel_err(x1.elements, x0.elements) <= (1e-12 if precision == "f64" else 1e-9)


@pytest.mark.parametrize("level,kappa", [(6, False), (8, True), (9, False)])
def test_fused_against_oracle(featlib, cuda, oracle_lib, level, kappa):
    """FP64 with the fused passes: the V-cycle bit for bit and the iterates within 1e-12 of the
    C restatement of the reference (which runs the steps one by one)."""
    fb = featlib
    levels, b = _problem(level, kappa)
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    x_ref, info = mg.solve(b)
    s = _solver(fb, levels, True)
    # the fused passes run on this problem's finest level
    s.time_kernel("mg_down", reps=1, flush_l2=False)
    s.time_kernel("mg_up", reps=1, flush_l2=False)
    assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, mg.vcycle(b))
    x = fb.DenseVector(b.size)
    assert fb.solve(s, x, fb.DenseVector(b)) == fb.Status.success
    assert s.get_num_iter() == info["iters"]
    assert rel_err(x.elements, x_ref) <= 1e-12
    for k in (1, 2):
        sk = fb.build_pcg_multigrid(levels, ordering="native", max_iter=k)
        xk = fb.DenseVector(b.size)
        fb.solve(sk, xk, fb.DenseVector(b))
        xk_ref, _ = mg.solve(b, max_iter=k)
        assert rel_err(xk.elements, xk_ref) <= 1e-12, k


@pytest.mark.parametrize("tail_rows", [0, 300, 5000])
def test_fused_tail_boundaries(featlib, cuda, oracle_lib, tail_rows):
    """The fused passes next to the single-block tail (which reads the restricted b, sol1 and skip
    flag they write) and without the tail (down to the coarsest level, which has no sol1)."""
    fb = featlib
    levels, b = _problem(7)
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    s = _solver(fb, levels, True, tail_rows=tail_rows)
    assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, mg.vcycle(b))


def test_fused_skip_fallback(featlib, cuda):
    """A zero defect: every smoother skips (its initial defect norm is zero), so the fused up pass's
    last block rewrites the level without the post-smoothing correction; the V-cycle returns zero
    like the unfused one, and the next, non-zero V-cycle is unaffected."""
    fb = featlib
    levels, b = _problem(6)
    s1 = _solver(fb, levels, True)
    s0 = _solver(fb, levels, False)
    zero = np.zeros_like(b)
    z1 = s1.apply_precond(fb.DenseVector(zero)).elements
    z0 = s0.apply_precond(fb.DenseVector(zero)).elements
    assert np.array_equal(z1, z0) and not np.any(z1)
    assert np.array_equal(s1.apply_precond(fb.DenseVector(b)).elements, s0.apply_precond(fb.DenseVector(b)).elements)


# ------------------------------------------------------------------ streamed form (k_fs_down / k_fs_up)
@pytest.mark.parametrize("level", [5, 7, 10])
@pytest.mark.parametrize("precision", ["f64", "f32", "f32_bf16"])
def test_streamed_equals_unfused(featlib, cuda, level, precision):
    """Every structured level streamed (fused tiles off), and the default split (tiles up to the
    fused threshold, streamed above), against one pass per step: the V-cycle bit for bit."""
    fb = featlib
    levels, b = _problem(level, kappa=True)
    s0 = _solver(fb, levels, False, precision)
    z0 = s0.apply_precond(fb.DenseVector(b)).elements
    for fused in (False, None):
        s1 = _solver(fb, levels, fused, precision, streamed=True)
        assert np.array_equal(s1.apply_precond(fb.DenseVector(b)).elements, z0), fused
    s1 = _solver(fb, levels, False, precision, streamed=True)
    x1, x0 = fb.DenseVector(b.size), fb.DenseVector(b.size)
    assert fb.solve(s1, x1, fb.DenseVector(b)) == fb.Status.success
    assert fb.solve(s0, x0, fb.DenseVector(b)) == fb.Status.success
    assert s1.get_num_iter() == s0.get_num_iter()
    assert rel_err(x1.elements, x0.elements) <= (1e-12 if precision == "f64" else 1e-9)


@pytest.mark.parametrize("level,kappa", [(6, False), (8, True), (9, False)])
def test_streamed_against_oracle(featlib, cuda, oracle_lib, level, kappa):
    """FP64, every structured level streamed: the V-cycle bit for bit and the iterates within 1e-12
    of the C restatement of the reference."""
    fb = featlib
    levels, b = _problem(level, kappa)
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    x_ref, info = mg.solve(b)
    s = _solver(fb, levels, False, streamed=True)
    s.time_kernel("mg_sdown", reps=1, flush_l2=False)
    s.time_kernel("mg_sup", reps=1, flush_l2=False)
    assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, mg.vcycle(b))
    x = fb.DenseVector(b.size)
    assert fb.solve(s, x, fb.DenseVector(b)) == fb.Status.success
    assert s.get_num_iter() == info["iters"]
    assert rel_err(x.elements, x_ref) <= 1e-12
    for k in (1, 2):
        sk = _solver(fb, levels, False, streamed=True, max_iter=k)
        xk = fb.DenseVector(b.size)
        fb.solve(sk, xk, fb.DenseVector(b))
        xk_ref, _ = mg.solve(b, max_iter=k)
        assert rel_err(xk.elements, xk_ref) <= 1e-12, k


@pytest.mark.parametrize("tail_rows", [0, 300, 5000])
def test_streamed_tail_boundaries(featlib, cuda, oracle_lib, tail_rows):
    fb = featlib
    levels, b = _problem(7)
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    s = _solver(fb, levels, False, streamed=True, tail_rows=tail_rows)
    assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, mg.vcycle(b))


def test_streamed_skip_fallback(featlib, cuda):
    """A zero defect through the streamed passes: the up pass's last block rewrites the level
    without the post-smoothing correction, as in the unfused cycle."""
    fb = featlib
    levels, b = _problem(6)
    s1 = _solver(fb, levels, False, streamed=True)
    s0 = _solver(fb, levels, False)
    zero = np.zeros_like(b)
    z1 = s1.apply_precond(fb.DenseVector(zero)).elements
    z0 = s0.apply_precond(fb.DenseVector(zero)).elements
    assert np.array_equal(z1, z0) and not np.any(z1)
    assert np.array_equal(s1.apply_precond(fb.DenseVector(b)).elements, s0.apply_precond(fb.DenseVector(b)).elements)

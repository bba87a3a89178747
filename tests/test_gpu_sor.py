"""SOR and SSOR smoothing on the device (the reference's SORPrecond / SSORPrecond inside Richardson,
kernel/solver/sor_precond.hpp:179-224, kernel/solver/ssor_precond.hpp; coloured sweeps of its CUDA
backend, kernel/solver/sor_precond.cu:26-41, ssor_precond.cu:25-60).

* sequential sweeps (dependency levels of the rows): the V-cycle bit for bit the reference's
  generic smoother (the C restatement, itself pinned bitwise to the reference binary), iterates
  and solution within 1e-12, also on the reference's own hierarchy against the reference binary;
* coloured sweeps (greedy colours): bit for bit the C restatement of the coloured algorithm with the
  same colouring;
* FP32 / BF16 V-cycles inside FP64 PCG: within 1e-7 of the FP64 oracle at residual 1e-8."""
import os

import numpy as np
import pytest

from helpers import rel_err, require_reference_binary, to_lafem_levels, to_oracle_levels

pytestmark = pytest.mark.gpu

PARITY = 1e-12


def _problem(level, dim=2, kappa=False, seed=6):
    from featb200 import assembly as AS
    field = AS.field_params(seed + 50) if kappa else None
    return AS.poisson_hierarchy(level, dim, rhs="gauss", gauss=AS.gauss_params(seed, dim), field=field)


@pytest.mark.parametrize("smoother", ["sor", "ssor"])
@pytest.mark.parametrize("omega", [1.0, 1.2])
@pytest.mark.parametrize("case", [(2, 6, False), (2, 7, True), (3, 4, False)], ids=["2d_l6", "2d_l7_kappa", "3d_l4"])
def test_sequential_sweeps_against_oracle(featlib, cuda, oracle_lib, smoother, omega, case):
    fb = featlib
    dim, level, kappa = case
    levels, b = _problem(level, dim, kappa)
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2, smoother=smoother, sor_omega=omega)
    x_ref, info = mg.solve(b)
    s = fb.build_pcg_multigrid(levels, smoother=smoother, smoother_omega=omega)
    assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, mg.vcycle(b))
    x = fb.DenseVector(b.size)
    assert fb.solve(s, x, fb.DenseVector(b)) == fb.Status.success
    assert s.get_num_iter() == info["iters"]
    assert rel_err(x.elements, x_ref) <= PARITY
    s2 = fb.build_pcg_multigrid(levels, smoother=smoother, smoother_omega=omega, max_iter=2)
    x2 = fb.DenseVector(b.size)
    fb.solve(s2, x2, fb.DenseVector(b))
    assert rel_err(x2.elements, mg.solve(b, max_iter=2)[0]) <= PARITY


@pytest.mark.parametrize("smoother", ["sor", "ssor"])
def test_sequential_sweeps_against_reference_binary(featlib, cuda, tmp_path, smoother):
    """The reference's own hierarchy (its numbering), solved by the reference binary with its SOR /
    SSOR smoother and by the device: same V-cycle, iterations and solution."""
    import oracle as O
    require_reference_binary()
    fb = featlib
    out = str(tmp_path / "ref")
    summ = O.feat_solve(out, dim=2, level=7, dump_levels=True, vcycle=True, iterates=2, smoother=smoother,
                        sor_omega=1.1)
    lv = to_lafem_levels(O.load_dump(out, 7))
    rhs = np.load(os.path.join(out, "rhs.npy"))
    s = fb.build_pcg_multigrid(lv, smoother=smoother, smoother_omega=1.1)
    assert np.array_equal(s.apply_precond(fb.DenseVector(rhs)).elements, np.load(os.path.join(out, "vcycle.npy")))
    x = fb.DenseVector(rhs.size)
    assert fb.solve(s, x, fb.DenseVector(rhs)) == fb.Status.success
    assert s.get_num_iter() == summ["iters"]
    assert rel_err(x.elements, np.load(os.path.join(out, "sol.npy"))) <= PARITY
    s2 = fb.build_pcg_multigrid(lv, smoother=smoother, smoother_omega=1.1, max_iter=2)
    x2 = fb.DenseVector(rhs.size)
    fb.solve(s2, x2, fb.DenseVector(rhs))
    assert rel_err(x2.elements, np.load(os.path.join(out, "iterate_2.npy"))) <= PARITY


@pytest.mark.parametrize("smoother", ["sor", "ssor"])
@pytest.mark.parametrize("level", [5, 8])
def test_coloured_sweeps_against_oracle(featlib, cuda, oracle_lib, smoother, level):
    fb = featlib
    levels, b = _problem(level, 2, kappa=True)
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2, smoother=smoother, sor_omega=1.0, coloured=True)
    x_ref, info = mg.solve(b)
    s = fb.build_pcg_multigrid(levels, smoother=smoother, smoother_omega=1.0, sweep="coloured")
    assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, mg.vcycle(b))
    x = fb.DenseVector(b.size)
    assert fb.solve(s, x, fb.DenseVector(b)) == fb.Status.success
    assert s.get_num_iter() == info["iters"]
    assert rel_err(x.elements, x_ref) <= PARITY


def test_sweeps_w_cycle_against_oracle(featlib, cuda, oracle_lib):
    fb = featlib
    levels, b = _problem(5, 2)
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2, cycle="W", smoother="ssor", sor_omega=1.0)
    s = fb.build_pcg_multigrid(levels, cycle="W", smoother="ssor", smoother_omega=1.0)
    assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, mg.vcycle(b))


@pytest.mark.parametrize("precision", ["f32", "f32_bf16"])
@pytest.mark.parametrize("sweep", ["sequential", "coloured"])
def test_sweeps_mixed_precision(featlib, cuda, oracle_lib, precision, sweep):
    fb = featlib
    levels, b = _problem(8, 2, kappa=True)
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2, smoother="sor", sor_omega=1.0)
    x_ref, _ = mg.solve(b)
    s = fb.build_pcg_multigrid(levels, precision=precision, smoother="sor", sweep=sweep)
    x = fb.DenseVector(b.size)
    assert fb.solve(s, x, fb.DenseVector(b)) == fb.Status.success
    A = levels[0]["matrix"].to_scipy()
    r = b - A @ x.elements
    r[levels[0]["filter"].indices.astype(np.int64)] = 0.0
    assert np.linalg.norm(r) <= 1.05e-8 * np.linalg.norm(b)
    assert rel_err(x.elements, x_ref) <= 1e-7


def test_sweeps_need_caller_numbering(featlib, cuda):
    fb = featlib
    levels, b = _problem(4, 2)
    with pytest.raises(fb.FeatB200Error):
        fb.build_pcg_multigrid(levels, ordering="rcm", smoother="sor")

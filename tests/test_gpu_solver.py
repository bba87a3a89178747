"""GPU parity of the solver seam (PCG + V-cycle) against the reference.

FP64 ("plain") mode: the V-cycle is bitwise equal to the reference (no global reductions inside it
other than the smoother's skip test), the PCG iterates and the solution agree to 1e-12 relative
(only the dot products and norms are summed in a different order).  Low-precision modes report
their error against the FP64 result (bound 1e-7 relative at residual 1e-8)."""
import os
import tempfile

import numpy as np
import pytest

from helpers import CASES, load_golden, rel_err, to_lafem_levels, to_oracle_levels, require_reference_binary

pytestmark = pytest.mark.gpu

PARITY = 1e-12


def _solve(fb, levels, rhs, **kw):
    s = fb.build_pcg_multigrid(levels, **kw)
    x = fb.DenseVector(rhs.size)
    st = fb.solve(s, x, fb.DenseVector(rhs))
    return s, x.elements, st


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("ordering,graph,tail,cluster", [("native", True, None, None), ("native", False, None, None),
                                                         ("rcm", True, None, None), ("native", True, None, 32767),
                                                         ("rcm", False, None, 32767), ("native", True, 0, 0),
                                                         ("rcm", False, 0, 0)])
def test_fp64_matches_reference(featlib, cuda, name, ordering, graph, tail, cluster):
    """Defaults: the coarse levels run in the single-block tail kernel; cluster 32767: every level
    below the finest in the cluster tail kernel; tail 0: one launch per pass."""
    fb = featlib
    g = load_golden(name)
    lv = to_lafem_levels(g["levels"])
    s, x, st = _solve(fb, lv, g["rhs"], ordering=ordering, use_graph=graph, tail_rows=tail, cluster_rows=cluster)
    z = s.apply_precond(fb.DenseVector(g["rhs"])).elements
    assert np.array_equal(z, g["vcycle"]), rel_err(z, g["vcycle"])
    assert st == fb.Status.success
    assert s.get_num_iter() == g["summary"]["iters"]
    assert rel_err(x, g["sol"]) <= PARITY
    assert abs(s.get_def_initial() - g["summary"]["def_init"]) <= PARITY * g["summary"]["def_init"]
    assert abs(s.get_def_final() - g["summary"]["def_final"]) <= 1e-9 * g["summary"]["def_final"]
    if ordering == "native" and graph:
        for k, xk_ref in enumerate(g["iterates"], start=1):
            sk, xk, stk = _solve(fb, lv, g["rhs"], ordering=ordering, use_graph=graph, max_iter=k, tail_rows=tail,
                                 cluster_rows=cluster)
            assert rel_err(xk, xk_ref) <= PARITY, k
            assert abs(sk.get_def_final() - g["defects"][k - 1]) <= 1e-9 * g["defects"][k - 1]


def _live_reference(tmp, level, dim=2, **kw):
    import oracle as O
    require_reference_binary()
    summ = O.feat_solve(tmp, dim=dim, level=level, dump_levels=True, vcycle=True, iterates=2, **kw)
    levels = O.load_dump(tmp, level)
    return summ, levels


@pytest.mark.parametrize("level,dim", [(7, 2), (9, 2), (5, 3)])
def test_fp64_matches_live_reference(featlib, cuda, level, dim):
    """Larger hierarchies straight from the reference's own assembly (reference numbering)."""
    import oracle as O
    from helpers import to_lafem_levels as conv
    fb = featlib
    with tempfile.TemporaryDirectory() as tmp:
        summ, levels = _live_reference(tmp, level, dim)
        rhs = np.load(os.path.join(tmp, "rhs.npy"))
        sol = np.load(os.path.join(tmp, "sol.npy"))
        vc = np.load(os.path.join(tmp, "vcycle.npy"))
        it2 = np.load(os.path.join(tmp, "iterate_2.npy"))
    lv = conv(levels)
    for ordering, tail, cluster in (("native", None, None), ("rcm", None, 32767), ("native", None, 32767),
                                    ("rcm", 0, 0)):
        s, x, st = _solve(fb, lv, rhs, ordering=ordering, tail_rows=tail, cluster_rows=cluster)
        assert np.array_equal(s.apply_precond(fb.DenseVector(rhs)).elements, vc)
        assert st == fb.Status.success and s.get_num_iter() == summ["iters"]
        assert rel_err(x, sol) <= PARITY
    s2, x2, _ = _solve(fb, lv, rhs, max_iter=2)
    assert rel_err(x2, it2) <= PARITY


def test_fp64_full_size_against_oracle(featlib, cuda, oracle_lib):
    """Level 10 (1,050,625 DOFs, Gaussian right-hand side): the product's own problem generator, the
    GPU solve and the C restatement on the same inputs."""
    from featb200 import assembly as AS
    fb = featlib
    levels, b = AS.poisson_hierarchy(10, 2, rhs="gauss", gauss=AS.gauss_params(1, 2))
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    x_ref, info = mg.solve(b)
    z_ref = mg.vcycle(b)
    # rcm: sliced ELL; native (lexicographic numbering): diagonal storage of the system matrices
    for ordering, diagonal in (("rcm", 1), ("native", 1), ("native", 0)):
        s, x, st = _solve(fb, levels, b, ordering=ordering, diagonal=diagonal)
        assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, z_ref), (ordering, diagonal)
        assert st == fb.Status.success and s.get_num_iter() == info["iters"]
        assert rel_err(x, x_ref) <= PARITY


@pytest.mark.parametrize("level", [6, 8])
@pytest.mark.parametrize("graph", [True, False])
def test_diagonal_storage_against_oracle(featlib, cuda, oracle_lib, level, graph):
    """Diagonal storage (native numbering of the generated problems): bitwise V-cycle and iterates
    against the C restatement, with and without the tail kernel, F and W cycles included."""
    from featb200 import assembly as AS
    fb = featlib
    levels, b = AS.poisson_hierarchy(level, 2, rhs="gauss", gauss=AS.gauss_params(2, 2))
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    x_ref, info = mg.solve(b)
    z_ref = mg.vcycle(b)
    for tail in (None, 0):
        s, x, st = _solve(fb, levels, b, use_graph=graph, tail_rows=tail, tma_rows=64)
        assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, z_ref), tail
        assert st == fb.Status.success and s.get_num_iter() == info["iters"]
        assert rel_err(x, x_ref) <= PARITY
    for cycle in ("F", "W"):
        s_e, x_e, _ = _solve(fb, levels, b, cycle=cycle, diagonal=0)
        s_d, x_d, _ = _solve(fb, levels, b, cycle=cycle, diagonal=1)
        assert np.array_equal(x_d, x_e) and s_d.get_num_iter() == s_e.get_num_iter()


@pytest.mark.parametrize("precision", ["f32", "f32_bf16"])
@pytest.mark.parametrize("level", [7, 10])
def test_mixed_precision_error_against_fp64(featlib, cuda, oracle_lib, precision, level):
    """FP32 (and BF16-value) V-cycle inside FP64 PCG: reaches relative residual 1e-8 and stays within
    1e-7 relative of the FP64 oracle's solution."""
    from featb200 import assembly as AS
    fb = featlib
    levels, b = AS.poisson_hierarchy(level, 2, rhs="gauss", gauss=AS.gauss_params(1, 2))
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    x_ref, info = mg.solve(b)
    s, x, st = _solve(fb, levels, b, precision=precision, ordering="rcm")
    assert st == fb.Status.success
    A = levels[0]["matrix"].to_scipy()
    r = b - A @ x
    r[levels[0]["filter"].indices.astype(np.int64)] = 0.0
    assert np.linalg.norm(r) <= 1.05e-8 * np.linalg.norm(b)
    assert rel_err(x, x_ref) <= 1e-7
    assert s.get_num_iter() <= info["iters"] + 2


def test_status_codes_without_fault(featlib, cuda):
    """Failure detection on the device, reported through the status word (no trap, no fault):
    zero rhs -> success after 0 iterations; NaN rhs -> aborted; max_iter reached -> max_iter."""
    fb = featlib
    g = load_golden("c1_L4")
    lv = to_lafem_levels(g["levels"])
    s = fb.build_pcg_multigrid(lv)
    x = fb.DenseVector(g["rhs"].size)
    assert fb.solve(s, x, fb.DenseVector(np.zeros_like(g["rhs"]))) == fb.Status.success
    assert s.get_num_iter() == 0 and np.all(x.elements == 0)
    bad = g["rhs"].copy()
    bad[bad.size // 2] = np.nan
    assert fb.solve(s, fb.DenseVector(bad.size), fb.DenseVector(bad)) == fb.Status.aborted
    s2 = fb.build_pcg_multigrid(lv, max_iter=2)
    assert fb.solve(s2, fb.DenseVector(bad.size), fb.DenseVector(g["rhs"])) == fb.Status.max_iter
    assert s2.get_num_iter() == 2
    # the context is still usable after the failures
    assert fb.solve(s, x, fb.DenseVector(g["rhs"])) == fb.Status.success


def test_device_entry_point_and_launch_count(featlib, cuda):
    """fb_solver_solve_device on torch CUDA tensors matches the host entry point; the library's
    launch counter advances by the reported number of kernels."""
    torch = cuda
    fb = featlib
    g = load_golden("c1_L5")
    lv = to_lafem_levels(g["levels"])
    s = fb.build_pcg_multigrid(lv, ordering="rcm")
    rhs = torch.tensor(g["rhs"], device="cuda")
    sol = torch.zeros_like(rhs)
    c0 = fb.launch_count()
    assert s.correct_device(sol, rhs) == fb.Status.success
    assert fb.launch_count() - c0 >= s.info.kernel_launches > 0
    assert rel_err(sol.cpu().numpy(), g["sol"]) <= PARITY


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("window,ordering", [(2, "native"), (1, "native"), (0, "native"), (1, "rcm"), (2, "rcm")])
def test_tma_staged_passes_match(featlib, cuda, name, precision, window, ordering):
    """The TMA-staged passes (bulk copies of matrix chunks into shared memory; window 1 also stages
    each chunk's window of the gathered vector there, window 2 prefetches it into L2) forced onto
    every level give the same results as
    the per-row kernels: bitwise V-cycles in FP64, identical iterations, solutions within rounding
    of the dot products."""
    fb = featlib
    g = load_golden(name)
    lv = to_lafem_levels(g["levels"])
    s_tma, x_tma, st1 = _solve(fb, lv, g["rhs"], precision=precision, tma_rows=32, tail_rows=0, cluster_rows=0,
                               tma_window=window, ordering=ordering)
    s_ref, x_ref, st2 = _solve(fb, lv, g["rhs"], precision=precision, tma_rows=0, tail_rows=0, cluster_rows=0,
                               ordering=ordering)
    assert st1 == st2 == fb.Status.success
    assert s_tma.get_num_iter() == s_ref.get_num_iter()
    z1 = s_tma.apply_precond(fb.DenseVector(g["rhs"])).elements
    z2 = s_ref.apply_precond(fb.DenseVector(g["rhs"])).elements
    assert np.array_equal(z1, z2)
    assert rel_err(x_tma, x_ref) <= (1e-12 if precision == "f64" else 1e-7)
    if precision == "f64":
        assert np.array_equal(z1, g["vcycle"])
        assert rel_err(x_tma, g["sol"]) <= PARITY


@pytest.mark.parametrize("ordering", ["native", "rcm"])
def test_tma_full_size(featlib, cuda, oracle_lib, ordering):
    """Level 10 with the default thresholds (TMA with staged vector windows on the large levels):
    bitwise V-cycle against the C oracle, solution within 1e-12."""
    from featb200 import assembly as AS
    fb = featlib
    levels, b = AS.poisson_hierarchy(10, 2, rhs="gauss", gauss=AS.gauss_params(3, 2))
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    x_ref, info = mg.solve(b)
    s, x, st = _solve(fb, levels, b, ordering=ordering)
    assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, mg.vcycle(b))
    assert st == fb.Status.success and s.get_num_iter() == info["iters"]
    assert rel_err(x, x_ref) <= PARITY


def test_cluster_tail_full_size(featlib, cuda, oracle_lib):
    """Level 10 with levels 7..1 in the cluster tail kernel (8 blocks, cluster barriers): bitwise
    V-cycle against the C oracle, same iterations, solution within 1e-12."""
    from featb200 import assembly as AS
    fb = featlib
    levels, b = AS.poisson_hierarchy(10, 2, rhs="gauss", gauss=AS.gauss_params(3, 2))
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    x_ref, info = mg.solve(b)
    s, x, st = _solve(fb, levels, b, ordering="rcm", cluster_rows=32767)
    assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, mg.vcycle(b))
    assert st == fb.Status.success and s.get_num_iter() == info["iters"]
    assert rel_err(x, x_ref) <= PARITY


@pytest.mark.parametrize("cycle", ["F", "W"])
@pytest.mark.parametrize("level,ordering,graph", [(5, "native", True), (6, "rcm", False)])
def test_fw_cycles_match_live_reference(featlib, cuda, cycle, level, ordering, graph):
    """F and W cycles (MultiGrid::_apply_cycle_f/_w) against the reference run with the same cycle:
    bitwise multigrid application, same PCG iterations, solution within 1e-12."""
    fb = featlib
    from helpers import to_lafem_levels as conv
    with tempfile.TemporaryDirectory() as tmp:
        summ, levels = _live_reference(tmp, level, 2, cycle=cycle.lower())
        rhs = np.load(os.path.join(tmp, "rhs.npy"))
        sol = np.load(os.path.join(tmp, "sol.npy"))
        vc = np.load(os.path.join(tmp, "vcycle.npy"))
    lv = conv(levels)
    # default tail threshold, no tail kernel, every level below the finest in the tail kernel
    for tail in (None, 0, 1 << 20):
        s, x, st = _solve(fb, lv, rhs, ordering=ordering, use_graph=graph, cycle=cycle, tail_rows=tail)
        assert np.array_equal(s.apply_precond(fb.DenseVector(rhs)).elements, vc), tail
        assert st == fb.Status.success and s.get_num_iter() == summ["iters"]
        assert rel_err(x, sol) <= PARITY


@pytest.mark.parametrize("cycle", ["F", "W"])
def test_fw_cycles_mixed_precision(featlib, cuda, cycle):
    from featb200 import assembly as AS
    fb = featlib
    levels, b = AS.poisson_hierarchy(8, 2, rhs="gauss", gauss=AS.gauss_params(5, 2))
    _, x64, st64 = _solve(fb, levels, b, cycle=cycle)
    s32, x32, st32 = _solve(fb, levels, b, cycle=cycle, precision="f32")
    assert st64 == st32 == fb.Status.success
    assert rel_err(x32, x64) <= 1e-7


@pytest.mark.parametrize("cgc", ["energy", "defect"])
@pytest.mark.parametrize("cycle", ["V", "F", "W"])
def test_adaptive_cgc_matches_live_reference(featlib, cuda, cgc, cycle):
    """MultiGridAdaptCGC::MinEnergy / MinDefect (multigrid.hpp:1880-1960) against the reference run with
    the same setting.  The step length comes from two dot products whose summation order differs
    from the reference's sequential loop, so the cycle agrees to rounding, not bitwise."""
    fb = featlib
    from helpers import to_lafem_levels as conv
    mode = {"energy": "MinEnergy", "defect": "MinDefect"}[cgc]
    with tempfile.TemporaryDirectory() as tmp:
        summ, levels = _live_reference(tmp, 6, 2, cycle=cycle.lower(), cgc=cgc)
        rhs = np.load(os.path.join(tmp, "rhs.npy"))
        sol = np.load(os.path.join(tmp, "sol.npy"))
        vc = np.load(os.path.join(tmp, "vcycle.npy"))
    lv = conv(levels)
    for tail, graph in ((None, True), (0, False), (1 << 20, True)):
        s, x, st = _solve(fb, lv, rhs, cycle=cycle, adapt_cgc=mode, tail_rows=tail, use_graph=graph)
        z = s.apply_precond(fb.DenseVector(rhs)).elements
        assert rel_err(z, vc) <= 1e-12, (tail, rel_err(z, vc))
        assert st == fb.Status.success and s.get_num_iter() == summ["iters"]
        assert rel_err(x, sol) <= 1e-11, (tail, rel_err(x, sol))


@pytest.mark.parametrize("cgc", ["MinEnergy", "MinDefect"])
def test_adaptive_cgc_mixed_precision(featlib, cuda, oracle_lib, cgc):
    from featb200 import assembly as AS
    fb = featlib
    levels, b = AS.poisson_hierarchy(9, 2, rhs="gauss", gauss=AS.gauss_params(4, 2))
    _, x64, st64 = _solve(fb, levels, b, adapt_cgc=cgc)
    _, x32, st32 = _solve(fb, levels, b, adapt_cgc=cgc, precision="f32")
    assert st64 == st32 == fb.Status.success
    assert rel_err(x32, x64) <= 1e-7


@pytest.mark.parametrize("graph", [True, False])
def test_diagonal_storage_3d_against_oracle(featlib, cuda, oracle_lib, graph):
    """3D Q1 (27 diagonals) in native numbering: the 27-wide diagonal-storage staged passes and row
    sums, bitwise V-cycle and iterates against the C restatement."""
    from featb200 import assembly as AS
    fb = featlib
    levels, b = AS.poisson_hierarchy(5, 3, rhs="gauss", gauss=AS.gauss_params(2, 3))
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    x_ref, info = mg.solve(b)
    z_ref = mg.vcycle(b)
    for tma in (None, 64):
        s, x, st = _solve(fb, levels, b, use_graph=graph, tma_rows=tma)
        assert np.array_equal(s.apply_precond(fb.DenseVector(b)).elements, z_ref), tma
        assert st == fb.Status.success and s.get_num_iter() == info["iters"]
        assert rel_err(x, x_ref) <= PARITY


@pytest.mark.parametrize("cycle", ["F", "W"])
@pytest.mark.parametrize("cgc", ["fixed", "energy", "defect"])
def test_cycles_diagonal_storage_against_oracle(featlib, cuda, oracle_lib, cycle, cgc):
    """F and W cycles, fixed and both adaptive coarse-grid corrections, on a lexicographically numbered
    problem (diagonal storage) against the C restatement: bitwise with the fixed correction, to
    1e-12 with the adaptive one (its step length sums dot products in another order)."""
    from featb200 import assembly as AS
    fb = featlib
    levels, b = AS.poisson_hierarchy(6, 2, rhs="gauss", gauss=AS.gauss_params(3, 2))
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2, cycle=cycle, cgc=cgc)
    x_ref, info = mg.solve(b)
    z_ref = mg.vcycle(b)
    mode = {"fixed": "Fixed", "energy": "MinEnergy", "defect": "MinDefect"}[cgc]
    s, x, st = _solve(fb, levels, b, cycle=cycle, adapt_cgc=mode, tma_rows=64)
    z = s.apply_precond(fb.DenseVector(b)).elements
    if cgc == "fixed":
        assert np.array_equal(z, z_ref)
    else:
        assert rel_err(z, z_ref) <= 1e-12
    assert st == fb.Status.success and s.get_num_iter() == info["iters"]
    assert rel_err(x, x_ref) <= 1e-11

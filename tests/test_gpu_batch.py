"""Batched uneven instances (fb_batch_*): every instance must follow its own single-system solve
(same iterations, FP64 results within 1e-12), including the reference's own problems, and the FP32
form stays within 1e-7 of FP64 at residual 1e-8."""
import numpy as np
import pytest

from helpers import load_golden, rel_err, to_lafem_levels

pytestmark = pytest.mark.gpu


def _family(levels_list, seed0=300, kappa=True):
    """Config-4 style instances: kappa = exp(random field), 8-Gaussian right-hand side."""
    from featb200 import assembly as AS
    out = []
    for k, L in enumerate(levels_list):
        field = AS.field_params(seed0 + 2 * k) if kappa else None
        lv, b = AS.poisson_hierarchy(L, 2, rhs="gauss", gauss=AS.gauss_params(seed0 + 2 * k + 1, 2), field=field)
        out.append((lv, b))
    return out


@pytest.mark.parametrize("ordering", ["native", "rcm"])
def test_batch_fp64_matches_single(featlib, cuda, ordering):
    fb = featlib
    inst = _family([4, 6, 3, 5, 4, 2])
    hs = [fb.build_hierarchy(lv) for lv, _ in inst]
    bat = fb.BatchPCG(hs, ordering=ordering)
    rhs = np.concatenate([b for _, b in inst])
    X = bat.split(bat.solve(np.zeros_like(rhs), rhs))
    for k, (lv, b) in enumerate(inst):
        s = fb.build_pcg_multigrid(lv, ordering=ordering)
        x = fb.DenseVector(b.size)
        assert fb.solve(s, x, fb.DenseVector(b)) == fb.Status.success
        assert bat.statuses()[k] == fb.Status.success
        assert bat.iterations()[k] == s.get_num_iter()
        assert rel_err(X[k], x.elements) <= 1e-12


def test_batch_reproduces_reference(featlib, cuda):
    """Instances straight from the reference's fixtures (reference numbering, noisy transfer
    matrices): each matches the reference's own solution."""
    fb = featlib
    names = ["c1_L4", "c1_L5", "gauss2d_L5", "kappa2d_L4"]
    gs = [load_golden(n) for n in names]
    hs = [fb.build_hierarchy(to_lafem_levels(g["levels"])) for g in gs]
    bat = fb.BatchPCG(hs)
    rhs = np.concatenate([g["rhs"] for g in gs])
    X = bat.split(bat.solve(np.zeros_like(rhs), rhs))
    for k, g in enumerate(gs):
        assert bat.iterations()[k] == g["summary"]["iters"]
        assert rel_err(X[k], g["sol"]) <= 1e-12


def test_batch_fp32_error(featlib, cuda):
    fb = featlib
    inst = _family([5, 7, 6, 8, 5, 9, 7, 6])
    hs = [fb.build_hierarchy(lv) for lv, _ in inst]
    rhs = np.concatenate([b for _, b in inst])
    b64 = fb.BatchPCG(hs, precision="f64")
    X64 = b64.split(b64.solve(np.zeros_like(rhs), rhs))
    b32 = fb.BatchPCG(hs, precision="f32")
    X32 = b32.split(b32.solve(np.zeros_like(rhs), rhs))
    for k, (lv, b) in enumerate(inst):
        assert b32.statuses()[k] == fb.Status.success
        A = lv[0]["matrix"].to_scipy()
        r = b - A @ X32[k]
        r[lv[0]["filter"].indices.astype(np.int64)] = 0.0
        assert np.linalg.norm(r) <= 1.05e-8 * np.linalg.norm(b)
        assert rel_err(X32[k], X64[k]) <= 1e-7


def test_batch_converged_instances_stop(featlib, cuda):
    """An instance with a zero right-hand side stops at iteration 0 while the others continue."""
    fb = featlib
    inst = _family([4, 5], kappa=False)
    hs = [fb.build_hierarchy(lv) for lv, _ in inst]
    bat = fb.BatchPCG(hs)
    rhs = np.concatenate([np.zeros_like(inst[0][1]), inst[1][1]])
    X = bat.split(bat.solve(np.zeros_like(rhs), rhs))
    assert bat.iterations()[0] == 0 and np.all(X[0] == 0)
    assert bat.statuses()[1] == fb.Status.success and bat.iterations()[1] > 0


@pytest.mark.parametrize("rows_per_block", [0, 64, 512])
def test_batch_rows_per_block(featlib, cuda, rows_per_block):
    """The autotuner (0) picks a block size per level from 64..512; any choice gives the same
    iterations and solutions as the single-system solves (block sizes change only which threads
    run which rows)."""
    fb = featlib
    inst = _family([5, 7, 3, 6], seed0=500)
    hs = [fb.build_hierarchy(lv) for lv, _ in inst]
    bat = fb.BatchPCG(hs, rows_per_block=rows_per_block)
    rpb = bat.rows_per_block()
    assert len(rpb) == 7
    if rows_per_block:
        assert np.all(rpb == rows_per_block)
    else:
        assert set(rpb.tolist()) <= {64, 128, 256, 512}
    rhs = np.concatenate([b for _, b in inst])
    X = bat.split(bat.solve(np.zeros_like(rhs), rhs))
    for k, (lv, b) in enumerate(inst):
        s = fb.build_pcg_multigrid(lv)
        x = fb.DenseVector(b.size)
        assert fb.solve(s, x, fb.DenseVector(b)) == fb.Status.success
        assert bat.iterations()[k] == s.get_num_iter()
        assert rel_err(X[k], x.elements) <= 1e-12

"""The layered forms at their configured sizes, each against the FP64 oracle.

* Many right-hand sides: 3D Q1 unit cube, level 6 (274,625 DOFs, 27-point stencil), 64 right-hand
  sides of 8 seeded Gaussians each, solved together (fb_msolver).  Sampled columns against the C
  restatement of the reference's PCG + V-cycle (iteration counts, iterates 1 and 2, final solution
  within 1e-12 in FP64; FP32 V-cycle within 1e-7 of that oracle at residual 1e-8), and one column
  on the reference's own hierarchy and load vector against the reference binary's solution.
* Uneven instances: all 256 instances of the batch (levels 5..9, kappa = exp(random field)), solved
  together (fb_batch).  One instance per level against the C restatement (FP64 within 1e-12, FP32
  within 1e-7), every instance's FP32 result within 1e-7 of its FP64 result, and one level-7
  instance on the reference's own kappa-weighted assembly against the reference binary.

The reference's PCG is kernel/solver/pcg.hpp:188-286 and its V-cycle kernel/solver/multigrid.hpp:
1335-1350; the oracle restates both (oracle/mg_oracle.c)."""
import multiprocessing as mp
import os
import tempfile

import numpy as np
import pytest

from helpers import rel_err, require_reference_binary, to_lafem_levels, to_oracle_levels

pytestmark = pytest.mark.gpu

PARITY = 1e-12
MIXED = 1e-7


def _residual_ok(levels, b, x, tol=1.05e-8):
    A = levels[0]["matrix"].to_scipy()
    r = b - A @ x
    r[levels[0]["filter"].indices.astype(np.int64)] = 0.0
    return np.linalg.norm(r) <= tol * np.linalg.norm(b)


# ------------------------------------------------------------------------------ many right-hand sides
@pytest.fixture(scope="module")
def rhs64_l6():
    from featb200 import assembly as AS
    return AS.rhs64_family(6, 3, 64)


def test_multi_rhs_l6_against_oracle(featlib, cuda, oracle_lib, rhs64_l6):
    fb = featlib
    levels, B = rhs64_l6
    h = fb.build_hierarchy(levels)
    m64 = fb.MultiRhsPCG(h, 64, precision="f64")
    X64 = m64.solve(np.zeros_like(B), B)
    m32 = fb.MultiRhsPCG(h, 64, precision="f32")
    X32 = m32.solve(np.zeros_like(B), B)
    assert all(s == fb.Status.success for s in m64.statuses())
    assert all(s == fb.Status.success for s in m32.statuses())
    mg = oracle_lib.MultigridPCG(to_oracle_levels(levels), 0.7, 2)
    cols = (0, 31, 63)
    refs = {}
    for j in cols:
        x_ref, info = mg.solve(B[:, j])
        refs[j] = x_ref
        assert info["status"] == "success"
        assert m64.iterations()[j] == info["iters"], j
        assert rel_err(X64[:, j], x_ref) <= PARITY, j
        assert rel_err(X32[:, j], x_ref) <= MIXED, j
        assert _residual_ok(levels, B[:, j], X32[:, j]), j
    for k in (1, 2):
        mk = fb.MultiRhsPCG(h, 64, precision="f64", max_iter=k)
        Xk = mk.solve(np.zeros_like(B), B)
        for j in cols:
            xk_ref, _ = mg.solve(B[:, j], max_iter=k)
            assert rel_err(Xk[:, j], xk_ref) <= PARITY, (k, j)


def test_multi_rhs_l6_reference_column(featlib, cuda, tmp_path):
    """Column 0 of the set assembled by the reference itself (its mesh hierarchy, numbering and
    load vector); the other 63 columns are the same load vector scaled.  Column 0 reproduces the
    reference binary's solution and iteration count."""
    import oracle as O
    from featb200 import assembly as AS
    require_reference_binary()
    fb = featlib
    params = str(tmp_path / "g.txt")
    AS.write_params(params, gauss=AS.rhs64_params(0, 3))
    out = str(tmp_path / "ref")
    summ = O.feat_solve(out, dim=3, level=6, rhs="gauss", params=params, dump_levels=True)
    lv = to_lafem_levels(O.load_dump(out, 6))
    rhs = np.load(os.path.join(out, "rhs.npy"))
    sol = np.load(os.path.join(out, "sol.npy"))
    B = np.outer(rhs, 1.0 + 0.125 * np.arange(64))
    ms = fb.MultiRhsPCG(fb.build_hierarchy(lv), 64, precision="f64", ordering="rcm")
    X = ms.solve(np.zeros_like(B), B)
    assert ms.iterations()[0] == summ["iters"]
    assert rel_err(X[:, 0], sol) <= PARITY


# ------------------------------------------------------------------------------ uneven instances
@pytest.fixture(scope="module")
def batch256():
    from featb200 import assembly as AS
    levels = AS.batch_family_levels()
    # set-up only (host assembly); spawn-started, so the workers hold no CUDA state
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        inst = pool.starmap(AS.batch_instance, [(L, k) for k, L in enumerate(levels)])
    return levels, inst


def test_batch256_against_oracle(featlib, cuda, oracle_lib, batch256):
    fb = featlib
    levels, inst = batch256
    hs = [fb.build_hierarchy(lv) for lv, _ in inst]
    rhs = np.concatenate([b for _, b in inst])
    b64 = fb.BatchPCG(hs, precision="f64")
    X64 = b64.split(b64.solve(np.zeros_like(rhs), rhs))
    b32 = fb.BatchPCG(hs, precision="f32")
    X32 = b32.split(b32.solve(np.zeros_like(rhs), rhs))
    assert all(s == fb.Status.success for s in b64.statuses())
    assert all(s == fb.Status.success for s in b32.statuses())
    for k in range(len(inst)):
        assert rel_err(X32[k], X64[k]) <= MIXED, k
    sample = {L: levels.index(L) for L in range(5, 10)}
    b2 = fb.BatchPCG(hs, precision="f64", max_iter=2)
    X2 = b2.split(b2.solve(np.zeros_like(rhs), rhs))
    for L, k in sample.items():
        lv, b = inst[k]
        mg = oracle_lib.MultigridPCG(to_oracle_levels(lv), 0.7, 2)
        x_ref, info = mg.solve(b)
        assert info["status"] == "success"
        assert b64.iterations()[k] == info["iters"], L
        assert rel_err(X64[k], x_ref) <= PARITY, L
        assert rel_err(X32[k], x_ref) <= MIXED, L
        assert _residual_ok(lv, b, X32[k]), L
        x2_ref, _ = mg.solve(b, max_iter=2)
        assert rel_err(X2[k], x2_ref) <= PARITY, L


def test_batch_kappa_reference_instance(featlib, cuda, tmp_path, batch256):
    """A level-7 instance of the batch assembled by the reference itself (kappa-weighted operator,
    its numbering), solved inside a batch with three lexicographic instances of other levels:
    it reproduces the reference binary's solution and iteration count."""
    import oracle as O
    from featb200 import assembly as AS
    require_reference_binary()
    fb = featlib
    levels, inst = batch256
    k7 = levels.index(7)
    g, f = AS.batch_instance_params(k7)
    gp, kp = str(tmp_path / "g.txt"), str(tmp_path / "k.txt")
    AS.write_params(gp, gauss=g)
    AS.write_params(kp, field=f)
    out = str(tmp_path / "ref")
    summ = O.feat_solve(out, dim=2, level=7, rhs="gauss", params=gp, kappa=kp, dump_levels=True)
    lv = to_lafem_levels(O.load_dump(out, 7))
    rhs = np.load(os.path.join(out, "rhs.npy"))
    sol = np.load(os.path.join(out, "sol.npy"))
    others = [inst[levels.index(L)] for L in (5, 9, 6)]
    hs = [fb.build_hierarchy(lv)] + [fb.build_hierarchy(o[0]) for o in others]
    bat = fb.BatchPCG(hs, precision="f64")
    packed = np.concatenate([rhs] + [o[1] for o in others])
    X = bat.split(bat.solve(np.zeros_like(packed), packed))
    assert bat.iterations()[0] == summ["iters"]
    assert rel_err(X[0], sol) <= PARITY

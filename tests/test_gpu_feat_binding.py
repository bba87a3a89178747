"""The library behind the reference's own API: FEAT compiled as a CUDA build whose CUDA backend is
the library's FEAT binding (feat3.doxytest_b200/feat/featb200_backend.cpp in place of FEAT's
kernel/util/cuda_util.cu and kernel/lafem/arch/*.cu, linked with libfeatb200.so), built by
oracle/Makefile into oracle/_ref/feat_b200.  Every FEAT container then lives in the managed memory
MemoryPool allocates in CUDA builds (kernel/util/memory_pool.hpp:79-104).

* op seam: FEAT's own Solver::PCG + Solver::MultiGrid + Richardson + JacobiPrecond with
  Backend::set_preferred_backend(PreferredBackend::cuda), so every LAFEM op (Apply::csr, Axpy,
  DotProduct, Norm2, ComponentProduct, ComponentInvert, UnitFilter, Diagonal, set_memory, copy)
  runs on the library (kernel/backend.hpp:55-92 dispatch).  The V-cycle is bitwise the generic
  backend's (rows summed in stored order, no FMA; FP64 products not rounded through float), PCG's
  iterates within 1e-12 (its dot products are tree-summed).
* solver seam: the whole solve handed to the library's solver object (featb200_solver.hpp), built
  from FEAT's MultiGridHierarchy: iterates and solution within 1e-12, same iteration counts.
Both are compared with the reference built from its sources with the generic backend
(oracle/_ref/feat_oracle) on the same problem."""
import json
import os

import numpy as np
import pytest

from helpers import rel_err, require_reference_binary

pytestmark = pytest.mark.gpu

PARITY = 1e-12


def _require_b200_binary():
    import oracle as O
    require_reference_binary()
    if not O.feat_b200_available():
        if os.environ.get("FEATB200_REQUIRE_REF") == "1":
            pytest.fail("oracle/_ref/feat_b200 not built (FEATB200_REQUIRE_REF=1)")
        pytest.skip("oracle/_ref/feat_b200 not built")


def _run(tmp_path, name, **kw):
    import oracle as O
    out = str(tmp_path / name)
    summ = O.feat_solve(out, iterates=2, **kw)
    ld = lambda f: np.load(os.path.join(out, f))
    res = {"summ": summ, "sol": ld("sol.npy"), "it1": ld("iterate_1.npy"), "it2": ld("iterate_2.npy")}
    if os.path.exists(os.path.join(out, "vcycle.npy")):
        res["vcycle"] = ld("vcycle.npy")
    return res


CASES = [dict(dim=2, level=7), dict(dim=3, level=4), dict(dim=2, level=6, rhs="gauss", kappa=True)]


def _case_kwargs(tmp_path, case):
    from featb200 import assembly as AS
    kw = dict(dim=case["dim"], level=case["level"], rhs=case.get("rhs", "sine"))
    if kw["rhs"] == "gauss":
        g, f = AS.batch_instance_params(3)
        kw["params"] = str(tmp_path / "g.txt")
        AS.write_params(kw["params"], gauss=g)
        if case.get("kappa"):
            kw["kappa"] = str(tmp_path / "k.txt")
            AS.write_params(kw["kappa"], field=f)
    return kw


@pytest.mark.parametrize("case", CASES, ids=["2d_l7", "3d_l4", "2d_l6_kappa"])
def test_feat_ops_on_library(featlib, cuda, tmp_path, case):
    _require_b200_binary()
    kw = _case_kwargs(tmp_path, case)
    ref = _run(tmp_path, "generic", vcycle=True, **kw)
    ops = _run(tmp_path, "ops", vcycle=True, b200="ops", **kw)
    assert ops["summ"]["backend"] == "b200" and ops["summ"]["solver"] == "feat"
    assert ops["summ"]["status"] == "success"
    assert np.array_equal(ops["vcycle"], ref["vcycle"])
    assert ops["summ"]["iters"] == ref["summ"]["iters"]
    assert rel_err(ops["it1"], ref["it1"]) <= PARITY
    assert rel_err(ops["it2"], ref["it2"]) <= PARITY
    assert rel_err(ops["sol"], ref["sol"]) <= PARITY
    assert abs(ops["summ"]["def_init"] - ref["summ"]["def_init"]) <= PARITY * ref["summ"]["def_init"]


@pytest.mark.parametrize("case", CASES, ids=["2d_l7", "3d_l4", "2d_l6_kappa"])
def test_feat_solver_object_on_library(featlib, cuda, tmp_path, case):
    _require_b200_binary()
    kw = _case_kwargs(tmp_path, case)
    ref = _run(tmp_path, "generic", **kw)
    sv = _run(tmp_path, "solver", b200="solver", **kw)
    assert sv["summ"]["solver"] == "b200" and sv["summ"]["status"] == "success"
    assert sv["summ"]["iters"] == ref["summ"]["iters"]
    assert rel_err(sv["it1"], ref["it1"]) <= PARITY
    assert rel_err(sv["it2"], ref["it2"]) <= PARITY
    assert rel_err(sv["sol"], ref["sol"]) <= PARITY
    assert abs(sv["summ"]["def_final"] - ref["summ"]["def_final"]) <= 1e-9 * ref["summ"]["def_final"]


def test_feat_generic_on_managed_memory(featlib, cuda, tmp_path):
    """The CUDA build with the generic backend (containers in managed memory, ops on the host):
    bit for bit the reference build, so the managed allocations themselves change nothing."""
    import subprocess
    import oracle as O
    _require_b200_binary()
    out_r, out_g = str(tmp_path / "r"), str(tmp_path / "g")
    O.feat_solve(out_r, dim=2, level=6, vcycle=True)
    os.makedirs(out_g, exist_ok=True)
    res = subprocess.run([O.FEAT_B200_BIN, "solve", "--dim", "2", "--level", "6", "--out", out_g, "--vcycle"],
                         check=True, capture_output=True, text=True, timeout=600)
    summ = json.loads(res.stdout.strip().splitlines()[-1])
    assert summ["backend"] == "generic" and summ["solver"] == "feat"
    for f in ("vcycle.npy", "sol.npy"):
        assert np.array_equal(np.load(os.path.join(out_g, f)), np.load(os.path.join(out_r, f)))


def test_feat_own_cuda_backend(featlib, cuda, tmp_path):
    """FEAT built on its own CUDA backend (oracle/_ref/feat_cuda: cuSPARSE SpMV, cuBLAS vector ops) and
    run with Backend::set_preferred_backend(cuda) solves the same problem as the generic build (its
    sums are ordered differently, so to solver tolerance, not bitwise): the problem behind the
    reference GPU timing column."""
    import oracle as O
    require_reference_binary()
    if not O.feat_cuda_available():
        if os.environ.get("FEATB200_REQUIRE_REF") == "1":
            pytest.fail("oracle/_ref/feat_cuda not built (FEATB200_REQUIRE_REF=1)")
        pytest.skip("oracle/_ref/feat_cuda not built")
    ref = _run(tmp_path, "generic", dim=2, level=7)
    cu = _run(tmp_path, "cuda", dim=2, level=7, b200="cuda")
    assert cu["summ"]["backend"] == "cuda" and cu["summ"]["status"] == "success"
    assert abs(cu["summ"]["iters"] - ref["summ"]["iters"]) <= 1
    assert rel_err(cu["sol"], ref["sol"]) <= 1e-7

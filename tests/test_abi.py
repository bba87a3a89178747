"""The C ABI without a GPU: the library loads, exports every entry point include/featb200.h
declares, and its host-side validation rejects malformed input like the reference's XASSERTs."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(fb_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol(featlib):
    lib = featlib.lib()
    declared = _declared()
    assert len(declared) >= 36
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # the Python mirror binds every declared entry point
    assert declared <= set(featlib.exported_symbols())


def test_built_for_sm100a(featlib):
    assert b"sm_100a" in featlib.lib().fb_version()


def test_no_cpu_fallback(featlib, monkeypatch, tmp_path):
    from featb200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(_lib.FeatB200Error):
        _lib.lib()


def test_config_defaults_match_reference(featlib):
    """IterativeSolver defaults (kernel/solver/iterative.hpp:200-235) and the configured V(2,2)."""
    from featb200 import _lib
    cfg = _lib.SolverConfig()
    featlib.lib().fb_solver_config_default(C.byref(cfg))
    eps = np.finfo(np.float64).eps
    assert cfg.tol_rel == 1e-8 and cfg.max_iter == 100 and cfg.min_iter == 0
    assert cfg.tol_abs == 1.0 / eps ** 2
    assert cfg.omega == 0.7 and cfg.smooth_steps == 2 and cfg.precision == 0
    # the multigrid's own defaults (multigrid.hpp:1068-1075): V cycle, fixed coarse-grid correction;
    # device choices on by default: diagonal storage where it applies, programmatic dependent launch
    assert cfg.cycle == 0 and cfg.adapt_cgc == 0
    assert cfg.diagonal == 1 and cfg.pdl == 1 and cfg.tail_rows == 300 and cfg.tma_rows == 1000


def _csr(rp, ci, val, shape):
    from featb200 import _lib
    keep = [np.ascontiguousarray(rp, dtype=np.uint64), np.ascontiguousarray(ci, dtype=np.uint64),
            np.ascontiguousarray(val, dtype=np.float64)]
    c = _lib.CsrHost(shape[0], shape[1], keep[2].size, keep[0].ctypes.data_as(C.c_void_p),
                     keep[1].ctypes.data_as(C.c_void_p), keep[2].ctypes.data_as(C.c_void_p))
    return c, keep


def test_hierarchy_validation(featlib):
    """Host-side checks run before anything touches a device."""
    from featb200 import _lib
    L = featlib.lib()
    h = C.c_void_p()
    assert L.fb_hierarchy_create(C.byref(h), 0) == 1
    assert L.fb_hierarchy_create(C.byref(h), 2) == 0
    fidx = np.zeros(0, dtype=np.uint64)
    ok, k1 = _csr([0, 1, 2], [0, 1], [2.0, 2.0], (2, 2))
    bad_rp, k2 = _csr([0, 2, 1], [0, 1], [2.0, 2.0], (2, 2))
    bad_col, k3 = _csr([0, 1, 2], [0, 5], [2.0, 2.0], (2, 2))
    # fine level without transfer matrices
    assert L.fb_hierarchy_set_level(h, 0, C.byref(ok), fidx.ctypes.data_as(C.c_void_p), None, 0, None, None) == 1
    assert b"P and R" in L.fb_last_error()
    # coarsest level with a non-monotone row pointer / out-of-range column
    assert L.fb_hierarchy_set_level(h, 1, C.byref(bad_rp), fidx.ctypes.data_as(C.c_void_p), None, 0, None, None) == 1
    assert b"row_ptr" in L.fb_last_error()
    assert L.fb_hierarchy_set_level(h, 1, C.byref(bad_col), fidx.ctypes.data_as(C.c_void_p), None, 0, None, None) == 1
    assert b"column" in L.fb_last_error()
    bad_f = np.array([7], dtype=np.uint64)
    assert L.fb_hierarchy_set_level(h, 1, C.byref(ok), bad_f.ctypes.data_as(C.c_void_p), None, 1, None, None) == 1
    assert b"filter" in L.fb_last_error()
    assert L.fb_hierarchy_set_level(h, 1, C.byref(ok), fidx.ctypes.data_as(C.c_void_p), None, 0, None, None) == 0
    # a solver cannot be built before every level is set
    s = C.c_void_p()
    assert L.fb_solver_create(C.byref(s), h, None) == 3
    L.fb_hierarchy_destroy(h)


def test_python_mirror_rejects_unsupported_configurations(featlib):
    """The mirror refuses configurations the device V-cycle does not implement instead of
    silently running something else."""
    from helpers import load_golden, to_lafem_levels
    fb = featlib
    lv = to_lafem_levels(load_golden("c1_L4")["levels"])
    h = fb.MultiGridHierarchy(len(lv))
    for d in lv[:-1]:
        sm = fb.new_richardson(d["matrix"], d["filter"], 0.8, fb.new_jacobi_precond(d["matrix"], d["filter"], 0.7))
        sm.set_min_iter(2)
        sm.set_max_iter(2)
        h.push_level(d["matrix"], d["filter"], d["transfer"], sm, sm, sm)
    h.push_level(lv[-1]["matrix"], lv[-1]["filter"], fb.new_coarse_inverse())
    with pytest.raises(fb.FeatB200Error):
        h.smoother_params()
    with pytest.raises(fb.FeatB200Error):
        fb.new_multigrid(h, "X")
    with pytest.raises(fb.FeatB200Error):
        fb.new_multigrid(h).set_adapt_cgc("MinEnergy")


def test_solver_create_rejects_bad_cycle_and_correction(featlib):
    """fb_solver_create validates the configuration before touching a device."""
    from featb200 import _lib
    from helpers import load_golden, to_lafem_levels
    fb = featlib
    L = featlib.lib()
    lv = to_lafem_levels(load_golden("c1_L4")["levels"])
    h = fb.MultiGridHierarchy(len(lv))
    for d in lv[:-1]:
        sm = fb.new_richardson(d["matrix"], d["filter"], 1.0, fb.new_jacobi_precond(d["matrix"], d["filter"], 0.7))
        h.push_level(d["matrix"], d["filter"], d["transfer"], sm, sm, sm)
    h.push_level(lv[-1]["matrix"], lv[-1]["filter"], fb.new_coarse_inverse())
    h.init()   # host-side upload of the levels: no device needed
    for field, bad in (("cycle", 3), ("adapt_cgc", 3), ("adapt_cgc", -1), ("precision", 7), ("smooth_steps", 0)):
        cfg = _lib.SolverConfig()
        L.fb_solver_config_default(C.byref(cfg))
        setattr(cfg, field, bad)
        s = C.c_void_p()
        assert L.fb_solver_create(C.byref(s), h._h, C.byref(cfg)) == 1, field
        assert b"bad configuration" in L.fb_last_error()

"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/_ref/libmgoracle.so`` (the C restatement in ``oracle/mg_oracle.c``) and runs the
reference-side driver ``oracle/_ref/feat_oracle`` (the reference's own CPU solver, built by
``oracle/Makefile``).  Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product never does.

Hierarchies are passed finest level first, as in the reference's ``MultiGridHierarchy``
(kernel/solver/multigrid.hpp:419-957): level i holds A_i, the unit-filter indices of level i, and
P_i (level i <- level i+1), R_i (level i+1 <- level i) for every level but the coarsest.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(REF_DIR, "libmgoracle.so")
FEAT_BIN = os.path.join(REF_DIR, "feat_oracle")
# the same driver built as a FEAT CUDA build on the library's FEAT binding
FEAT_B200_BIN = os.path.join(REF_DIR, "feat_b200")
FEAT_CUDA_BIN = os.path.join(REF_DIR, "feat_cuda")
# the reference source tree the reference binary is compiled from (only where it exists)
REF_SRC = os.environ.get("FEAT_REF", "/root/reference")

STATUS = {0: "progress", 1: "success", 2: "aborted", 3: "diverged", 4: "max_iter"}


class _Csr(C.Structure):
    _fields_ = [("rows", C.c_uint64), ("cols", C.c_uint64), ("row_ptr", C.c_void_p),
                ("col_ind", C.c_void_p), ("val", C.c_void_p)]


class _LevelIn(C.Structure):
    _fields_ = [("A", _Csr), ("P", _Csr), ("R", _Csr), ("fidx", C.c_void_p), ("fval", C.c_void_p),
                ("nf", C.c_uint64)]


def build():
    """Compile the C restatement (and the reference driver when the reference tree exists)."""
    targets = ["port"]
    if os.path.isdir(REF_SRC):
        targets.append("ref")
        # the FEAT build on the library's binding links the built library
        if os.path.exists(os.path.join(os.path.dirname(HERE), "feat3.doxytest_b200", "featb200", "libfeatb200.so")):
            targets.append("b200")
    subprocess.run(["make", "-s", "-j8", "-C", HERE, f"FEAT_REF={REF_SRC}"] + targets, check=True)
    if os.path.isdir(REF_SRC):
        # FEAT on its own CUDA backend: only a timing column beside the library, so a failure to
        # build it (e.g. without the toolkit's cuSPARSE) leaves the checkers usable
        r = subprocess.run(["make", "-s", "-j8", "-C", HERE, f"FEAT_REF={REF_SRC}", "cuda"], capture_output=True,
                           text=True)
        if r.returncode != 0:
            print("oracle: FEAT's CUDA-backend build (feat_cuda) skipped:", (r.stderr or r.stdout).strip()[-300:])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.oc_csr_apply.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_void_p,
                                   C.POINTER(_Csr), C.c_int]
        L.oc_axpy.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_uint64]
        L.oc_dot.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64]
        L.oc_dot.restype = C.c_double
        L.oc_norm2.argtypes = [C.c_void_p, C.c_uint64]
        L.oc_norm2.restype = C.c_double
        L.oc_mg_create.argtypes = [C.c_int, C.POINTER(_LevelIn), C.c_double, C.c_int]
        L.oc_mg_create.restype = C.c_void_p
        L.oc_mg_destroy.argtypes = [C.c_void_p]
        L.oc_mg_vcycle.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oc_mg_set_cycle.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.oc_mg_set_smoother.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int]
        L.oc_mg_colours.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.oc_pcg_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                   C.c_void_p, C.POINTER(C.c_int)]
        L.oc_pcg_jacobi.argtypes = [C.POINTER(_Csr), C.c_void_p, C.c_uint64, C.c_double, C.c_void_p,
                                    C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_int)]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


@dataclass
class Csr:
    """A CSR matrix with the reference's default index type (u64) and FP64 values."""
    row_ptr: np.ndarray
    col_ind: np.ndarray
    val: np.ndarray
    shape: tuple

    @staticmethod
    def of(row_ptr, col_ind, val, shape):
        return Csr(np.ascontiguousarray(row_ptr, dtype=np.uint64),
                   np.ascontiguousarray(col_ind, dtype=np.uint64),
                   np.ascontiguousarray(val, dtype=np.float64), (int(shape[0]), int(shape[1])))

    def c(self):
        return _Csr(self.shape[0], self.shape[1], _ptr(self.row_ptr), _ptr(self.col_ind), _ptr(self.val))


def csr_apply(A: Csr, x, a=1.0, b=0.0, y=None, transposed=False):
    """r = a * op(A) x + b * y, restated from Apply::csr_generic."""
    nout = A.shape[1] if transposed else A.shape[0]
    r = np.zeros(nout) if y is None else np.array(y, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    yy = r if y is not None else None
    cs = A.c()
    lib().oc_csr_apply(_ptr(r), a, _ptr(x), b, _ptr(yy) if yy is not None else _ptr(r), C.byref(cs),
                       1 if transposed else 0)
    return r


def dot(x, y):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return lib().oc_dot(_ptr(x), _ptr(y), x.size)


def norm2(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().oc_norm2(_ptr(x), x.size)


class MultigridPCG:
    """The FP64 PCG + multigrid (V, F or W cycle with `steps` pre- and post-smoothing steps; fixed,
    energy- or defect-minimising coarse-grid correction) of the reference, restated in C."""

    def __init__(self, levels, omega=0.7, steps=2, cycle="V", cgc="fixed", smoother="jacobi", sor_omega=1.0,
                 coloured=False):
        self._keep = []
        arr = (_LevelIn * len(levels))()
        for i, lv in enumerate(levels):
            A = lv["A"]
            fidx = np.ascontiguousarray(lv["filter_idx"], dtype=np.uint64)
            fval = np.ascontiguousarray(lv.get("filter_val", np.zeros(fidx.size)), dtype=np.float64)
            self._keep += [A, fidx, fval]
            arr[i].A = A.c()
            if "P" in lv and lv["P"] is not None:
                self._keep += [lv["P"], lv["R"]]
                arr[i].P = lv["P"].c()
                arr[i].R = lv["R"].c()
            arr[i].fidx = _ptr(fidx)
            arr[i].fval = _ptr(fval)
            arr[i].nf = fidx.size
        self._arr = arr
        self.n = levels[0]["A"].shape[0]
        self.sizes = [lv["A"].shape[0] for lv in levels]
        self._h = lib().oc_mg_create(len(levels), arr, omega, steps)
        if lib().oc_mg_set_cycle(self._h, {"V": 0, "F": 1, "W": 2}[cycle.upper()],
                                 {"fixed": 0, "energy": 1, "defect": 2}[cgc]) != 0:
            raise ValueError("unsupported cycle / coarse-grid correction")
        if lib().oc_mg_set_smoother(self._h, {"jacobi": 0, "sor": 1, "ssor": 2}[smoother], float(sor_omega),
                                    1 if coloured else 0) != 0:
            raise ValueError("unsupported smoother")

    def colours(self, level):
        """(order, offsets) of the greedy colouring of `level` (coloured smoothers only)."""
        nc = lib().oc_mg_colours(self._h, level, None, None)
        if nc < 0:
            raise ValueError("no colouring")
        order = np.zeros(self.sizes[level], dtype=np.uint32)
        cofs = np.zeros(nc + 1, dtype=np.uint32)
        lib().oc_mg_colours(self._h, level, _ptr(order), _ptr(cofs))
        return order, cofs

    def vcycle(self, d):
        d = np.ascontiguousarray(d, dtype=np.float64)
        z = np.zeros(self.n)
        lib().oc_mg_vcycle(self._h, _ptr(z), _ptr(d))
        return z

    def solve(self, rhs, x0=None, tol_rel=1e-8, max_iter=100):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        defects = np.zeros(max_iter + 1)
        it = C.c_int(0)
        st = lib().oc_pcg_solve(self._h, _ptr(x), _ptr(rhs), tol_rel, max_iter, _ptr(defects),
                                C.byref(it))
        return x, {"status": STATUS[st], "iters": it.value, "defects": defects[: it.value + 1]}

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oc_mg_destroy(self._h)
            self._h = None


def pcg_jacobi(A: Csr, rhs, filter_idx, omega=1.0, tol_rel=1e-8, max_iter=1000):
    """Plain PCG (omega = 0: no preconditioner; else Jacobi(omega)) from a zero guess."""
    fidx = np.ascontiguousarray(filter_idx, dtype=np.uint64)
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(A.shape[0])
    it = C.c_int(0)
    cs = A.c()
    st = lib().oc_pcg_jacobi(C.byref(cs), _ptr(fidx), fidx.size, omega, _ptr(x), _ptr(rhs), tol_rel,
                             max_iter, C.byref(it))
    return x, STATUS[st], it.value


# ------------------------------------------------------------------ reference-side driver
def feat_available():
    return os.path.exists(FEAT_BIN)


def feat_b200_available():
    return os.path.exists(FEAT_B200_BIN)


def feat_cuda_available():
    return os.path.exists(FEAT_CUDA_BIN)


def feat_solve(out_dir, dim=2, level=7, rhs="sine", params=None, kappa=None, omega=0.7, steps=2,
               tol=1e-8, iterates=0, vcycle=False, dump_levels=False, time_reps=0, dump=True,
               level_min=1, timeout=3600, cycle="v", cgc="fixed", b200=None, smoother="jacobi", sor_omega=1.0):
    """Run the reference's own solver through oracle/_ref/feat_oracle; returns its JSON summary.
    b200 = "ops" or "solver": the same program built as a FEAT CUDA build on the library's FEAT
    binding (oracle/_ref/feat_b200), with every LAFEM op on the library ("ops") or the whole solve
    handed to the library's solver object ("solver"); b200 = "cuda": the FEAT CUDA build on FEAT's
    own GPU backend (oracle/_ref/feat_cuda), every LAFEM op on FEAT's cuSPARSE / cuBLAS kernels."""
    exe = FEAT_BIN if b200 is None else (FEAT_CUDA_BIN if b200 == "cuda" else FEAT_B200_BIN)
    cmd = [exe, "solve", "--dim", str(dim), "--level", str(level), "--level-min", str(level_min),
           "--out", out_dir, "--rhs", rhs, "--omega", repr(omega), "--steps", str(steps), "--tol",
           repr(tol), "--iterates", str(iterates), "--time", str(time_reps), "--cycle", cycle, "--cgc", cgc]
    if smoother != "jacobi":
        cmd += ["--smoother", smoother, "--sor-omega", repr(float(sor_omega))]
    if params:
        cmd += ["--params", params]
    if kappa:
        cmd += ["--kappa", kappa]
    if vcycle:
        cmd.append("--vcycle")
    if dump_levels:
        cmd.append("--dump-levels")
    if not dump:
        cmd.append("--no-dump")
    if b200 == "ops":
        cmd += ["--backend", "b200"]
    elif b200 == "solver":
        cmd.append("--b200-solver")
    elif b200 == "cuda":
        cmd += ["--backend", "cuda"]
    elif b200 is not None:
        raise ValueError(b200)
    os.makedirs(out_dir, exist_ok=True)
    res = subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout)
    return json.loads(res.stdout.strip().splitlines()[-1])


def feat_io(csr_in, dv_in, out_dir, timeout=300):
    """The reference's own container readers and writers (oracle/_ref/feat_oracle io): reads the
    binary CSR matrix and dense vector, writes rt.csr, rt.dv, rt_matrix.mtx, rt_vector.mtx and
    rt_vector.exp into out_dir; returns its JSON summary."""
    os.makedirs(out_dir, exist_ok=True)
    res = subprocess.run([FEAT_BIN, "io", csr_in, dv_in, out_dir], check=True, capture_output=True, text=True,
                         timeout=timeout)
    return json.loads(res.stdout.strip().splitlines()[-1])


def load_dump(out_dir, level, level_min=1):
    """Read a feat_oracle dump (written with --dump-levels) into a finest-first level list."""
    def ld(name):
        return np.load(os.path.join(out_dir, name + ".npy"))

    def csr(prefix):
        return Csr.of(ld(prefix + "_row_ptr"), ld(prefix + "_col_ind"), ld(prefix + "_val"),
                      ld(prefix + "_shape"))

    levels = []
    for lv in range(level, level_min - 1, -1):
        d = {"A": csr(f"L{lv}_A"), "filter_idx": ld(f"L{lv}_filter_idx"),
             "filter_val": ld(f"L{lv}_filter_val"), "coords": ld(f"L{lv}_coords")}
        if lv > level_min:
            d["P"] = csr(f"L{lv}_P")
            d["R"] = csr(f"L{lv}_R")
        levels.append(d)
    return levels

"""Host-side mirror of the reference's Solver API for the PCG + geometric-multigrid path.

Reads like the reference's own set-up (tutorials/tutorial_05_multigrid.cpp:363-460):

    hierarchy = MultiGridHierarchy(len(levels))
    for lvl in fine levels:
        jacobi = new_jacobi_precond(lvl.matrix, lvl.filter, 0.7)
        smoother = new_richardson(lvl.matrix, lvl.filter, 1.0, jacobi)
        smoother.set_min_iter(2); smoother.set_max_iter(2)
        hierarchy.push_level(lvl.matrix, lvl.filter, lvl.transfer, smoother, smoother, smoother)
    hierarchy.push_level(coarse.matrix, coarse.filter, new_coarse_inverse())
    multigrid = new_multigrid(hierarchy, MultiGridCycle.V)
    solver = new_pcg(fine.matrix, fine.filter, multigrid)
    solver.set_tol_rel(1e-8)
    hierarchy.init(); solver.init()
    status = solve(solver, vec_sol, vec_rhs, fine.matrix, fine.filter)

Everything below ``solver.init()`` runs on the GPU through the C ABI (fb_hierarchy_* /
fb_solver_*).  The device V-cycle implements exactly the configuration above (Richardson(1) +
Jacobi(omega) with min_iter = max_iter for pre- and post-smoothing, exact coarse solve); any other
configuration raises ``FeatB200Error`` instead of running something else.
"""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from . import _lib
from .lafem import DenseVector, SparseMatrixCSR, Transfer, UnitFilter


class Status(enum.IntEnum):
    undefined = 0
    progress = 1
    success = 2
    aborted = 3
    diverged = 4
    max_iter = 5
    stagnated = 6


def status_success(st):
    return st == Status.success


class MultiGridCycle(enum.Enum):
    V = 0
    F = 1
    W = 2


class MultiGridAdaptCGC(enum.Enum):
    """Coarse-grid correction (kernel/solver/multigrid.hpp:39-47)."""
    Fixed = 0
    MinEnergy = 1
    MinDefect = 2


class JacobiPrecond:
    def __init__(self, matrix, filter, omega=1.0):
        self.matrix, self.filter, self.omega = matrix, filter, float(omega)


class Richardson:
    def __init__(self, matrix, filter, omega=1.0, precond=None):
        self.matrix, self.filter, self.omega, self.precond = matrix, filter, float(omega), precond
        self.min_iter, self.max_iter = 0, 100

    def set_min_iter(self, k):
        self.min_iter = int(k)

    def set_max_iter(self, k):
        self.max_iter = int(k)


class CoarseInverse:
    """Exact coarse-grid solve: inverse of the matrix restricted to the free DOFs."""


def new_jacobi_precond(matrix, filter, omega=1.0):
    return JacobiPrecond(matrix, filter, omega)


def new_richardson(matrix, filter, omega=1.0, precond=None):
    return Richardson(matrix, filter, omega, precond)


def new_coarse_inverse(*_args):
    return CoarseInverse()


class MultiGridHierarchy:
    """MultiGridHierarchy<SparseMatrixCSR, UnitFilter, Transfer> (kernel/solver/multigrid.hpp:419)."""

    def __init__(self, size):
        self.size = int(size)
        self.levels = []
        self._h = None

    def push_level(self, matrix, filter, transfer_or_coarse, smoother_pre=None, smoother_post=None,
                   smoother_peak=None):
        if isinstance(transfer_or_coarse, Transfer):
            self.levels.append({"matrix": matrix, "filter": filter, "transfer": transfer_or_coarse,
                                "pre": smoother_pre, "post": smoother_post, "peak": smoother_peak})
        else:
            if not isinstance(transfer_or_coarse, CoarseInverse):
                raise _lib.FeatB200Error("the device multigrid supports the exact coarse inverse only")
            self.levels.append({"matrix": matrix, "filter": filter, "coarse": transfer_or_coarse})

    def smoother_params(self):
        omega = steps = None
        for lv in self.levels[:-1]:
            for sm in (lv["pre"], lv["post"]):
                if not isinstance(sm, Richardson) or sm.omega != 1.0 or sm.min_iter != sm.max_iter or \
                        not isinstance(sm.precond, JacobiPrecond):
                    raise _lib.FeatB200Error(
                        "the device V-cycle implements Richardson(omega=1)+Jacobi smoothing with "
                        "min_iter == max_iter on every level")
                if omega is None:
                    omega, steps = sm.precond.omega, sm.max_iter
                elif (omega, steps) != (sm.precond.omega, sm.max_iter):
                    raise _lib.FeatB200Error("all levels must use the same smoother parameters")
        return (0.7 if omega is None else omega), (2 if steps is None else steps)

    def init(self):
        if len(self.levels) != self.size:
            raise _lib.FeatB200Error(f"hierarchy has {len(self.levels)} of {self.size} levels")
        if "coarse" not in self.levels[-1]:
            raise _lib.FeatB200Error("the last pushed level must carry the coarse solver")
        L = _lib.lib()
        h = C.c_void_p()
        _lib.check(L.fb_hierarchy_create(C.byref(h), self.size), "fb_hierarchy_create")
        self._h = h
        for i, lv in enumerate(self.levels):
            A = lv["matrix"].c_host()
            f: UnitFilter = lv["filter"]
            if "transfer" in lv:
                Pm, Rm = lv["transfer"].prol, lv["transfer"].rest
                Pc, Rc = Pm.c_host(), Rm.c_host()
                _lib.check(L.fb_hierarchy_set_level(h, i, C.byref(A), f.indices.ctypes.data_as(C.c_void_p),
                                                    f.values.ctypes.data_as(C.c_void_p), f.indices.size,
                                                    C.byref(Pc), C.byref(Rc)), "fb_hierarchy_set_level")
            else:
                _lib.check(L.fb_hierarchy_set_level(h, i, C.byref(A), f.indices.ctypes.data_as(C.c_void_p),
                                                    f.values.ctypes.data_as(C.c_void_p), f.indices.size,
                                                    None, None), "fb_hierarchy_set_level")

    def done(self):
        if self._h is not None:
            _lib.lib().fb_hierarchy_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.done()
        except Exception:
            pass


class MultiGrid:
    def __init__(self, hierarchy, cycle=MultiGridCycle.V):
        """V, F or W cycle (MultiGrid::_apply_cycle_v/_f/_w, kernel/solver/multigrid.hpp:1350-1440);
        the peak smoother is the pre/post smoother (push_level with the same smoother three times)."""
        if cycle not in (MultiGridCycle.V, MultiGridCycle.F, MultiGridCycle.W):
            raise _lib.FeatB200Error("unknown multigrid cycle")
        if cycle != MultiGridCycle.V:
            # the device applies the peak smoother once, as the reference does when one is pushed;
            # without one the reference would run pre- and post-smoother in turn
            for lv in hierarchy.levels[:-1]:
                pk = lv.get("peak")
                if pk is None or not (pk is lv["pre"] or (isinstance(pk, Richardson) and isinstance(lv["pre"], Richardson)
                                                          and (pk.omega, pk.min_iter, pk.max_iter) ==
                                                          (lv["pre"].omega, lv["pre"].min_iter, lv["pre"].max_iter))):
                    raise _lib.FeatB200Error("F/W cycles need the peak smoother to be the pre/post smoother")
        self.hierarchy, self.cycle = hierarchy, cycle
        self.adapt_cgc = MultiGridAdaptCGC.Fixed

    def set_adapt_cgc(self, adapt_cgc):
        """MultiGrid::set_adapt_cgc (multigrid.hpp:1091): scale each coarse-grid correction by the
        step length minimising the energy or the defect."""
        if not isinstance(adapt_cgc, MultiGridAdaptCGC):
            raise _lib.FeatB200Error("adapt_cgc must be a MultiGridAdaptCGC")
        self.adapt_cgc = adapt_cgc


EVENT_NAMES = ("pre", "def", "res", "crs", "pro", "post", "post_top", "proc", "postc", "postc_top")


def cycle_events(cycle="V", num_levels=2, adapt_cgc="Fixed"):
    """The events one multigrid cycle runs, [(name, level)] (fb_multigrid_cycle_events): what the
    device executes for MultiGrid::_apply_cycle_v/_f/_w over num_levels levels, finest = 0."""
    import numpy as np
    cyc = {"V": 0, "F": 1, "W": 2}[cycle]
    cgc = MultiGridAdaptCGC[adapt_cgc].value
    n = C.c_uint64()
    _lib.check(_lib.lib().fb_multigrid_cycle_events(cyc, cgc, int(num_levels), None, None, 0, C.byref(n)),
               "fb_multigrid_cycle_events")
    ops = np.zeros(max(1, n.value), dtype=np.uint8)
    lvl = np.zeros(max(1, n.value), dtype=np.uint8)
    _lib.check(_lib.lib().fb_multigrid_cycle_events(cyc, cgc, int(num_levels), ops.ctypes.data_as(C.c_void_p),
                                                     lvl.ctypes.data_as(C.c_void_p), n.value, C.byref(n)),
               "fb_multigrid_cycle_events")
    return [(EVENT_NAMES[int(o)], int(l)) for o, l in zip(ops[:n.value], lvl[:n.value])]


def storage_plan(matrix, empty_rows=None, ordering="native", diagonal=True):
    """How the solver stores `matrix` (a SparseMatrixCSR) on the device (fb_matrix_storage_plan):
    dict(kind='sliced'|'ell'|'diagonal', width, narrow, diagonals, entries)."""
    c = matrix.c_host()
    er = np.ascontiguousarray(np.zeros(0) if empty_rows is None else empty_rows, dtype=np.uint64)
    out = _lib.StoragePlan()
    _lib.check(_lib.lib().fb_matrix_storage_plan(C.byref(c), er.ctypes.data_as(C.c_void_p), er.size,
                                                  1 if ordering == "rcm" else 0, 1 if diagonal else 0,
                                                  C.byref(out)), "fb_matrix_storage_plan")
    return {"kind": ("sliced", "ell", "diagonal")[out.kind], "width": int(out.width), "narrow": bool(out.narrow),
            "diagonals": int(out.diagonals), "entries": int(out.entries)}


def new_multigrid(hierarchy, cycle=MultiGridCycle.V):
    return MultiGrid(hierarchy, cycle)


class PCG:
    """PCG<SparseMatrixCSR, UnitFilter> preconditioned by MultiGrid (kernel/solver/pcg.hpp)."""

    def __init__(self, matrix, filter, precond: MultiGrid):
        if not isinstance(precond, MultiGrid):
            raise _lib.FeatB200Error("the device PCG is preconditioned by the multigrid V-cycle")
        self.matrix, self.filter, self.precond = matrix, filter, precond
        self.cfg = _lib.SolverConfig()
        _lib.lib().fb_solver_config_default(C.byref(self.cfg))
        self._s = None
        self.info = _lib.SolveInfo()
        self.plot_mode = "none"

    # IterativeSolver setters (kernel/solver/iterative.hpp:258-300)
    def set_tol_rel(self, v):
        self.cfg.tol_rel = float(v)

    def set_tol_abs(self, v):
        self.cfg.tol_abs = float(v)

    def set_max_iter(self, k):
        self.cfg.max_iter = int(k)

    def set_min_iter(self, k):
        self.cfg.min_iter = int(k)

    def set_plot_mode(self, mode):
        self.plot_mode = str(mode)

    # device options
    def set_precision(self, p):
        self.cfg.precision = _lib.PREC[p]

    def set_ordering(self, o):
        self.cfg.ordering = _lib.ORDER[o]

    def set_use_graph(self, flag):
        self.cfg.use_graph = 1 if flag else 0

    def set_tma_rows(self, rows):
        """Uniform-width levels with at least `rows` rows use the TMA-staged passes (0 = off)."""
        self.cfg.tma_rows = int(rows)

    def set_tma_window(self, mode):
        """Window of the gathered vector per TMA-staged chunk: 0 = neither (default), 1 = staged in
        shared memory, 2 = prefetched into L2."""
        self.cfg.tma_window = int(mode)

    def set_cluster_rows(self, rows):
        """Levels with at most `rows` rows (below the finest) run in one kernel on a cluster of 8
        thread blocks (0 = off; takes precedence over set_tail_rows)."""
        self.cfg.cluster_rows = int(rows)

    def set_diagonal(self, on):
        """Store system matrices that lie on at most 27 diagonals of the device numbering as
        diagonals without column indices (1, default) or always as sliced ELL (0)."""
        self.cfg.diagonal = int(bool(on))

    def set_pdl(self, on):
        """Launch the solve's kernels with programmatic dependent launch (1, default) or in plain
        stream order (0)."""
        self.cfg.pdl = int(bool(on))

    def set_fused(self, rows):
        """Fused V(2,2) passes on structured 2D levels of at most `rows` rows (default 70000;
        True = every level, False / 0 = none): one pass for pre-smoothing, defect and restriction,
        one for prolongation and post-smoothing."""
        self.cfg.fused = (2 ** 31 - 1) if rows is True else int(rows)

    def set_streamed(self, rows):
        """Streamed fused passes on structured 2D levels with more rows than the `fused` threshold
        and at least `rows` rows (True = every such level, False / 0 = none): the same two fused
        passes, swept row by row through bands of coarse rows with their rows staged in shared
        memory."""
        self.cfg.streamed = 1 if rows is True else int(rows)

    def set_smoother(self, kind="jacobi", omega=1.0, sweep="sequential"):
        """The Richardson smoother's preconditioner: "jacobi" (JacobiPrecond with the hierarchy's
        damping), "sor" or "ssor" (SORPrecond / SSORPrecond with damping `omega`); SOR / SSOR sweep
        in the rows' dependency levels ("sequential": the reference's generic sweep, bit for bit) or
        in greedy colours ("coloured": the reference's coloured CUDA sweeps)."""
        self.cfg.smoother = {"jacobi": 0, "sor": 1, "ssor": 2}[kind]
        self.cfg.smoother_omega = float(omega)
        self.cfg.sweep_colouring = {"sequential": 0, "coloured": 1}[sweep]

    def set_tail_rows(self, rows):
        """Levels with at most `rows` rows (below the finest) run in one single-block kernel."""
        self.cfg.tail_rows = int(rows)

    def init(self):
        h = self.precond.hierarchy
        omega, steps = h.smoother_params()
        self.cfg.omega = omega
        self.cfg.smooth_steps = steps
        self.cfg.cycle = {MultiGridCycle.V: 0, MultiGridCycle.F: 1, MultiGridCycle.W: 2}[self.precond.cycle]
        self.cfg.adapt_cgc = self.precond.adapt_cgc.value
        if h._h is None:
            h.init()
        s = C.c_void_p()
        _lib.check(_lib.lib().fb_solver_create(C.byref(s), h._h, C.byref(self.cfg)), "fb_solver_create")
        self._s = s

    def done(self):
        if self._s is not None:
            _lib.lib().fb_solver_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.done()
        except Exception:
            pass

    def correct(self, vec_sol: DenseVector, vec_rhs: DenseVector):
        if self._s is None:
            raise _lib.FeatB200Error("PCG.init() was not called")
        _lib.check(_lib.lib().fb_solver_solve(self._s, vec_sol.elements.ctypes.data_as(C.c_void_p),
                                              vec_rhs.elements.ctypes.data_as(C.c_void_p), C.byref(self.info)),
                   "fb_solver_solve")
        st = Status(self.info.status)
        if self.plot_mode != "none":
            print(f"PCG: {self.info.iterations} iterations, |d0| {self.info.def_init:.6e} -> "
                  f"|d| {self.info.def_final:.6e} ({st.name}, {self.info.solve_ms:.3f} ms)")
        return st

    def correct_device(self, sol, rhs, stream=None):
        """Solve with CUDA tensors (caller numbering) on `stream` (default: torch's current)."""
        if stream is None:
            import torch
            stream = torch.cuda.current_stream()
        _lib.check(_lib.lib().fb_solver_solve_device(self._s, C.c_void_p(sol.data_ptr()), C.c_void_p(rhs.data_ptr()),
                                                     C.c_void_p(stream.cuda_stream), C.byref(self.info)),
                   "fb_solver_solve_device")
        return Status(self.info.status)

    def set_tolerances(self, tol_rel, tol_abs):
        """Stopping test of the following solves: ||d|| <= tol_abs and ||d|| <= tol_rel ||d_0||."""
        _lib.check(_lib.lib().fb_solver_set_tolerances(self._s, float(tol_rel), float(tol_abs)),
                   "fb_solver_set_tolerances")

    def update_matrix(self, level, values, stream=None):
        """New values for the system matrix of `level` (0 = finest) in the pattern and entry order
        it was pushed with: a CUDA float64 tensor of nnz entries.  Refreshes the level's Jacobi
        diagonal and, on the coarsest level, the exact coarse inverse -- what the reference's
        init_numeric() does after the matrix values changed (kernel/solver/multigrid.hpp:776-790,
        kernel/solver/jacobi_precond.hpp:136-165)."""
        if stream is None:
            import torch
            stream = torch.cuda.current_stream()
        _lib.check(_lib.lib().fb_solver_update_matrix(self._s, int(level), C.c_void_p(values.data_ptr()),
                                                      C.c_void_p(stream.cuda_stream)), "fb_solver_update_matrix")

    def apply_precond(self, vec_def: DenseVector):
        """One V-cycle: MultiGrid::apply (kernel/solver/multigrid.hpp:1270)."""
        out = DenseVector(vec_def.size())
        _lib.check(_lib.lib().fb_solver_vcycle(self._s, out.elements.ctypes.data_as(C.c_void_p),
                                               vec_def.elements.ctypes.data_as(C.c_void_p)), "fb_solver_vcycle")
        return out

    def get_num_iter(self):
        return int(self.info.iterations)

    def get_def_initial(self):
        return float(self.info.def_init)

    def get_def_final(self):
        return float(self.info.def_final)

    def get_status(self):
        return Status(self.info.status)

    def time_kernel(self, which="pcg_spmv", reps=20, flush_l2=True):
        """Mean launch time (ms) and stored bytes per launch of one solver kernel timed alone:
        pcg_spmv, mg_defect, mg_smooth, mg_post1, mg_post2, mg_restrict, mg_prolong (finest-level
        passes), mg_down / mg_up (the fused passes of a structured finest level), mg_sdown / mg_sup
        (the same in their streamed form), mg_tail (the
        coarse-level tail kernel) or mg_cycle (one whole multigrid cycle)."""
        code = {"pcg_spmv": 0, "mg_defect": 1, "mg_tail": 2, "mg_cycle": 3, "mg_smooth": 4, "mg_post1": 5,
                "mg_post2": 6, "mg_restrict": 7, "mg_prolong": 8, "mg_down": 9, "mg_up": 10, "mg_sdown": 11,
                "mg_sup": 12}[which]
        ms, by = C.c_double(), C.c_double()
        _lib.check(_lib.lib().fb_solver_time_kernel(self._s, code, int(reps), 1 if flush_l2 else 0, C.byref(ms),
                                                     C.byref(by)), "fb_solver_time_kernel")
        return ms.value, by.value

    def level_info(self):
        n = len(self.precond.hierarchy.levels)
        out = np.zeros(3 * n, dtype=np.uint64)
        _lib.check(_lib.lib().fb_solver_level_info(self._s, out.ctypes.data_as(C.c_void_p)), "fb_solver_level_info")
        return out.reshape(n, 3)


def new_pcg(matrix, filter, precond):
    return PCG(matrix, filter, precond)


def solve(solver, vec_sol, vec_rhs, matrix=None, filter=None):
    """Solver::solve (kernel/solver/iterative.hpp:930-939): calls solver.correct(sol, rhs)."""
    return solver.correct(vec_sol, vec_rhs)


def build_pcg_multigrid(levels, omega=0.7, steps=2, tol_rel=1e-8, max_iter=100, precision="f64",
                        ordering="native", use_graph=True, tail_rows=None, tma_rows=None, tma_window=None,
                        cluster_rows=None, cycle="V", diagonal=None, pdl=None, adapt_cgc="Fixed", fused=None,
                        smoother="jacobi", smoother_omega=1.0, sweep="sequential", streamed=None):
    """Convenience set-up from a finest-first list of level dicts with keys matrix, filter,
    transfer (all but the coarsest)."""
    h = MultiGridHierarchy(len(levels))
    for lv in levels[:-1]:
        jac = new_jacobi_precond(lv["matrix"], lv["filter"], omega)
        sm = new_richardson(lv["matrix"], lv["filter"], 1.0, jac)
        sm.set_min_iter(steps)
        sm.set_max_iter(steps)
        h.push_level(lv["matrix"], lv["filter"], lv["transfer"], sm, sm, sm)
    h.push_level(levels[-1]["matrix"], levels[-1]["filter"], new_coarse_inverse())
    mg = new_multigrid(h, MultiGridCycle[cycle])
    mg.set_adapt_cgc(MultiGridAdaptCGC[adapt_cgc])
    s = new_pcg(levels[0]["matrix"], levels[0]["filter"], mg)
    s.set_tol_rel(tol_rel)
    s.set_max_iter(max_iter)
    s.set_precision(precision)
    s.set_ordering(ordering)
    s.set_use_graph(use_graph)
    if tail_rows is not None:
        s.set_tail_rows(tail_rows)
    if tma_rows is not None:
        s.set_tma_rows(tma_rows)
    if tma_window is not None:
        s.set_tma_window(tma_window)
    if cluster_rows is not None:
        s.set_cluster_rows(cluster_rows)
    if diagonal is not None:
        s.set_diagonal(diagonal)
    if pdl is not None:
        s.set_pdl(pdl)
    if fused is not None:
        s.set_fused(fused)
    if streamed is not None:
        s.set_streamed(streamed)
    s.set_smoother(smoother, smoother_omega, sweep)
    h.init()
    s.init()
    return s


class MultiRhsPCG:
    """PCG + V-cycle for K = 32 or 64 right-hand sides at once (fb_msolver_*): every right-hand side
    follows the single-RHS algorithm with its own scalars and stopping test; the matrices are read
    once per pass for all of them.  Vectors are [rows, K] (right-hand side index fastest), the
    element layout of the reference's DenseVectorBlocked."""

    def __init__(self, hierarchy: MultiGridHierarchy, num_rhs, tol_rel=1e-8, max_iter=100, precision="f64",
                 ordering="native", use_graph=True, stencil=False):
        omega, steps = hierarchy.smoother_params()
        self.k = int(num_rhs)
        self.cfg = _lib.SolverConfig()
        _lib.lib().fb_solver_config_default(C.byref(self.cfg))
        self.cfg.omega, self.cfg.smooth_steps = omega, steps
        self.cfg.tol_rel, self.cfg.max_iter = float(tol_rel), int(max_iter)
        self.cfg.precision, self.cfg.ordering = _lib.PREC[precision], _lib.ORDER[ordering]
        self.cfg.use_graph = 1 if use_graph else 0
        # stencil=True: system matrices with the Q1 stencil pattern in the device numbering run in the
        # stencil form (strips of rows sharing their gathers; row sums bitwise those of the CSR form).
        # Off by default: on one B200 it measured no faster than the CSR form (10.29 against 9.95 ms
        # for 64 solves at 3D L6).
        self.cfg.diagonal = 1 if stencil else 0
        if hierarchy._h is None:
            hierarchy.init()
        self.hierarchy = hierarchy
        s = C.c_void_p()
        _lib.check(_lib.lib().fb_msolver_create(C.byref(s), hierarchy._h, C.byref(self.cfg), self.k),
                   "fb_msolver_create")
        self._s = s
        self.info = (_lib.SolveInfo * self.k)()

    def solve(self, sol, rhs):
        """sol (initial guesses, overwritten) and rhs: float64 arrays of shape [rows, K]."""
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        _lib.check(_lib.lib().fb_msolver_solve(self._s, sol.ctypes.data_as(C.c_void_p), rhs.ctypes.data_as(C.c_void_p),
                                               self.info), "fb_msolver_solve")
        return sol

    def solve_device(self, sol, rhs, stream=None):
        if stream is None:
            import torch
            stream = torch.cuda.current_stream()
        _lib.check(_lib.lib().fb_msolver_solve_device(self._s, C.c_void_p(sol.data_ptr()), C.c_void_p(rhs.data_ptr()),
                                                      C.c_void_p(stream.cuda_stream), self.info),
                   "fb_msolver_solve_device")

    def statuses(self):
        return [Status(i.status) for i in self.info]

    def iterations(self):
        return [int(i.iterations) for i in self.info]

    def done(self):
        if self._s is not None:
            _lib.lib().fb_msolver_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.done()
        except Exception:
            pass


def build_hierarchy(levels, omega=0.7, steps=2):
    """MultiGridHierarchy of Richardson(1)+Jacobi(omega) smoothers and the exact coarse inverse
    from a finest-first list of level dicts (matrix, filter, transfer)."""
    h = MultiGridHierarchy(len(levels))
    for lv in levels[:-1]:
        jac = new_jacobi_precond(lv["matrix"], lv["filter"], omega)
        sm = new_richardson(lv["matrix"], lv["filter"], 1.0, jac)
        sm.set_min_iter(steps)
        sm.set_max_iter(steps)
        h.push_level(lv["matrix"], lv["filter"], lv["transfer"], sm, sm, sm)
    h.push_level(levels[-1]["matrix"], levels[-1]["filter"], new_coarse_inverse())
    h.init()
    return h


class BatchPCG:
    """Many independent PCG + V-cycle solves of uneven size (fb_batch_*): every V-cycle pass is one
    launch over all instances; each instance has its own scalars and stopping test.  Vectors are
    packed: the instances' fine-level vectors concatenated in order."""

    def __init__(self, hierarchies, tol_rel=1e-8, max_iter=100, precision="f64", ordering="native",
                 use_graph=True, rows_per_block=0):
        omega, steps = hierarchies[0].smoother_params()
        for h in hierarchies:
            if h.smoother_params() != (omega, steps):
                raise _lib.FeatB200Error("all instances must use the same smoother parameters")
            if h._h is None:
                h.init()
        self.hierarchies = list(hierarchies)
        self.j = len(self.hierarchies)
        self.cfg = _lib.SolverConfig()
        _lib.lib().fb_solver_config_default(C.byref(self.cfg))
        self.cfg.omega, self.cfg.smooth_steps = omega, steps
        self.cfg.tol_rel, self.cfg.max_iter = float(tol_rel), int(max_iter)
        self.cfg.precision, self.cfg.ordering = _lib.PREC[precision], _lib.ORDER[ordering]
        self.cfg.use_graph = 1 if use_graph else 0
        self.cfg.rows_per_block = int(rows_per_block)
        arr = (C.c_void_p * self.j)(*[h._h.value for h in self.hierarchies])
        s = C.c_void_p()
        _lib.check(_lib.lib().fb_batch_create(C.byref(s), self.j, arr, C.byref(self.cfg)), "fb_batch_create")
        self._s = s
        sizes = np.zeros(self.j, dtype=np.uint64)
        _lib.check(_lib.lib().fb_batch_sizes(self._s, sizes.ctypes.data_as(C.c_void_p)), "fb_batch_sizes")
        self.sizes = sizes.astype(np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])
        self.info = (_lib.SolveInfo * self.j)()

    def rows_per_block(self):
        """Rows per block of the V-cycle passes per global level, finest first (autotuned unless
        given at construction)."""
        n = C.c_int(0)
        _lib.check(_lib.lib().fb_batch_rows_per_block(self._s, None, C.byref(n)), "fb_batch_rows_per_block")
        out = np.zeros(n.value, dtype=np.int32)
        _lib.check(_lib.lib().fb_batch_rows_per_block(self._s, out.ctypes.data_as(C.c_void_p), C.byref(n)),
                   "fb_batch_rows_per_block")
        return out

    def solve(self, sol, rhs):
        """sol (initial guesses, overwritten) and rhs: packed float64 arrays."""
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        _lib.check(_lib.lib().fb_batch_solve(self._s, sol.ctypes.data_as(C.c_void_p), rhs.ctypes.data_as(C.c_void_p),
                                             self.info), "fb_batch_solve")
        return sol

    def solve_device(self, sol, rhs, stream=None):
        if stream is None:
            import torch
            stream = torch.cuda.current_stream()
        _lib.check(_lib.lib().fb_batch_solve_device(self._s, C.c_void_p(sol.data_ptr()), C.c_void_p(rhs.data_ptr()),
                                                    C.c_void_p(stream.cuda_stream), self.info), "fb_batch_solve_device")

    def split(self, packed):
        return [packed[self.offsets[k]:self.offsets[k + 1]] for k in range(self.j)]

    def statuses(self):
        return [Status(i.status) for i in self.info]

    def iterations(self):
        return [int(i.iterations) for i in self.info]

    def done(self):
        if self._s is not None:
            _lib.lib().fb_batch_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.done()
        except Exception:
            pass

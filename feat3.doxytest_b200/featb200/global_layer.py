"""The reference's global layer for the overlapping domain decomposition, one process per GPU.

Every rank owns the DOFs of its patch; DOFs on an interface between patches exist on every rank
that shares them.  Vectors come in two kinds (kernel/global/gate.hpp:320-470):

* type 0: each rank holds its partial sum (a patch-local assembly, the result of a patch-local
  matrix product); the global value of a shared DOF is the sum over the sharing ranks;
* type 1: every rank holds the full global value.

`Gate` mirrors `Global::Gate`: per neighbour rank a mirror (the local indices of the DOFs shared with
that rank, in an order both sides agree on), the frequencies 1 / (number of ranks sharing a DOF)
(`compile`, gate.hpp:265-285), `sync_0` (type 0 -> type 1: add the neighbours' entries of the shared
DOFs; `SynchVectorTicket`, synch_vec.hpp:28-223: gather into a buffer per neighbour, exchange,
scatter-add the received buffers in neighbour order), `sync_1` (type 1 -> type 1 after rounding
drift: scale by the frequencies, then `sync_0`), and the global dot product `dot` = the sum over the
ranks of the frequency-weighted local triple product (gate.hpp:476-492).

`GlobalMatrix` is `Global::Matrix::apply` (kernel/global/matrix.hpp): the patch-local product of a
type-0 matrix with a type-1 vector, then `sync_0`.  `global_pcg` is `Solver::PCG` on these global
types with the global Jacobi preconditioner (the type-1 diagonal from `sync_0` of the patch-local
diagonals, `Solver::JacobiPrecond` with a global matrix).

The multigrid on these types: `GlobalTransfer` is `Global::Transfer` (kernel/global/transfer.hpp:
252-336): the patch-local restriction followed by `sync_0` of the coarse vector, the patch-local
prolongation followed by `sync_0` of the fine vector, which is exact because the patch-local
prolongation's rows are scaled by the inverse of the globally summed assembly weights
(`prolongation_row_scaling`, control/scalar_basic.hpp:308-324).  `Muxer` is `Global::Muxer`
(kernel/global/muxer.hpp:344-530): the coarse levels below a chosen level live on one parent rank,
`join` gathers the children's type-0 vectors into the parent's merged vector, `split` hands the
type-1 result back.  A rank that is a child but not the parent holds a ghost transfer: it sends its
restriction (`rest_send`) and waits for the prolongation (`prol_recv`) while the parent runs the
coarse levels (kernel/solver/multigrid.hpp:1783-1790, 1871-1877).  `GlobalMultiGrid` is the V-cycle
with the Richardson-Jacobi smoother and an exact coarse solve on these global levels, in the
operation order of the single-system solve, and `global_pcg` takes it as its preconditioner.

Vectors are torch tensors: on CUDA devices with the NCCL backend the exchange runs over NVLink,
on the CPU with gloo (the tests).  The exchange is point-to-point (`isend` / `irecv` of the gathered
buffers) because only neighbours share DOFs; the muxer's join and split are a gather to and a
scatter from the parent.  The local matrix, prolongation and restriction products are callables, so
that the product path can use the library's device SpMV and the tests a host CSR product.
"""
from __future__ import annotations

import math

import torch


class Gate:
    def __init__(self, dist=None):
        """dist: the torch.distributed module with an initialised process group (None = one rank)."""
        self.dist = dist
        self.ranks: list[int] = []
        self.mirrors: list[torch.Tensor] = []
        self.freqs: torch.Tensor | None = None

    def push(self, rank: int, mirror):
        """Gate::push: the local indices of the DOFs shared with `rank`, in the order that `rank`
        lists the same DOFs."""
        self.ranks.append(int(rank))
        self.mirrors.append(torch.as_tensor(mirror, dtype=torch.long))

    def compile(self, n: int, device="cpu", dtype=torch.float64):
        """Gate::compile: frequencies 1 / (1 + number of mirrors listing the DOF)."""
        f = torch.ones(n, dtype=dtype, device=device)
        self.mirrors = [m.to(device) for m in self.mirrors]
        for m in self.mirrors:
            f.index_add_(0, m, torch.ones(m.numel(), dtype=dtype, device=device))
        self.freqs = 1.0 / f
        return self

    def _world(self):
        return 1 if self.dist is None else self.dist.get_world_size()

    def from_1_to_0(self, v: torch.Tensor):
        if self.ranks:
            v.mul_(self.freqs)
        return v

    def sync_0(self, v: torch.Tensor):
        """Type 0 -> type 1, in place: every shared entry becomes the sum over the sharing ranks."""
        if not self.ranks:
            return v
        sends = [v.index_select(0, m).contiguous() for m in self.mirrors]
        recvs = [torch.empty_like(s) for s in sends]
        reqs = []
        for r, s, b in zip(self.ranks, sends, recvs):
            reqs.append(self.dist.isend(s, dst=r))
            reqs.append(self.dist.irecv(b, src=r))
        for q in reqs:
            q.wait()
        # scatter-add in neighbour order (a fixed summation order on every rank)
        for m, b in zip(self.mirrors, recvs):
            v.index_add_(0, m, b)
        return v

    def sync_1(self, v: torch.Tensor):
        """Type 1 -> type 1: scale by the frequencies, then sum over the sharing ranks."""
        if self.ranks:
            self.from_1_to_0(v)
            self.sync_0(v)
        return v

    def _sum(self, local: torch.Tensor) -> float:
        """The sum over the ranks of a one-element tensor, all-reduced on its own device (no host
        copy before the reduction; one synchronisation to read the result)."""
        if self._world() == 1:
            return float(local)
        t = local.reshape(1).clone()
        self.dist.all_reduce(t)
        return float(t.item())

    def dot(self, x: torch.Tensor, y: torch.Tensor) -> float:
        """Global dot product of two type-1 vectors (gate.hpp:476-492)."""
        if self._world() == 1 or not self.ranks:
            return self._sum(torch.dot(x, y))
        return self._sum(torch.sum(self.freqs * x * y))

    def norm2(self, x: torch.Tensor) -> float:
        return math.sqrt(self.dot(x, x))


def device_csr_apply(csr):
    """The patch-local product on the device for a type-0 `SparseMatrixCSR`: the library's CSR
    kernel (`fb_apply_csr_f64_u64`, the `Arch::Apply::csr` drop-in) on CUDA tensors."""
    rp = torch.as_tensor(csr.row_ptr.astype("int64"), device="cuda")
    ci = torch.as_tensor(csr.col_ind.astype("int64"), device="cuda")
    val = torch.as_tensor(csr.val, device="cuda")
    rows, cols = csr.rows(), csr.columns()

    def apply(x: torch.Tensor) -> torch.Tensor:
        from .lafem import arch
        r = torch.empty(rows, dtype=torch.float64, device="cuda")
        arch.apply_csr(r, 1.0, x, 0.0, None, val, ci, rp, cols)
        return r
    return apply


class GlobalMatrix:
    """Global::Matrix::apply: r = sync_0(A_local x) for a type-0 matrix and a type-1 vector."""

    def __init__(self, local_apply, gate: Gate, local_diag: torch.Tensor):
        self.local_apply, self.gate = local_apply, gate
        self.local_diag = local_diag

    def apply(self, r: torch.Tensor, x: torch.Tensor):
        r.copy_(self.local_apply(x))
        return self.gate.sync_0(r)

    def apply_axpy(self, r: torch.Tensor, x: torch.Tensor, y: torch.Tensor, alpha=1.0):
        """r = y + alpha A x (matrix.hpp:365-378): y to type 0, the local product added, sync_0."""
        r.copy_(y)
        self.gate.from_1_to_0(r)
        r.add_(self.local_apply(x), alpha=alpha)
        return self.gate.sync_0(r)

    def diagonal(self) -> torch.Tensor:
        """The global (type-1) main diagonal."""
        return self.gate.sync_0(self.local_diag.clone())


class GlobalUnitFilter:
    """Global::Filter over a UnitFilter: the Dirichlet DOFs of the patch (shared ones on every
    sharing rank)."""

    def __init__(self, indices, values=None):
        self.idx = torch.as_tensor(indices, dtype=torch.long)
        self.vals = None if values is None else torch.as_tensor(values, dtype=torch.float64)

    def to(self, device):
        self.idx = self.idx.to(device)
        if self.vals is not None:
            self.vals = self.vals.to(device)
        return self

    def filter_def(self, v: torch.Tensor):
        v[self.idx] = 0.0
        return v

    filter_cor = filter_def

    def filter_sol(self, v: torch.Tensor):
        v[self.idx] = 0.0 if self.vals is None else self.vals
        return v


def prolongation_row_scaling(weight: torch.Tensor, gate: Gate) -> torch.Tensor:
    """The row scaling of a patch-local prolongation (control/scalar_basic.hpp:308-324).  The patch
    assembles its prolongation summed over its own coarse cells together with a weight vector that
    counts, per fine DOF, the cells that contributed; the global weight is the `sync_0` of the patch
    weights, and the patch's rows are scaled by its inverse.  A shared fine DOF then receives a part
    of the global row on every sharing rank, and `sync_0` of the patch products is the global
    prolongation.  Returns the scaling vector (type 1)."""
    w = gate.sync_0(weight.clone())
    return 1.0 / w


class Muxer:
    """Global::Muxer (kernel/global/muxer.hpp:69-533) with the whole process group as the sibling
    communicator: every rank is a child, and rank `parent` holds the merged coarse levels.

    Every rank sends the entries its parent mirror lists (`push_parent`; the patch's coarse DOFs);
    the parent knows, per rank, where those entries sit in its merged vector (`push_child`, in rank
    order).  `join` sums the children's type-0 vectors into the merged vector (gather, then
    scatter-add in rank order: muxer.hpp:380-432), `split` hands each child its entries of the merged
    type-1 vector (gather per child, scatter: muxer.hpp:481-530).  Buffers have the length of the
    largest parent mirror over the ranks."""

    def __init__(self, dist=None, parent=0):
        self.dist, self.parent = dist, int(parent)
        self.parent_mirror: torch.Tensor | None = None
        self.child_mirrors: list[torch.Tensor] = []
        self.bufsize = 0

    def _size(self):
        return 1 if self.dist is None else self.dist.get_world_size()

    def _rank(self):
        return 0 if self.dist is None else self.dist.get_rank()

    def is_child(self) -> bool:
        return self._size() > 1

    def is_parent(self) -> bool:
        return self._rank() == self.parent

    def is_ghost(self) -> bool:
        """A child that is not the parent holds no coarser level (muxer.hpp:249-252)."""
        return self.is_child() and not self.is_parent()

    def push_parent(self, mirror):
        self.parent_mirror = torch.as_tensor(mirror, dtype=torch.long)

    def push_child(self, mirror):
        self.child_mirrors.append(torch.as_tensor(mirror, dtype=torch.long))

    def compile(self, device="cpu"):
        if self.parent_mirror is None:
            raise ValueError("Muxer.compile: push_parent first")
        if self.is_child() and self.is_parent() and len(self.child_mirrors) != self._size():
            raise ValueError("Muxer.compile: the parent needs one child mirror per rank")
        self.parent_mirror = self.parent_mirror.to(device)
        self.child_mirrors = [m.to(device) for m in self.child_mirrors]
        n = torch.tensor([self.parent_mirror.numel()], dtype=torch.int64, device=device)
        if self.is_child():
            self.dist.all_reduce(n, op=self.dist.ReduceOp.MAX)
        self.bufsize = int(n.item())
        self.device = device
        return self

    def _own_buffer(self, v: torch.Tensor) -> torch.Tensor:
        buf = torch.zeros(self.bufsize, dtype=v.dtype, device=v.device)
        buf[: self.parent_mirror.numel()] = v.index_select(0, self.parent_mirror)
        return buf

    def _from_buffer(self, buf: torch.Tensor, n_local: int) -> torch.Tensor:
        v = torch.zeros(n_local, dtype=buf.dtype, device=buf.device)
        return v.index_add_(0, self.parent_mirror, buf[: self.parent_mirror.numel()])

    def join_send(self, v: torch.Tensor):
        self.dist.gather(self._own_buffer(v), None, dst=self.parent)

    def join(self, v: torch.Tensor, n_trg: int) -> torch.Tensor:
        if not self.is_child():
            return v.clone()
        bufs = [torch.empty(self.bufsize, dtype=v.dtype, device=v.device) for _ in range(self._size())]
        self.dist.gather(self._own_buffer(v), bufs, dst=self.parent)
        trg = torch.zeros(n_trg, dtype=v.dtype, device=v.device)
        for m, b in zip(self.child_mirrors, bufs):
            trg.index_add_(0, m, b[: m.numel()])
        return trg

    def split_recv(self, n_local: int, dtype=torch.float64) -> torch.Tensor:
        buf = torch.empty(self.bufsize, dtype=dtype, device=self.device)
        self.dist.scatter(buf, None, src=self.parent)
        return self._from_buffer(buf, n_local)

    def split(self, v: torch.Tensor, n_local: int) -> torch.Tensor:
        if not self.is_child():
            return v.clone()
        bufs = []
        for m in self.child_mirrors:
            b = torch.zeros(self.bufsize, dtype=v.dtype, device=v.device)
            b[: m.numel()] = v.index_select(0, m)
            bufs.append(b)
        buf = torch.empty(self.bufsize, dtype=v.dtype, device=v.device)
        self.dist.scatter(buf, bufs, src=self.parent)
        return self._from_buffer(buf, n_local)


class GlobalTransfer:
    """Global::Transfer (kernel/global/transfer.hpp:252-336) between a fine level and the next
    coarser one.

    prol / rest: the patch-local products (callables returning new tensors): the row-scaled
    prolongation (patch coarse -> patch fine) and its transpose.  gate_fine: the fine level's gate;
    gate_coarse: the coarse level's gate (on the parent, the merged level's; unused on a ghost).
    With a muxer the coarse level is merged on its parent: coarse_local_size is this rank's patch-local
    coarse size, coarse_size the merged level's size on the parent."""

    def __init__(self, prol, rest, gate_fine: Gate, gate_coarse: Gate | None = None, muxer: Muxer | None = None,
                 coarse_local_size: int | None = None, coarse_size: int | None = None):
        self._prol, self._rest = prol, rest
        self.gate_fine, self.gate_coarse, self.muxer = gate_fine, gate_coarse, muxer
        self.coarse_local_size, self.coarse_size = coarse_local_size, coarse_size
        if muxer is not None and muxer.is_child() and coarse_local_size is None:
            raise ValueError("GlobalTransfer: a muxed transfer needs coarse_local_size")

    def _muxed(self) -> bool:
        return self.muxer is not None and self.muxer.is_child()

    def is_ghost(self) -> bool:
        return self.muxer is not None and self.muxer.is_ghost()

    def rest(self, vec_fine: torch.Tensor) -> torch.Tensor:
        """Type-1 fine defect -> type-1 coarse defect."""
        tmp = self._rest(vec_fine)
        vec_coarse = self.muxer.join(tmp, self.coarse_size) if self._muxed() else tmp
        if self.gate_coarse is not None:
            self.gate_coarse.sync_0(vec_coarse)
        return vec_coarse

    def rest_send(self, vec_fine: torch.Tensor):
        self.muxer.join_send(self._rest(vec_fine))

    def prol(self, vec_coarse: torch.Tensor) -> torch.Tensor:
        """Type-1 coarse vector -> type-1 fine vector."""
        tmp = self.muxer.split(vec_coarse, self.coarse_local_size) if self._muxed() else vec_coarse
        return self.gate_fine.sync_0(self._prol(tmp))

    def prol_recv(self, dtype=torch.float64) -> torch.Tensor:
        return self.gate_fine.sync_0(self._prol(self.muxer.split_recv(self.coarse_local_size, dtype)))


def coarse_inverse(A: torch.Tensor, filter_idx):
    """The exact coarse solve: the inverse of the dense coarse matrix restricted to its free
    (unfiltered) DOFs; the solution is zero on the filtered DOFs."""
    n = A.shape[0]
    free = torch.ones(n, dtype=torch.bool, device=A.device)
    free[torch.as_tensor(filter_idx, dtype=torch.long, device=A.device)] = False
    inv = torch.linalg.inv(A[free][:, free])

    def solve(b: torch.Tensor) -> torch.Tensor:
        x = torch.zeros_like(b)
        x[free] = inv @ b[free]
        return x
    return solve


class GlobalMultiGrid:
    """Solver::MultiGrid (kernel/solver/multigrid.hpp:1270-2000) on global levels: the V, F or W
    cycle (_apply_cycle_v / _f / _w, :1335-1510) with the fixed or an adaptive coarse-grid
    correction (MultiGridAdaptCGC MinEnergy / MinDefect, :1880-1960), `steps` Richardson steps
    preconditioned by Jacobi omega / diag(A) (the global diagonal) as pre-, post- and peak smoother
    (kernel/solver/richardson.hpp:160-228) and an exact coarse solve.

    levels: finest first, dicts with "matrix" (GlobalMatrix), "filter" (GlobalUnitFilter) and, on
    every level but the coarsest, "transfer" (GlobalTransfer).  On a ghost rank the list ends with
    the level whose transfer is a ghost; there `coarse_solve` is unused.  The coarse solve runs on
    the coarsest level: the parent's merged one, or every rank's without a muxer.  Every rank runs
    the cycle over its own levels, its last level being the coarse level or, on a ghost rank, one
    past its ghost level (multigrid.hpp:1386, 1445); the F and W cycles then cross the muxed transfer
    in the same order on every rank, as rest_send / prol_recv on the ghosts."""

    EPS = 2.220446049250313e-16

    def __init__(self, levels, coarse_solve=None, omega=0.7, steps=2, cycle="V", cgc="fixed"):
        self.levels, self.coarse_solve, self.steps = levels, coarse_solve, int(steps)
        if cycle not in ("V", "F", "W") or cgc not in ("fixed", "energy", "defect"):
            raise ValueError("GlobalMultiGrid: cycle is V, F or W and cgc fixed, energy or defect")
        self.cycle, self.cgc = cycle, cgc
        last = levels[-1]
        self.ghost = "transfer" in last and last["transfer"].is_ghost()
        if not self.ghost and "transfer" in last:
            raise ValueError("GlobalMultiGrid: the coarsest level has a transfer that is not a ghost")
        if not self.ghost and coarse_solve is None:
            raise ValueError("GlobalMultiGrid: the coarsest level needs a coarse solve")
        self.last = len(levels) if self.ghost else len(levels) - 1
        self.dinv = []
        for lv in levels:
            if "transfer" in lv:
                self.dinv.append(omega / lv["matrix"].diagonal())
            else:
                self.dinv.append(None)

    def _smooth(self, k: int, rhs: torch.Tensor) -> torch.Tensor:
        """Richardson from a zero start with the initial-defect test (iterative.hpp:492-507):
        nothing to do for a non-finite or vanishing defect; min_iter = max_iter = steps."""
        A, filt = self.levels[k]["matrix"], self.levels[k]["filter"]
        out = torch.zeros_like(rhs)
        d = rhs.clone()
        def_init = A.gate.norm2(d)
        if not math.isfinite(def_init) or def_init <= self.EPS * self.EPS:
            return out
        for _ in range(self.steps):
            z = self.dinv[k] * d
            filt.filter_cor(z)
            out.add_(z)
            A.apply_axpy(d, out, rhs, -1.0)
            filt.filter_def(d)
            if def_init > 1.0 / (self.EPS * self.EPS):
                break                                # Status::diverged
        return out

    def _rest(self, cur: int, smooth: bool):
        """_apply_rest (multigrid.hpp:1713-1838): pre-smoothing and defect on every level from cur
        (not on cur itself unless smooth), restriction to the next level; a ghost sends it."""
        L = self.levels
        for i in range(cur, self.last):
            A, filt, T = L[i]["matrix"], L[i]["filter"], L[i]["transfer"]
            if smooth or i > cur:
                self.sol[i] = self._smooth(i, self.rhs[i])
                if self.dfc[i] is None:
                    self.dfc[i] = torch.empty_like(self.rhs[i])
                A.apply_axpy(self.dfc[i], self.sol[i], self.rhs[i], -1.0)
            filt.filter_def(self.dfc[i])
            if T.is_ghost():
                T.rest_send(self.dfc[i])
                return
            self.rhs[i + 1] = T.rest(self.dfc[i])
            L[i + 1]["filter"].filter_def(self.rhs[i + 1])

    def _coarse(self):
        """_apply_coarse: nothing on a rank without the coarse level."""
        if not self.ghost:
            c = len(self.levels) - 1
            self.sol[c] = self.coarse_solve(self.rhs[c])

    def _prol(self, cur: int, smooth: bool):
        """_apply_prol (multigrid.hpp:1845-2000): prolongation (a ghost receives it), coarse-grid
        correction, post-smoothing on every level down to cur (not on cur itself unless smooth)."""
        L = self.levels
        for i in range(self.last - 1, cur - 1, -1):
            A, filt, T = L[i]["matrix"], L[i]["filter"], L[i]["transfer"]
            cor = T.prol_recv(self.dtype) if T.is_ghost() else T.prol(self.sol[i + 1])
            filt.filter_def(cor)
            w = 1.0
            if self.cgc != "fixed":
                tmp = torch.empty_like(cor)
                A.apply(tmp, cor)
                filt.filter_def(tmp)
                if self.cgc == "energy":
                    w = A.gate.dot(self.dfc[i], cor) / A.gate.dot(tmp, cor)
                else:
                    w = A.gate.dot(self.dfc[i], tmp) / A.gate.dot(tmp, tmp)
            self.sol[i].add_(cor, alpha=w)
            if smooth or i > cur:
                if self.cgc != "fixed":
                    self.dfc[i].add_(tmp, alpha=-w)
                else:
                    A.apply_axpy(self.dfc[i], self.sol[i], self.rhs[i], -1.0)
                    filt.filter_def(self.dfc[i])
                self.sol[i].add_(self._smooth(i, self.dfc[i]))

    def _peak(self, k: int):
        """_apply_smooth_peak + _apply_smooth_def (multigrid.hpp:1591-1700)."""
        A, filt = self.levels[k]["matrix"], self.levels[k]["filter"]
        A.apply_axpy(self.dfc[k], self.sol[k], self.rhs[k], -1.0)
        filt.filter_def(self.dfc[k])
        cor = self._smooth(k, self.dfc[k])
        filt.filter_def(cor)
        self.sol[k].add_(cor)
        A.apply_axpy(self.dfc[k], self.sol[k], self.rhs[k], -1.0)
        filt.filter_def(self.dfc[k])

    def vcycle(self, d: torch.Tensor) -> torch.Tensor:
        """One cycle: the correction for the type-1 defect d on the finest level."""
        n = len(self.levels)
        self.dtype = d.dtype
        self.rhs, self.sol, self.dfc = [None] * n, [None] * n, [None] * n
        self.rhs[0] = d.clone()
        self._rest(0, True)
        if self.cycle == "F":
            for pk in range(self.last - 1, 0, -1):
                self._coarse()
                self._prol(pk, False)
                self._peak(pk)
                self._rest(pk, False)
        elif self.cycle == "W":
            self._coarse()
            counters = [0] * (self.last + 1)
            for _ in range(1, 1 << self.last):
                pk = self.last
                while pk > 0:
                    pk -= 1
                    if counters[pk] == 0:
                        break
                for i in range(self.last - 1, pk, -1):
                    counters[i] = 0
                counters[pk] += 1
                self._prol(pk, False)
                self._peak(pk)
                self._rest(pk, False)
                self._coarse()
        if self.cycle != "W":
            self._coarse()
        self._prol(0, True)
        return self.sol[0]

    __call__ = vcycle


def global_pcg(A: GlobalMatrix, filt: GlobalUnitFilter, rhs: torch.Tensor, x: torch.Tensor, omega=1.0,
               tol_rel=1e-8, max_iter=1000, precond=None):
    """Solver::PCG (kernel/solver/pcg.hpp:188-286) on global vectors.  The preconditioner is
    `precond` (a callable on a type-1 defect, e.g. a `GlobalMultiGrid`) or, when None, the global
    Jacobi omega / diag(A) (kernel/solver/jacobi_precond.hpp:136-165).  rhs and x are type 1; x holds
    the initial guess and receives the solution.  Returns (iterations, def_init, def_final,
    converged)."""
    gate = A.gate
    if precond is None:
        dinv = omega / A.diagonal()
        filt.filter_cor(dinv)                   # the filtered rows never contribute

        def precond(v):
            return dinv * v
    r = torch.empty_like(x)
    A.apply_axpy(r, x, rhs, -1.0)
    filt.filter_def(r)
    d0 = gate.norm2(r)
    dc = d0
    if not math.isfinite(d0):
        return 0, d0, dc, False                 # Status::aborted
    if d0 <= GlobalMultiGrid.EPS * GlobalMultiGrid.EPS:
        return 0, d0, dc, True
    z = precond(r)
    filt.filter_cor(z)
    p = z.clone()
    gamma = gate.dot(r, z)
    q = torch.empty_like(x)
    it = 0
    while it < max_iter:
        A.apply(q, p)
        filt.filter_def(q)
        alpha = gamma / gate.dot(q, p)
        x.add_(p, alpha=alpha)
        r.add_(q, alpha=-alpha)
        it += 1
        dc = gate.norm2(r)
        if dc <= tol_rel * d0:
            return it, d0, dc, True
        z = precond(r)
        filt.filter_cor(z)
        gamma_new = gate.dot(r, z)
        p = z + (gamma_new / gamma) * p
        gamma = gamma_new
    return it, d0, dc, False

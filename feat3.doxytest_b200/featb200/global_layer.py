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

Vectors are torch tensors: on CUDA devices with the NCCL backend the exchange runs over NVLink,
on the CPU with gloo (the tests).  The exchange is point-to-point (`isend` / `irecv` of the gathered
buffers) because only neighbours share DOFs.  The local matrix product is a callable, so that the
product path can use the library's device SpMV and the tests a host CSR product.
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

    def _sum(self, x: float) -> float:
        if self._world() == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64)
        if self.freqs is not None and self.freqs.is_cuda:
            t = t.cuda()
        self.dist.all_reduce(t)
        return float(t.item())

    def dot(self, x: torch.Tensor, y: torch.Tensor) -> float:
        """Global dot product of two type-1 vectors (gate.hpp:476-492)."""
        if self._world() == 1:
            return float(torch.dot(x, y))
        if not self.ranks:
            return self._sum(float(torch.dot(x, y)))
        return self._sum(float(torch.sum(self.freqs * x * y)))

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


def global_pcg(A: GlobalMatrix, filt: GlobalUnitFilter, rhs: torch.Tensor, x: torch.Tensor, omega=1.0,
               tol_rel=1e-8, max_iter=1000):
    """Solver::PCG (kernel/solver/pcg.hpp:188-286) on global vectors with the global Jacobi
    preconditioner omega / diag(A) (kernel/solver/jacobi_precond.hpp:136-165).  rhs and x are type 1;
    x holds the initial guess and receives the solution.  Returns (iterations, def_init, def_final,
    converged)."""
    gate = A.gate
    dinv = omega / A.diagonal()
    filt.filter_cor(dinv)                       # the filtered rows never contribute
    r = torch.empty_like(x)
    A.apply_axpy(r, x, rhs, -1.0)
    filt.filter_def(r)
    z = dinv * r
    filt.filter_cor(z)
    p = z.clone()
    gamma = gate.dot(r, z)
    d0 = gate.norm2(r)
    dc = d0
    q = torch.empty_like(x)
    it = 0
    if d0 <= 0.0:
        return 0, d0, dc, True
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
        z = dinv * r
        filt.filter_cor(z)
        gamma_new = gate.dot(r, z)
        p = z + (gamma_new / gamma) * p
        gamma = gamma_new
    return it, d0, dc, False

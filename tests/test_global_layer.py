"""The global layer (overlapping domain decomposition, kernel/global/gate.hpp and matrix.hpp) over a
world_size-2 gloo process group on CPU: a 2D Q1 Poisson problem split into two patches that share
one column of vertices.  Each rank assembles its patch (type-0 matrix and load vector); the gate's
sync_0 and dot, the global matrix product and the global Jacobi-PCG are checked against the same
problem assembled and solved in one piece."""
import os
import socket

import numpy as np
import pytest
import scipy.sparse as sp
import torch.multiprocessing as mp

from featb200 import assembly as AS

LEVEL = 5


def _assemble_cells(level, cells_sel):
    """Stiffness matrix and sine-bubble load vector over a subset of the level's cells (global
    vertex numbering): the patch-local (type-0) contributions."""
    N = 2 ** level
    h = 1.0 / N
    pts, w, val, grad = AS._q1_ref(2)
    fac = (h / 2.0) ** 2 * (2.0 / h) ** 2
    kloc = fac * np.einsum("q,qvu->vu", w, np.einsum("qvd,qud->qvu", grad, grad))
    conn, idx = AS._cells(level, 2)
    conn, idx = conn[cells_sel], idx[:, cells_sel]
    nv = (N + 1) ** 2
    rows = np.repeat(conn, 4, axis=1).ravel()
    cols = np.tile(conn, (1, 4)).ravel()
    A = sp.coo_matrix((np.broadcast_to(kloc, (conn.shape[0], 4, 4)).ravel(), (rows, cols)), shape=(nv, nv)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    xq = [(idx[d][:, None] + (1.0 + pts[None, :, d]) / 2.0) * h for d in range(2)]
    fq = AS.sine_bubble_rhs(*xq)
    loc = (h / 2.0) ** 2 * np.einsum("cq,q,qv->cv", fq, w, val)
    b = np.bincount(conn.ravel(), weights=loc.ravel(), minlength=nv)
    return A, b


def _patch(level, rank):
    """Cells with x-index in the rank's half; the rank's vertices in global order; the mirror of the
    shared column; the Dirichlet DOFs; patch matrix and load vector in local numbering."""
    N = 2 ** level
    _, idx = AS._cells(level, 2)
    sel = (idx[0] < N // 2) if rank == 0 else (idx[0] >= N // 2)
    A, b = _assemble_cells(level, sel)
    vx = np.arange((N + 1) ** 2) % (N + 1)
    mine = np.nonzero(vx <= N // 2)[0] if rank == 0 else np.nonzero(vx >= N // 2)[0]
    Al = A[mine][:, mine].tocsr()
    shared = np.nonzero(vx[mine] == N // 2)[0]
    bnd = np.isin(mine, AS.boundary_dofs(level).astype(np.int64))
    return mine, Al, b[mine], shared, np.nonzero(bnd)[0]


def _global_problem(level):
    N = 2 ** level
    A, b = _assemble_cells(level, np.ones(N * N, dtype=bool))
    return A, b, AS.boundary_dofs(level).astype(np.int64)


def _pcg_reference(A, b, bnd, omega=1.0, tol=1e-8, max_iter=1000):
    dinv = omega / A.diagonal()
    dinv[bnd] = 0.0
    x = np.zeros_like(b)
    r = b - A @ x
    r[bnd] = 0.0
    z = dinv * r
    p = z.copy()
    gamma = r @ z
    d0 = np.linalg.norm(r)
    for it in range(1, max_iter + 1):
        q = A @ p
        q[bnd] = 0.0
        alpha = gamma / (q @ p)
        x += alpha * p
        r -= alpha * q
        if np.linalg.norm(r) <= tol * d0:
            return x, it
        z = dinv * r
        gn = r @ z
        p = z + (gn / gamma) * p
        gamma = gn
    return x, max_iter


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    from featb200.global_layer import Gate, GlobalMatrix, GlobalUnitFilter, global_pcg
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine, Al, bl, shared, bnd = _patch(LEVEL, rank)
        gate = Gate(dist)
        gate.push(1 - rank, shared)
        gate.compile(len(mine))
        Ag, bg, bndg = _global_problem(LEVEL)
        # sync_0 turns the patch load vectors into the global one; dot is the global dot product
        b = torch.tensor(bl)
        gate.sync_0(b)
        err_b = float(np.abs(b.numpy() - bg[mine]).max())
        xg = np.sin(np.arange(bg.size) * 0.37)
        xl = torch.tensor(xg[mine])
        dot_err = abs(gate.dot(xl, xl) - float(xg @ xg)) / float(xg @ xg)
        # the global matrix product
        A = GlobalMatrix(lambda v: torch.tensor(Al @ v.numpy()), gate, torch.tensor(Al.diagonal()))
        r = torch.empty_like(xl)
        A.apply(r, xl)
        err_ax = float(np.abs(r.numpy() - (Ag @ xg)[mine]).max() / np.abs(Ag @ xg).max())
        # the global Jacobi-PCG against the same solver on the assembled problem
        x = torch.zeros(len(mine), dtype=torch.float64)
        it, d0, dc, ok = global_pcg(A, GlobalUnitFilter(bnd), b, x, omega=1.0, tol_rel=1e-8)
        xr, itr = _pcg_reference(Ag, bg, bndg)
        sol_err = float(np.abs(x.numpy() - xr[mine]).max() / np.abs(xr).max())
        q.put((rank, err_b, dot_err, err_ax, it, itr, ok, sol_err))
    finally:
        dist.destroy_process_group()


def test_global_layer_two_patches_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, err_b, dot_err, err_ax, it, itr, ok, sol_err in res:
        assert err_b <= 1e-15, (rank, err_b)
        assert dot_err <= 1e-13, (rank, dot_err)
        assert err_ax <= 1e-14, (rank, err_ax)
        assert ok and it == itr, (rank, it, itr)
        assert sol_err <= 1e-12, (rank, sol_err)
    assert res[0][4] == res[1][4]


def test_gate_single_rank_is_local():
    import torch
    from featb200.global_layer import Gate
    g = Gate(None).compile(5)
    x = torch.arange(5, dtype=torch.float64)
    assert g.dot(x, x) == float(x @ x)
    y = x.clone()
    assert torch.equal(g.sync_0(y), x) and torch.equal(g.sync_1(y), x)


@pytest.mark.gpu
def test_global_pcg_on_device_one_rank(featlib, cuda):
    """The device form of the global layer with one rank: the patch product through the library's
    CSR kernel on CUDA tensors, the PCG on device vectors; same iterations and solution as the
    assembled problem."""
    torch = cuda
    from featb200.global_layer import Gate, GlobalMatrix, GlobalUnitFilter, device_csr_apply, global_pcg
    from featb200.lafem import SparseMatrixCSR
    Ag, bg, bnd = _global_problem(LEVEL)
    gate = Gate(None).compile(bg.size, device="cuda")
    A = GlobalMatrix(device_csr_apply(SparseMatrixCSR.from_scipy(Ag)), gate,
                     torch.tensor(Ag.diagonal(), device="cuda"))
    x = torch.zeros(bg.size, dtype=torch.float64, device="cuda")
    it, d0, dc, ok = global_pcg(A, GlobalUnitFilter(bnd).to("cuda"), torch.tensor(bg, device="cuda"), x)
    xr, itr = _pcg_reference(Ag, bg, bnd)
    assert ok and it == itr
    assert float(np.abs(x.cpu().numpy() - xr).max() / np.abs(xr).max()) <= 1e-12

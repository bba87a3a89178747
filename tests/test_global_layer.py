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


def _strip_bounds(level, world, base):
    """x-index bounds of the ranks' vertical strips at `level`: floor(r 2^base / world) cell columns
    on level `base`, refined by 2 per level, so that every patch is the refinement of its patch on
    the coarser levels down to `base`."""
    nb = 2 ** base
    f = 2 ** (level - base)
    return [(r * nb // world) * f for r in range(world + 1)]


def _strip_vertices(level, rank, world=2, base=None):
    b = _strip_bounds(level, world, level if base is None else base)
    vx = np.arange((2 ** level + 1) ** 2) % (2 ** level + 1)
    return np.nonzero((vx >= b[rank]) & (vx <= b[rank + 1]))[0]


def _strip_cells(level, rank, world=2, base=None):
    b = _strip_bounds(level, world, level if base is None else base)
    _, idx = AS._cells(level, 2)
    return (idx[0] >= b[rank]) & (idx[0] < b[rank + 1])


def _patch(level, rank, world=2, base=None):
    """The rank's vertical strip of cells: its vertices in global order, the patch matrix and load
    vector in local numbering (type 0), the mirrors [(neighbour rank, local indices of the shared
    column in ascending global order)] and the Dirichlet DOFs."""
    N = 2 ** level
    b = _strip_bounds(level, world, level if base is None else base)
    A, bv = _assemble_cells(level, _strip_cells(level, rank, world, base))
    vx = np.arange((N + 1) ** 2) % (N + 1)
    mine = _strip_vertices(level, rank, world, base)
    Al = A[mine][:, mine].tocsr()
    nbrs = []
    if rank > 0:
        nbrs.append((rank - 1, np.nonzero(vx[mine] == b[rank])[0]))
    if rank < world - 1:
        nbrs.append((rank + 1, np.nonzero(vx[mine] == b[rank + 1])[0]))
    bnd = np.isin(mine, AS.boundary_dofs(level).astype(np.int64))
    return mine, Al, bv[mine], nbrs, np.nonzero(bnd)[0]


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
        mine, Al, bl, nbrs, bnd = _patch(LEVEL, rank)
        gate = Gate(dist)
        for nb, shared in nbrs:
            gate.push(nb, shared)
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



def test_muxer_and_transfer_single_rank():
    """Without siblings the muxer is no child: join and split copy, the transfer is the patch-local
    one, and a muxer without a parent mirror refuses to compile."""
    import torch
    from featb200.global_layer import Gate, GlobalTransfer, Muxer
    with pytest.raises(ValueError):
        Muxer(None).compile()
    m = Muxer(None)
    m.push_parent([0, 1, 2])
    m.push_child([0, 1, 2])
    m.compile()
    assert not m.is_child() and m.is_parent() and not m.is_ghost() and m.bufsize == 3
    v = torch.tensor([1.0, 2.0, 3.0], dtype=torch.float64)
    assert torch.equal(m.join(v, 3), v) and torch.equal(m.split(v, 3), v)
    P = torch.tensor([[1.0, 0.0], [0.5, 0.5], [0.0, 1.0]], dtype=torch.float64)
    T = GlobalTransfer(lambda c: P @ c, lambda f: P.T @ f, Gate(None).compile(3), Gate(None).compile(2), m,
                       coarse_local_size=2, coarse_size=2)
    assert not T.is_ghost()
    assert torch.equal(T.rest(v), P.T @ v)
    c = torch.tensor([4.0, 6.0], dtype=torch.float64)
    assert torch.equal(T.prol(c), P @ c)

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


# --- the global multigrid: Global::Transfer, Global::Muxer and the V-cycle on global levels ---

def _prolongation_cells(level_f, csel):
    """Assembly::GridTransfer::assemble_prolongation over the selected coarse cells of level_f - 1:
    every coarse cell adds the bilinear interpolation weights of the 3x3 fine vertices it covers, and
    1 to the weight of each of them.  Returns the summed matrix and the weight vector."""
    Nf = 2 ** level_f
    Nc = Nf // 2
    _, idx = AS._cells(level_f - 1, 2)
    cx, cy = idx[0][csel], idx[1][csel]
    rows, cols, vals, wrows = [], [], [], []
    for a in range(3):
        for b in range(3):
            fine = (2 * cy + b) * (Nf + 1) + 2 * cx + a
            wrows.append(fine)
            for p in range(2):
                for q in range(2):
                    v = (a / 2.0 if p else 1.0 - a / 2.0) * (b / 2.0 if q else 1.0 - b / 2.0)
                    if v != 0.0:
                        rows.append(fine)
                        cols.append((cy + q) * (Nc + 1) + cx + p)
                        vals.append(np.full(fine.size, v))
    P = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=((Nf + 1) ** 2, (Nc + 1) ** 2)).tocsr()
    P.sum_duplicates()
    P.sort_indices()
    w = np.bincount(np.concatenate(wrows), minlength=(Nf + 1) ** 2).astype(np.float64)
    return P, w


def _mg_levels(rank, merge, dist, world):
    """Rank's global levels, finest first: levels LEVEL..merge+1 split into `world` vertical strips
    (bounds fixed on level `merge`, so every patch refines a set of the merged level's cells), levels
    merge..1 merged on rank 0 (the muxer's parent) and absent on the other ranks (ghosts below
    merge + 1)."""
    import torch
    from featb200.global_layer import (Gate, GlobalMatrix, GlobalTransfer, GlobalUnitFilter, Muxer,
                                       coarse_inverse, prolongation_row_scaling)

    def csr_op(M):
        return lambda v: torch.tensor(M @ v.numpy())

    levels = []
    for lv in range(LEVEL, merge, -1):
        mine, Al, _, nbrs, bnd = _patch(lv, rank, world, merge)
        gate = Gate(dist)
        for nb, shared in nbrs:
            gate.push(nb, shared)
        gate.compile(len(mine))
        levels.append({"matrix": GlobalMatrix(csr_op(Al), gate, torch.tensor(Al.diagonal())),
                       "filter": GlobalUnitFilter(bnd), "mine": mine})
    parent = rank == 0
    if parent:
        for lv in range(merge, 0, -1):
            A, _, bnd = _global_problem(lv)
            levels.append({"matrix": GlobalMatrix(csr_op(A), Gate(None).compile(A.shape[0]),
                                                  torch.tensor(A.diagonal())),
                           "filter": GlobalUnitFilter(bnd)})
    # transfers: patch -> patch, the muxed patch -> merged one, merged -> merged
    for k in range(len(levels) - (0 if not parent else 1)):
        lv = LEVEL - k
        fine = levels[k]
        if lv > merge:
            mine_f = fine["mine"]
            Nc = 2 ** (lv - 1)
            Psum, w = _prolongation_cells(lv, _strip_cells(lv - 1, rank, world, merge))
            mine_c = _strip_vertices(lv - 1, rank, world, merge)
            Ploc = Psum[mine_f][:, mine_c]
            s = prolongation_row_scaling(torch.tensor(w[mine_f]), fine["matrix"].gate).numpy()
            Ploc = sp.diags(s) @ Ploc
            Rloc = Ploc.T.tocsr()
            if lv - 1 > merge:
                T = GlobalTransfer(csr_op(Ploc), csr_op(Rloc), fine["matrix"].gate, levels[k + 1]["matrix"].gate)
            else:
                mux = Muxer(dist, parent=0)
                mux.push_parent(np.arange(mine_c.size))
                if parent:
                    for r in range(world):
                        mux.push_child(_strip_vertices(lv - 1, r, world, merge))
                mux.compile()
                T = GlobalTransfer(csr_op(Ploc), csr_op(Rloc), fine["matrix"].gate,
                                   levels[k + 1]["matrix"].gate if parent else None, mux,
                                   coarse_local_size=mine_c.size, coarse_size=(Nc + 1) ** 2)
        else:
            P = AS.prolongation(lv)
            T = GlobalTransfer(csr_op(P), csr_op(P.T.tocsr()), fine["matrix"].gate, levels[k + 1]["matrix"].gate)
        fine["transfer"] = T
    coarse = None
    if parent:
        A1, _, bnd1 = _global_problem(1)
        coarse = coarse_inverse(torch.tensor(A1.toarray()), bnd1)
    return levels, coarse


def _mg_worker(rank, world, port, q, configs):
    import datetime

    import torch
    import torch.distributed as dist
    from featb200.global_layer import GlobalMultiGrid, global_pcg
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = {}
        for merge, cycle, cgc in configs:
            levels, coarse = _mg_levels(rank, merge, dist, world)
            mg = GlobalMultiGrid(levels, coarse, omega=0.7, steps=2, cycle=cycle, cgc=cgc)
            top = levels[0]
            mine = top["mine"]
            # one V-cycle on a fixed (filtered, type-1) defect
            Ag, bg, bndg = _global_problem(LEVEL)
            dg = np.sin(np.arange(bg.size) * 0.61)
            dg[bndg] = 0.0
            z = mg.vcycle(torch.tensor(dg[mine]))
            # PCG preconditioned by the global multigrid, from the patch load vectors
            _, _, bl, _, _ = _patch(LEVEL, rank, world, merge)
            b = top["matrix"].gate.sync_0(torch.tensor(bl))
            top["filter"].filter_def(b)
            x = torch.zeros(len(mine), dtype=torch.float64)
            it, d0, dc, ok = global_pcg(top["matrix"], top["filter"], b, x, tol_rel=1e-8, max_iter=100,
                                        precond=mg)
            out[(merge, cycle, cgc)] = (mine, z.numpy(), x.numpy(), it, ok, mg.ghost)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_prolongation_assembly_weights_give_the_interpolation():
    """The summed cell contributions divided by the weights are the Q1 interpolation, on the whole
    mesh and, after prolongation_row_scaling's global weights, as the sum of the two patches."""
    import torch
    from featb200.global_layer import Gate, prolongation_row_scaling
    for lv in (2, 5):
        Nc = 2 ** (lv - 1)
        Psum, w = _prolongation_cells(lv, np.ones(Nc * Nc, dtype=bool))
        P = AS.prolongation(lv)
        assert abs(sp.diags(1.0 / w) @ Psum - P).max() == 0.0
        parts = [_prolongation_cells(lv, _strip_cells(lv - 1, r)) for r in range(2)]
        wsum = parts[0][1] + parts[1][1]        # what sync_0 forms on the shared DOFs
        Pg = sp.diags(1.0 / wsum) @ (parts[0][0] + parts[1][0])
        assert abs(Pg - P).max() == 0.0
    g = Gate(None).compile(3)
    s = prolongation_row_scaling(torch.tensor([2.0, 4.0, 1.0], dtype=torch.float64), g)
    assert torch.equal(s, torch.tensor([0.5, 0.25, 1.0], dtype=torch.float64))


def _oracle_mg_reference(O, cycle="V", cgc="fixed"):
    """The oracle's single-system cycle of the fixed defect and PCG-multigrid solution."""
    lv_ref = []
    for lv in range(LEVEL, 0, -1):
        A, _, bnd = _global_problem(lv)
        d = {"A": O.Csr.of(A.indptr, A.indices, A.data, A.shape), "filter_idx": bnd.astype(np.uint64)}
        if lv > 1:
            P = AS.prolongation(lv)
            R = P.T.tocsr()
            d["P"] = O.Csr.of(P.indptr, P.indices, P.data, P.shape)
            d["R"] = O.Csr.of(R.indptr, R.indices, R.data, R.shape)
        lv_ref.append(d)
    mg = O.MultigridPCG(lv_ref, 0.7, 2, cycle=cycle, cgc=cgc)
    Ag, bg, bndg = _global_problem(LEVEL)
    dg = np.sin(np.arange(bg.size) * 0.61)
    dg[bndg] = 0.0
    z_ref = mg.vcycle(dg)
    b = bg.copy()
    b[bndg] = 0.0
    x_ref, info = mg.solve(b, tol_rel=1e-8, max_iter=100)
    assert info["status"] == "success"
    return z_ref, x_ref, info["iters"]


def _run_strips(oracle_lib, world, configs, tol_z, tol_x):
    from helpers import rel_err
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mg_worker, args=(r, world, port, q, configs)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    refs = {}
    for cfg in configs:
        key = cfg[1:]
        if key not in refs:
            refs[key] = _oracle_mg_reference(oracle_lib, *key)
        z_ref, x_ref, iters = refs[key]
        covered = np.zeros(z_ref.size, dtype=bool)
        for rank in range(world):
            mine, z, x, it, ok, ghost = res[rank][cfg]
            covered[mine] = True
            assert ghost == (rank != 0)
            assert rel_err(z, z_ref[mine]) <= tol_z, (cfg, rank, rel_err(z, z_ref[mine]))
            assert ok and it == iters, (cfg, rank, it, iters)
            assert rel_err(x, x_ref[mine]) <= tol_x, (cfg, rank, rel_err(x, x_ref[mine]))
        assert covered.all()


@pytest.mark.parametrize("world,merges", [(2, (1, 3, 4)), (3, (2, 3)), (4, (2,))])
def test_global_multigrid_strips_gloo(oracle_lib, world, merges):
    """`world` gloo ranks, each holding one vertical strip of the 2D Q1 hierarchy on levels
    5..merge+1 (uneven strips for three ranks; the middle ranks have two neighbours), the levels
    merge..1 muxed onto rank 0 (merge 4: only the finest level is split): one global V-cycle and the
    multigrid-preconditioned global PCG against the oracle's single-system V-cycle and PCG on the
    whole hierarchy (same operation order; only the split sums of the shared rows differ in
    rounding)."""
    _run_strips(oracle_lib, world, [(m, "V", "fixed") for m in merges], 1e-13, 1e-12)


@pytest.mark.parametrize("world,merge", [(2, 1), (3, 2)])
def test_global_multigrid_fw_cycles_gloo(oracle_lib, world, merge):
    """F and W cycles and the adaptive coarse-grid corrections on the strips, with the coarse
    levels muxed onto rank 0: the ghost ranks cross the muxed transfer in the parent's order (the
    test would hang or fail otherwise); cycle and solution against the oracle run with the same
    cycle and correction (the adaptive step lengths come from global dot products, summed in
    another order than the oracle's)."""
    configs = [(merge, "F", "fixed"), (merge, "W", "fixed"), (merge, "V", "energy"), (merge, "F", "defect"),
               (merge, "W", "energy")]
    _run_strips(oracle_lib, world, configs, 1e-12, 1e-12)


@pytest.mark.gpu
def test_global_multigrid_on_device_one_rank(featlib, cuda, oracle_lib):
    """The device form of the global multigrid with one rank: every patch product (matrix,
    prolongation, restriction) through the library's CSR kernel on CUDA tensors; same iterations as
    the oracle's PCG-multigrid and the same solution to rounding."""
    torch = cuda
    O = oracle_lib
    from featb200.global_layer import (Gate, GlobalMatrix, GlobalMultiGrid, GlobalTransfer, GlobalUnitFilter,
                                       coarse_inverse, device_csr_apply, global_pcg)
    from featb200.lafem import SparseMatrixCSR
    from helpers import rel_err
    levels, lv_ref = [], []
    for lv in range(LEVEL, 0, -1):
        A, _, bnd = _global_problem(lv)
        gate = Gate(None).compile(A.shape[0], device="cuda")
        levels.append({"matrix": GlobalMatrix(device_csr_apply(SparseMatrixCSR.from_scipy(A)), gate,
                                              torch.tensor(A.diagonal(), device="cuda")),
                       "filter": GlobalUnitFilter(bnd).to("cuda")})
        d = {"A": O.Csr.of(A.indptr, A.indices, A.data, A.shape), "filter_idx": bnd.astype(np.uint64)}
        if lv > 1:
            P = AS.prolongation(lv)
            R = P.T.tocsr()
            levels[-1]["P"] = (P, R)
            d["P"] = O.Csr.of(P.indptr, P.indices, P.data, P.shape)
            d["R"] = O.Csr.of(R.indptr, R.indices, R.data, R.shape)
        lv_ref.append(d)
    for k in range(len(levels) - 1):
        P, R = levels[k].pop("P")
        levels[k]["transfer"] = GlobalTransfer(device_csr_apply(SparseMatrixCSR.from_scipy(P)),
                                               device_csr_apply(SparseMatrixCSR.from_scipy(R)),
                                               levels[k]["matrix"].gate, levels[k + 1]["matrix"].gate)
    A1, _, bnd1 = _global_problem(1)
    mg = GlobalMultiGrid(levels, coarse_inverse(torch.tensor(A1.toarray(), device="cuda"), bnd1), 0.7, 2)
    Ag, bg, bndg = _global_problem(LEVEL)
    b = bg.copy()
    b[bndg] = 0.0
    x = torch.zeros(bg.size, dtype=torch.float64, device="cuda")
    it, d0, dc, ok = global_pcg(levels[0]["matrix"], levels[0]["filter"], torch.tensor(b, device="cuda"), x,
                                tol_rel=1e-8, max_iter=100, precond=mg)
    ref = O.MultigridPCG(lv_ref, 0.7, 2)
    x_ref, info = ref.solve(b, tol_rel=1e-8, max_iter=100)
    assert ok and it == info["iters"]
    assert rel_err(x.cpu().numpy(), x_ref) <= 1e-12

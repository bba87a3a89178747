"""Device assembly of the 2D Q1 family and the solver's numeric update.

* fb_q1_pattern_2d (host code) gives exactly the pattern of the host assembler's CSR matrix.
* fb_q1_assemble_2d matches the host assembler (featb200.assembly, pinned to the reference's
  assembly by test_assembly) to 1e-12 relative: the stiffness and load vector are sums of a few
  products, and kappa = exp(g) is evaluated by a differently ordered Fourier sum.
* fb_solver_update_matrix on a solver built for kappa = 1 gives BITWISE the V-cycle, iterates and
  solution of a solver built directly from the new matrices (same pattern), in every precision.
"""
import numpy as np
import pytest

from featb200 import assembly as AS

TOL = 1e-12


def test_pattern_matches_host_assembler(featlib):
    from featb200.assembly_gpu import q1_pattern_2d
    for level in (0, 1, 3, 6):
        rp, ci = q1_pattern_2d(level)
        A = AS.stiffness(level, 2)
        assert np.array_equal(rp, A.indptr.astype(np.uint64))
        assert np.array_equal(ci, A.indices.astype(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("level", [2, 5, 7])
@pytest.mark.parametrize("with_field", [False, True])
def test_assembly_matches_host(featlib, cuda, level, with_field):
    torch = cuda
    from featb200.assembly_gpu import Q1Assembler2D
    fp = AS.field_params(40 + level) if with_field else None
    gp = AS.gauss_params(50 + level, 2)
    asm = Q1Assembler2D(level)
    vals, b = asm.assemble(fp, gp)
    torch.cuda.synchronize()
    kappa = None
    if fp is not None:
        def kappa(x, y, _fp=fp):
            xs, ys = np.unique(x), np.unique(y)
            G = AS.field_eval_grid(_fp, xs, ys)
            return np.exp(G[np.searchsorted(ys, y), np.searchsorted(xs, x)])
    A = AS.stiffness(level, 2, kappa)
    b_ref = AS.load_vector(level, lambda *xs: AS.gauss_eval(gp, *xs), 2)
    b_ref[AS.boundary_dofs(level, 2).astype(np.int64)] = 0.0
    v = vals.cpu().numpy()
    assert np.abs(v - A.data).max() <= TOL * np.abs(A.data).max()
    bb = b.cpu().numpy()
    assert np.abs(bb - b_ref).max() <= TOL * max(np.abs(b_ref).max(), 1e-300)


@pytest.mark.gpu
def test_assembly_values_only_and_rhs_only(featlib, cuda):
    torch = cuda
    from featb200.assembly_gpu import Q1Assembler2D
    asm = Q1Assembler2D(4)
    v1, b1 = asm.assemble(None, AS.gauss_params(1, 2))
    v2, _ = asm.assemble(None, None, rhs=False)
    _, b2 = asm.assemble(None, AS.gauss_params(1, 2), values=False)
    torch.cuda.synchronize()
    assert torch.equal(v1, v2) and torch.equal(b1, b2)


def _levels(level, field):
    return AS.poisson_hierarchy(level, 2, rhs="gauss", gauss=AS.gauss_params(3, 2), field=field)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32", "f32_bf16"])
@pytest.mark.parametrize("ordering", ["native", "rcm"])
def test_update_matrix_equals_fresh_solver(featlib, cuda, precision, ordering):
    fb, torch = featlib, cuda
    lv1, b1 = _levels(6, AS.field_params(4))
    lv0, _ = _levels(6, None)
    fresh = fb.build_pcg_multigrid(lv1, precision=precision, ordering=ordering)
    upd = fb.build_pcg_multigrid(lv0, precision=precision, ordering=ordering)
    for l, L in enumerate(lv1):
        upd.update_matrix(l, torch.tensor(L["matrix"].val, device="cuda"))
    z_f = fresh.apply_precond(fb.DenseVector(b1)).elements
    z_u = upd.apply_precond(fb.DenseVector(b1)).elements
    assert np.array_equal(z_f, z_u)
    x_f = fb.DenseVector(b1.size)
    x_u = fb.DenseVector(b1.size)
    st_f = fb.solve(fresh, x_f, fb.DenseVector(b1))
    st_u = fb.solve(upd, x_u, fb.DenseVector(b1))
    assert st_f == st_u == fb.Status.success
    assert fresh.get_num_iter() == upd.get_num_iter()
    assert np.array_equal(x_f.elements, x_u.elements)


@pytest.mark.gpu
def test_update_matrix_from_device_assembly(featlib, cuda):
    """The whole set-up on the device: assemble every level with a kappa field, update, solve; the
    result equals the solver built from the host assembler's matrices to the assembly tolerance."""
    fb, torch = featlib, cuda
    from featb200.assembly_gpu import Q1Assembler2D
    fp = AS.field_params(11)
    gp = AS.gauss_params(12, 2)
    lv_host, b_host = AS.poisson_hierarchy(6, 2, rhs="gauss", gauss=gp, field=fp)
    lv0, _ = _levels(6, None)
    s = fb.build_pcg_multigrid(lv0, precision="f64")
    b = None
    for l, L in enumerate(lv0):
        vals, bl = Q1Assembler2D(L["level"]).assemble(fp, gp if l == 0 else None, rhs=(l == 0))
        s.update_matrix(l, vals)
        if l == 0:
            b = bl
    x = torch.zeros_like(b)
    st = s.correct_device(x, b)
    torch.cuda.synchronize()
    assert st == fb.Status.success
    ref = fb.build_pcg_multigrid(lv_host, precision="f64")
    xr = fb.DenseVector(b_host.size)
    assert fb.solve(ref, xr, fb.DenseVector(b_host)) == fb.Status.success
    xx = x.cpu().numpy()
    assert np.abs(xx - xr.elements).max() <= 1e-9 * np.abs(xr.elements).max()


@pytest.mark.gpu
def test_update_matrix_rejects_bad_level(featlib, cuda):
    fb, torch = featlib, cuda
    lv0, _ = _levels(3, None)
    s = fb.build_pcg_multigrid(lv0, precision="f64")
    v = torch.zeros(10, dtype=torch.float64, device="cuda")
    with pytest.raises(fb.FeatB200Error):
        s.update_matrix(len(lv0), v)
    with pytest.raises(fb.FeatB200Error):
        s.update_matrix(-1, v)


@pytest.mark.gpu
@pytest.mark.parametrize("level", [1, 2, 5, 8])
def test_prolongation_matches_host(featlib, cuda, level):
    from featb200.assembly_gpu import q1_prolongation_2d
    rp, ci, v = q1_prolongation_2d(level)
    cuda.cuda.synchronize()
    P = AS.prolongation(level, 2).tocsr()
    P.sort_indices()
    assert np.array_equal(rp.cpu().numpy(), P.indptr.astype(np.int64))
    assert np.array_equal(ci.cpu().numpy(), P.indices.astype(np.int64))
    assert np.array_equal(v.cpu().numpy(), P.data)


def test_pattern_3d_matches_host_assembler(featlib):
    from featb200.assembly_gpu import q1_pattern_3d
    for level in (0, 1, 2, 4):
        rp, ci = q1_pattern_3d(level)
        A = AS.stiffness(level, 3)
        assert np.array_equal(rp, A.indptr.astype(np.uint64))
        assert np.array_equal(ci, A.indices.astype(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("level", [1, 3, 5])
def test_assembly_3d_matches_host(featlib, cuda, level):
    """The hexahedral Q1 Laplacian and the Gaussian load vector on the unit cube against the host
    assembler (pinned to the reference's assembly by test_assembly)."""
    torch = cuda
    from featb200.assembly_gpu import Q1Assembler3D
    gp = AS.gauss_params(70 + level, 3, width=(0.03, 0.12))
    vals, b = Q1Assembler3D(level).assemble(gp)
    torch.cuda.synchronize()
    A = AS.stiffness(level, 3)
    b_ref = AS.load_vector(level, lambda *xs: AS.gauss_eval(gp, *xs), 3)
    b_ref[AS.boundary_dofs(level, 3).astype(np.int64)] = 0.0
    v = vals.cpu().numpy()
    assert np.abs(v - A.data).max() <= TOL * np.abs(A.data).max()
    bb = b.cpu().numpy()
    assert np.abs(bb - b_ref).max() <= TOL * max(np.abs(b_ref).max(), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("level", [1, 2, 4])
def test_prolongation_3d_matches_host(featlib, cuda, level):
    from featb200.assembly_gpu import q1_prolongation_3d
    rp, ci, v = q1_prolongation_3d(level)
    P = AS.prolongation(level, 3)
    assert np.array_equal(rp.cpu().numpy(), P.indptr.astype(np.int64))
    assert np.array_equal(ci.cpu().numpy(), P.indices.astype(np.int64))
    assert np.array_equal(v.cpu().numpy(), P.data)


@pytest.mark.gpu
def test_device_assembled_3d_hierarchy_solves(featlib, cuda, oracle_lib):
    """A 3D level-5 hierarchy assembled entirely on the device (stiffness, load vector and
    prolongations; R = P^T) gives the solve of the host-assembled one."""
    from featb200.assembly_gpu import Q1Assembler3D, q1_prolongation_3d
    from helpers import rel_err
    import scipy.sparse as sp
    fb = featlib
    L = 5
    gp = AS.gauss_params(9, 3, width=(0.03, 0.12))
    host_levels, b_host = AS.poisson_hierarchy(L, 3, rhs="gauss", gauss=gp)
    levels = []
    b_dev = None
    for lv in range(L, 0, -1):
        asm = Q1Assembler3D(lv)
        vals, b = asm.assemble(gp if lv == L else None, rhs=(lv == L))
        n = asm.n
        A = sp.csr_matrix((vals.cpu().numpy(), asm.col_ind.astype(np.int64), asm.row_ptr.astype(np.int64)), shape=(n, n))
        d = {"matrix": fb.SparseMatrixCSR.from_scipy(A), "filter": fb.UnitFilter(AS.boundary_dofs(lv, 3))}
        if lv == L:
            b_dev = b.cpu().numpy()
        if lv > 1:
            rp, ci, v = q1_prolongation_3d(lv)
            nc = (2 ** (lv - 1) + 1) ** 3
            P = sp.csr_matrix((v.cpu().numpy(), ci.cpu().numpy(), rp.cpu().numpy()), shape=(n, nc))
            d["transfer"] = fb.Transfer(fb.SparseMatrixCSR.from_scipy(P), fb.SparseMatrixCSR.from_scipy(P.T.tocsr()))
        levels.append(d)
    assert rel_err(b_dev, b_host) <= 1e-12
    s_dev = fb.build_pcg_multigrid(levels)
    s_host = fb.build_pcg_multigrid(host_levels)
    x_dev, x_host = fb.DenseVector(b_dev.size), fb.DenseVector(b_host.size)
    assert fb.solve(s_dev, x_dev, fb.DenseVector(b_dev)) == fb.Status.success
    assert fb.solve(s_host, x_host, fb.DenseVector(b_host)) == fb.Status.success
    assert s_dev.get_num_iter() == s_host.get_num_iter()
    assert rel_err(x_dev.elements, x_host.elements) <= 1e-10

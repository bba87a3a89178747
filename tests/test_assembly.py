"""The product's problem generator against the reference's own assembly (golden fixtures), through
the vertex-coordinate map between the reference's hierarchical and the lexicographic numbering."""
import numpy as np
import pytest
import scipy.sparse as sp

from helpers import load_golden, lex_index


def _perm(coords, level):
    lex = lex_index(coords, level)
    n = lex.size
    return sp.csr_matrix((np.ones(n), (lex, np.arange(n))), shape=(n, n))


def _scipy(c):
    return sp.csr_matrix((c.val, c.col_ind.astype(np.int64), c.row_ptr.astype(np.int64)), shape=c.shape)


@pytest.mark.parametrize("name", ["c1_L5", "gauss2d_L5", "kappa2d_L4", "c3d_L3", "gauss3d_L3"])
def test_assembly_matches_reference(name):
    from featb200 import assembly as AS
    g = load_golden(name)
    raw = g["raw"]
    dim, L = g["dim"], g["level"]
    gauss = raw.get("gauss_params")
    field = None
    if "field_kx" in raw:
        field = (raw["field_kx"], raw["field_ky"], raw["field_xi"], raw["field_eta"], float(raw["field_s"][0]))
    levels, b = AS.poisson_hierarchy(L, dim, rhs="gauss" if gauss is not None else "sine", gauss=gauss, field=field)
    for i, ref in enumerate(g["levels"]):
        lv = ref["level"]
        Pm = _perm(ref["coords"], lv)
        A_ref = (Pm @ _scipy(ref["A"]) @ Pm.T).tocsr()
        A = levels[i]["matrix"].to_scipy()
        scale = np.abs(A_ref).max()
        assert abs(A_ref - A).max() <= 1e-13 * scale
        assert set(lex_index(ref["coords"], lv)[ref["filter_idx"].astype(np.int64)]) == \
            set(levels[i]["filter"].indices.astype(np.int64))
        if "P" in ref:
            Pc = _perm(g["levels"][i + 1]["coords"], lv - 1)
            P_ref = (Pm @ _scipy(ref["P"]) @ Pc.T).tocsr()
            assert abs(P_ref - levels[i]["transfer"].prol.to_scipy()).max() <= 1e-14
            R_ref = (Pc @ _scipy(ref["R"]) @ Pm.T).tocsr()
            assert abs(R_ref - levels[i]["transfer"].rest.to_scipy()).max() <= 1e-14
    lex = lex_index(g["levels"][0]["coords"], L)
    b_ref = np.zeros_like(b)
    b_ref[lex] = g["rhs"]
    assert np.abs(b - b_ref).max() <= 1e-13 * np.abs(b_ref).max()


def test_field_statistics():
    """The log-kappa field has zero mean and unit variance (over seeds and points)."""
    from featb200 import assembly as AS
    xs = np.linspace(0, 1, 33)
    vals = np.concatenate([AS.field_eval_grid(AS.field_params(s), xs, xs).ravel() for s in range(40)])
    assert abs(vals.mean()) < 0.1
    assert abs(vals.std() - 1.0) < 0.1


@pytest.mark.parametrize("dim,level", [(2, 5), (2, 7), (3, 3), (3, 5)])
def test_gauss_load_vector_by_direction(dim, level):
    """The Gaussian load vector formed by direction equals the cell-wise Gauss-rule assembly to
    rounding (the same integral, factored per coordinate)."""
    from featb200 import assembly as AS
    for seed in (0, 17, 63):
        g = AS.rhs64_params(seed, dim) if dim == 3 else AS.gauss_params(seed, 2)
        ref = AS.load_vector(level, lambda *xs: AS.gauss_eval(g, *xs), dim)
        b = AS.gauss_load_vector(level, g, dim)
        assert np.abs(b - ref).max() <= 1e-14 * np.abs(ref).max()

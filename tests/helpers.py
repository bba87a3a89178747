"""Shared test helpers: golden-fixture loading and numbering maps."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

CASES_2D = ["c1_L4", "c1_L5", "gauss2d_L5", "kappa2d_L4"]
CASES_3D = ["c3d_L3", "gauss3d_L3"]
CASES = CASES_2D + CASES_3D


def require_reference_binary():
    """Skip the calling test when the reference binary (oracle/_ref/feat_oracle, built from the
    reference's sources by oracle/Makefile) is absent; with FEATB200_REQUIRE_REF=1 in the
    environment its absence fails the test instead, so a run that expects the binary cannot pass on
    skipped pins."""
    import pytest
    import oracle as O
    if O.feat_available():
        return
    if os.environ.get("FEATB200_REQUIRE_REF") == "1":
        pytest.fail("reference binary oracle/_ref/feat_oracle not built (FEATB200_REQUIRE_REF=1)")
    pytest.skip("reference binary oracle/_ref/feat_oracle not built")


def load_golden(name):
    """A golden fixture as a dict: levels (finest first), rhs, sol, vcycle, iterates, defects, summary."""
    import oracle as O
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    g = {k: z[k] for k in z.files}
    summary = json.loads(bytes(g["summary_json"]).decode())
    out = {"summary": summary, "raw": g}
    if "level" not in summary:
        return out
    L, dim = summary["level"], summary["dim"]

    def csr(prefix):
        return O.Csr.of(g[prefix + "_row_ptr"], g[prefix + "_col_ind"], g[prefix + "_val"], g[prefix + "_shape"])

    levels = []
    for lv in range(L, 0, -1):
        d = {"A": csr(f"L{lv}_A"), "filter_idx": g[f"L{lv}_filter_idx"].astype(np.uint64),
             "filter_val": g[f"L{lv}_filter_val"], "coords": g[f"L{lv}_coords"].reshape(-1, dim), "level": lv}
        if lv > 1:
            d["P"] = csr(f"L{lv}_P")
            d["R"] = csr(f"L{lv}_R")
        levels.append(d)
    out.update(levels=levels, rhs=g["rhs"], sol=g["sol"], vcycle=g["vcycle"], defects=g["defects"],
               iterates=[g[f"iterate_{k}"] for k in range(1, summary["iters"] + 1)], dim=dim, level=L)
    return out


def lex_index(coords, level):
    """Reference (hierarchical) DOF -> lexicographic DOF of the same vertex."""
    N = 2 ** level
    ijk = np.rint(coords * N).astype(np.int64)
    idx = np.zeros(coords.shape[0], dtype=np.int64)
    for d in range(coords.shape[1] - 1, -1, -1):
        idx = idx * (N + 1) + ijk[:, d]
    return idx


def to_lafem_levels(levels):
    """Golden levels -> featb200 LAFEM containers (reference numbering, u64 indices)."""
    import featb200 as fb
    out = []
    for d in levels:
        A = d["A"]
        lv = {"matrix": fb.SparseMatrixCSR(A.row_ptr, A.col_ind, A.val, A.shape),
              "filter": fb.UnitFilter(d["filter_idx"], d["filter_val"])}
        if "P" in d:
            P, R = d["P"], d["R"]
            lv["transfer"] = fb.Transfer(fb.SparseMatrixCSR(P.row_ptr, P.col_ind, P.val, P.shape),
                                         fb.SparseMatrixCSR(R.row_ptr, R.col_ind, R.val, R.shape))
        out.append(lv)
    return out


def to_oracle_levels(lafem_levels):
    """featb200 LAFEM levels -> oracle level dicts."""
    import oracle as O
    out = []
    for lv in lafem_levels:
        m = lv["matrix"]
        d = {"A": O.Csr.of(m.row_ptr, m.col_ind, m.val, m.shape), "filter_idx": lv["filter"].indices,
             "filter_val": lv["filter"].values}
        if "transfer" in lv:
            P, R = lv["transfer"].prol, lv["transfer"].rest
            d["P"] = O.Csr.of(P.row_ptr, P.col_ind, P.val, P.shape)
            d["R"] = O.Csr.of(R.row_ptr, R.col_ind, R.val, R.shape)
        out.append(d)
    return out


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))

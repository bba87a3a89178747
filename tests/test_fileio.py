"""The reference's container file formats (featb200.fileio), pinned against the reference's own
readers and writers (oracle/_ref/feat_oracle io): a binary CSR matrix and dense vector written here
are read by the reference and written back byte for byte identically; its Matrix Market and
exponential ASCII output reads back here to the values' printed precision."""
import os

import numpy as np
import pytest

from helpers import require_reference_binary

from featb200 import assembly as AS
from featb200 import fileio
from featb200.lafem import DenseVector, SparseMatrixCSR


def _matrix():
    return SparseMatrixCSR.from_scipy(AS.stiffness(3, 2, None))


def test_binary_roundtrip_here(tmp_path):
    A = _matrix()
    p = str(tmp_path / "a.csr")
    A.write_out("csr", p)
    B = SparseMatrixCSR.read_from("csr", p)
    assert B.shape == A.shape
    assert np.array_equal(B.row_ptr, A.row_ptr) and np.array_equal(B.col_ind, A.col_ind)
    assert np.array_equal(B.val, A.val)
    v = DenseVector(np.random.default_rng(0).standard_normal(77))
    q = str(tmp_path / "v.dv")
    v.write_out("dv", q)
    assert np.array_equal(DenseVector.read_from("dv", q).elements, v.elements)
    with open(p, "rb") as f:
        head = np.frombuffer(f.read(88), dtype="<u8")
    assert head[0] == os.path.getsize(p) and head[1] == fileio.FM_CSR


def test_reference_reads_and_rewrites_identically(tmp_path, oracle_lib):
    O = oracle_lib
    require_reference_binary()
    A = _matrix()
    v = DenseVector(np.random.default_rng(1).standard_normal(A.rows()))
    p, q = str(tmp_path / "a.csr"), str(tmp_path / "v.dv")
    A.write_out("csr", p)
    v.write_out("dv", q)
    out = str(tmp_path / "rt")
    summ = O.feat_io(p, q, out)
    assert (summ["rows"], summ["columns"], summ["used_elements"], summ["size"]) == \
        (A.rows(), A.columns(), A.used_elements(), v.size())
    for mine, theirs in ((p, "rt.csr"), (q, "rt.dv")):
        with open(mine, "rb") as f1, open(os.path.join(out, theirs), "rb") as f2:
            assert f1.read() == f2.read(), theirs
    # the reference's ASCII output, read here, and ours, written here, agree
    M = SparseMatrixCSR.read_from("mtx", os.path.join(out, "rt_matrix.mtx"))
    assert np.array_equal(M.row_ptr, A.row_ptr) and np.array_equal(M.col_ind, A.col_ind)
    assert np.allclose(M.val, A.val, rtol=1e-6)
    mine = str(tmp_path / "mine.mtx")
    A.write_out("mtx", mine)
    with open(mine) as f1, open(os.path.join(out, "rt_matrix.mtx")) as f2:
        assert f1.read() == f2.read()
    for mode, name in (("mtx", "rt_vector.mtx"), ("exp", "rt_vector.exp")):
        w = DenseVector.read_from(mode, os.path.join(out, name))
        assert np.allclose(w.elements, v.elements, rtol=1e-6)
        mine = str(tmp_path / ("mine." + mode))
        v.write_out(mode, mine)
        with open(mine) as f1, open(os.path.join(out, name)) as f2:
            assert f1.read() == f2.read(), name


def test_rejects_wrong_mode(tmp_path):
    v = DenseVector(np.ones(5))
    q = str(tmp_path / "v.dv")
    v.write_out("dv", q)
    with pytest.raises(ValueError):
        SparseMatrixCSR.read_from("csr", q)
    with pytest.raises(ValueError):
        v.write_out("ell", q)
